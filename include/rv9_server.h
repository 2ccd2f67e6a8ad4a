/*
 * rv9_server.h — serving many VP9 streams on one GPU.
 *
 * No counterpart in the reference, whose Decoder serves one stream per
 * caller (src/decoder/mod.rs:150-216). This is the continuous-batching form:
 * an engine holds many live streams, each with its eight reference slots and
 * frame contexts resident on the device. A stream is admitted when the
 * engine's HBM budget can hold its reservation, and waits (pending) until
 * streams close otherwise. Decode requests (packets) are parsed on a pool of
 * host threads, and each stream's reconstruction runs on its own CUDA stream,
 * so requests of different streams overlap on the device as they arrive.
 * Every result is bit-identical to decoding the stream alone with
 * rv9_decode_all.
 *
 * Each completion reports the request's latency: from rv9_submit to the
 * moment its frames are in host memory.
 */
#ifndef RV9_SERVER_H
#define RV9_SERVER_H

#include <stddef.h>
#include <stdint.h>

#include "rv9.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rv9_engine rv9_engine;

/* An engine on `device` (-1: current) admitting streams within
 * `hbm_budget_bytes`, with `workers` host threads parsing (0: one per core).
 * NULL when no usable device is present (rv9_last_global_error says why).
 * Each stream's frames are reconstructed on its own CUDA stream. */
rv9_engine* rv9_engine_create(int device, uint64_t hbm_budget_bytes, uint32_t workers);
/* The same engine with the streams' reconstruction batched on the device:
 * the streams are split round-robin into `groups` groups (0: one), and each
 * group's launcher reconstructs the next parsed frame of every stream of the
 * group that has one together, one launch per stage (the stage kernels take
 * their work from all of those frames), on the group's CUDA stream. A
 * launcher keeps at most two steps queued on the device, so frames that
 * arrive while the GPU is busy join the next step. Results are bit-identical
 * to the plain engine's. */
rv9_engine* rv9_engine_create_batched(int device, uint64_t hbm_budget_bytes, uint32_t workers, uint32_t groups);
/* Closes every stream, waits for their submitted requests, then frees the
 * engine, with any completions not yet released. */
void rv9_engine_free(rv9_engine* eng);
/* Device parsing for the streams opened after this call (plain form only;
 * RV9_UNSUPPORTED for a batched engine). A worker that takes a stream with
 * two or more queued requests takes up to `window` of them (0: 8, at most
 * 64) and parses their frames on the GPU as one batch, as
 * rv9_decoder_set_device_parse does; a lone request is parsed on the host
 * as before (a batch takes as long as its longest tile column, hundreds of
 * milliseconds at 2160p), and so is any frame the device parser does not
 * take. At most `max_batches` batches are on the device at once (0: 32);
 * the engine adds that many workers, which sleep while their batch parses.
 * Each such stream keeps 2 x `window` output buffers and reserves room for
 * a batch's device records (rv9_engine_stream_reservation). A frame that
 * fails fails its request and the requests of the same batch after it.
 * `on` = 0 stops further batches; streams opened later reserve nothing
 * for them. Results are bit-identical to host parsing. */
rv9_status rv9_engine_set_device_parse(rv9_engine* eng, int on, uint32_t window, uint32_t max_batches);

/* The largest frame a stream will carry, which sizes its reservation. */
typedef struct rv9_stream_spec {
  uint32_t max_width, max_height;
  uint32_t bit_depth;   /* 8, 10 or 12 */
  uint32_t ss_x, ss_y;  /* chroma subsampling: 1,1 for 4:2:0; 0,0 for 4:4:4 */
} rv9_stream_spec;

/* Device bytes the engine reserves for a stream of this spec: its pooled
 * frames (eight slots and two in flight), record staging and scratch. Needs
 * no device. */
uint64_t rv9_stream_reservation(const rv9_stream_spec* spec);
/* The bytes a stream of this spec reserves in `eng`: rv9_stream_reservation
 * plus, when the engine parses on the device, the device parser's buffers
 * for a batch (rv9_engine_set_device_parse). */
uint64_t rv9_engine_stream_reservation(rv9_engine* eng, const rv9_stream_spec* spec);

/* Opens a stream; *id receives its handle. The stream is admitted at once
 * when the budget allows, else it is pending and its requests wait until
 * other streams close. RV9_UNSUPPORTED when the spec alone exceeds the
 * budget. */
rv9_status rv9_stream_open(rv9_engine* eng, const rv9_stream_spec* spec, int64_t* id);
/* Closes a stream once its submitted requests are done (a pending stream
 * is admitted in turn first); its reservation then returns to the budget. */
rv9_status rv9_stream_close(rv9_engine* eng, int64_t id);

/* Queues one packet (a frame or a superframe) for the stream. The packet is
 * copied; `tag` comes back in its completion. Requests of one stream complete
 * in submission order. */
rv9_status rv9_submit(rv9_engine* eng, int64_t id, const uint8_t* packet, size_t len, uint64_t tag);

typedef struct rv9_completion {
  int64_t stream;
  uint64_t tag;
  rv9_status status;    /* RV9_OK or the request's error */
  uint32_t n_frames;    /* shown frames in frames[] (at most 2) */
  double submit_ms;     /* submission time, ms since the engine was created */
  double latency_ms;    /* submission to frames in host memory */
  rv9_frame frames[2];  /* owned by the engine until rv9_completion_release */
  void* handle;
} rv9_completion;

/* Up to `cap` finished requests, in completion order; waits up to
 * `timeout_ms` for the first (0: no wait). Returns how many were written. */
size_t rv9_poll(rv9_engine* eng, rv9_completion* out, size_t cap, int timeout_ms);
/* Returns a completion's frame buffers to its stream. A stream holds four
 * output buffers (twice the window with device parsing), each one frame of
 * its largest size: requests wait while all are out. */
void rv9_completion_release(rv9_engine* eng, rv9_completion* c);

typedef struct rv9_engine_stats {
  uint64_t streams_open, streams_pending;
  uint64_t requests_submitted, requests_completed;
  uint64_t frames_decoded;
  uint64_t reserved_bytes, budget_bytes;
  uint64_t batched_steps, batched_frames; /* batched form: steps launched and frames in them */
  /* rv9_engine_set_device_parse: batches, the frames parsed on the device,
   * the workers' time waiting for their batches' parse on the device, and
   * their time on the batches in all (microseconds, summed over workers) */
  uint64_t device_parse_batches, device_parsed_frames;
  uint64_t device_parse_wait_us, device_parse_batch_us;
} rv9_engine_stats;
void rv9_engine_get_stats(rv9_engine* eng, rv9_engine_stats* out);

/* ---- Several GPUs of one node ----
 *
 * A cluster is a serving engine per device. Streams are independent and a
 * stream's frames chain through its own reference slots, so each stream is
 * placed whole on one device and stays there; devices exchange nothing (no
 * collective, no peer memory). A new stream goes to the device with the
 * fewest reserved bytes among those whose budget has room for its
 * reservation (rv9_stream_reservation), else to the least loaded device that
 * could ever hold it, where it waits pending. Stream ids are the cluster's;
 * completions of every device come back through rv9_cluster_poll. */
typedef struct rv9_cluster rv9_cluster;
/* Engines on devices[0..n) (each as rv9_engine_create(devices[i],
 * hbm_budget_per_device, workers_per_device)). NULL when any fails. */
rv9_cluster* rv9_cluster_create(const int* devices, size_t n, uint64_t hbm_budget_per_device,
                                uint32_t workers_per_device);
void rv9_cluster_free(rv9_cluster* c);
/* rv9_engine_set_device_parse on every device's engine (streams are then
 * placed by rv9_engine_stream_reservation). */
rv9_status rv9_cluster_set_device_parse(rv9_cluster* c, int on, uint32_t window, uint32_t max_batches);
/* Opens a stream on the device the placement rule picks; *device receives
 * that device's ordinal (may be NULL). RV9_UNSUPPORTED when no device's
 * budget could ever hold the stream. */
rv9_status rv9_cluster_stream_open(rv9_cluster* c, const rv9_stream_spec* spec, int64_t* id, int* device);
rv9_status rv9_cluster_stream_close(rv9_cluster* c, int64_t id);
rv9_status rv9_cluster_submit(rv9_cluster* c, int64_t id, const uint8_t* packet, size_t len, uint64_t tag);
/* Finished requests of all devices (completion.stream is the cluster's id);
 * waits up to timeout_ms for the first. */
size_t rv9_cluster_poll(rv9_cluster* c, rv9_completion* out, size_t cap, int timeout_ms);
void rv9_cluster_completion_release(rv9_cluster* c, rv9_completion* comp);
/* The engine statistics of the cluster's device_index-th device. */
void rv9_cluster_get_stats(rv9_cluster* c, int device_index, rv9_engine_stats* out);
/* The placement rule on its own (no device needed): the index of the device
 * a stream needing `need` bytes goes to, given each device's reserved bytes
 * and budget; -1 when none could ever hold it. */
int rv9_place_least_loaded(const uint64_t* load, const uint64_t* budget, size_t n, uint64_t need);

#ifdef __cplusplus
}
#endif

#endif /* RV9_SERVER_H */

/*
 * rv9.h — C ABI of the B200 VP9 decoder.
 *
 * The drop-in for rivet-vp9's decoder API (safewords/rivet-vp9):
 *
 *   rv9_decoder_new         replaces Decoder::new          src/decoder/mod.rs:150
 *   rv9_decoder_set_threads replaces Decoder::set_threads  src/decoder/mod.rs:174
 *   rv9_decoder_set_max_pixels  Decoder::set_max_pixels    src/decoder/mod.rs:186
 *   rv9_decoder_frames_decoded  Decoder::frames_decoded    src/decoder/mod.rs:214
 *   rv9_decode              replaces Decoder::decode       src/decoder/mod.rs:193
 *   rv9_decode_all          replaces Decoder::decode_all   src/decoder/mod.rs:198
 *   rv9_frame               is Frame (data, planes)        src/frame.rs:115-137
 *   rv9_status              is Error (Bitstream, Unsupported, InvalidInput)
 *                                                          src/lib.rs:66-81
 *
 * Parsing runs on the host (tile columns on threads); reconstruction —
 * dequantisation, inverse transforms, inter and intra prediction, compound
 * averaging and the loop filter — runs as CUDA kernels for sm_100a on the
 * decoder's GPU. There is no CPU reconstruction path: without a usable CUDA
 * device rv9_decoder_new returns NULL and rv9_last_global_error says why.
 * The host parser is built for x86-64-v3 (AVX2, BMI2, LZCNT); on a CPU
 * without it rv9_decoder_new likewise returns NULL.
 *
 * Frames come back in the reference's Frame layout: the visible Y, U, V
 * planes one after another, tightly packed (stride == width), one byte per
 * sample at 8 bits and little-endian uint16 above.
 */
#ifndef RV9_H
#define RV9_H

#include <stddef.h>
#include <stdint.h>

#include "rv9_records.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef enum rv9_status {
  RV9_OK = 0,
  RV9_BITSTREAM = 1,     /* malformed stream (Error::Bitstream) */
  RV9_UNSUPPORTED = 2,   /* valid but not supported, e.g. over max pixels */
  RV9_INVALID_INPUT = 3, /* unusable argument (Error::InvalidInput) */
  RV9_DEVICE = 4,        /* CUDA error or a device-side wait that timed out */
} rv9_status;

typedef enum rv9_chroma {
  RV9_YUV420 = 0,
  RV9_YUV422 = 1,
  RV9_YUV440 = 2,
  RV9_YUV444 = 3,
} rv9_chroma;

typedef struct rv9_plane {
  size_t offset;   /* byte offset of the plane in data */
  uint32_t width;  /* samples */
  uint32_t height;
} rv9_plane;

typedef struct rv9_frame {
  uint32_t width, height;      /* luma size */
  uint32_t bit_depth;          /* 8, 10, 12 */
  uint32_t chroma;             /* rv9_chroma */
  uint32_t color_space;        /* as coded, 0..7 (7 = sRGB) */
  uint32_t full_range;         /* color_range */
  uint32_t render_width, render_height;
  uint8_t* data;               /* owned by the frame: rv9_frame_release */
  size_t size;                 /* bytes in data */
  rv9_plane planes[3];         /* Y, U, V */
} rv9_frame;

typedef struct rv9_decoder rv9_decoder;

/* A decoder on CUDA device `device` (-1: the current device). NULL when no
 * usable device is present or the kernels fail to load. */
rv9_decoder* rv9_decoder_new(int device);
void rv9_decoder_free(rv9_decoder* dec);
/* Host parsing threads: 0 = one per core (default), 1 = the calling thread. */
void rv9_decoder_set_threads(rv9_decoder* dec, uint32_t threads);
/* Frames rv9_decode_packets and rv9_sequence_load parse at once (0: one per
 * two host threads, at most 8). Frames that depend on an earlier frame's
 * parse (adapted contexts, previous motion vectors) still wait for it; key
 * and error-resilient frames do not. Results are identical either way. */
void rv9_decoder_set_parse_depth(rv9_decoder* dec, uint32_t frames);
/* The number of host threads parsing uses (replaces Decoder::threads,
 * src/decoder/mod.rs:179-181): the set_threads value, or the core count when
 * it is 0. */
uint32_t rv9_decoder_threads(const rv9_decoder* dec);
/* Frames of more than `pixels` luma samples are refused (RV9_UNSUPPORTED). */
void rv9_decoder_set_max_pixels(rv9_decoder* dec, uint64_t pixels);

/* Device parsing (no counterpart in the reference, which parses tiles on its
 * host threads: src/decoder/block.rs:1776-1866). With `on`,
 * rv9_decode_packets and rv9_sequence_load parse the tiles of every frame
 * that allows it on the GPU, one thread per tile column and the columns of up
 * to `window_frames` frames (0: 64) at once, and build the reconstruction's
 * work lists there too; the host keeps the frame headers. A frame allows it
 * when nothing of it adapts probabilities from its symbol counts, reads or
 * writes segment ids, or needs the legacy 4:4:4 layout probe: key frames and
 * error-resilient or frame-parallel frames of streams without segmentation
 * (every frame of the generated streams but 4:2:2 / 4:4:4 key frames). The
 * other frames parse on the host, in order. Results are identical to host
 * parsing. rv9_sequence_load takes the device path only when every frame
 * allows it. With `on` = RV9_DEVICE_PARSE_SHARED, rv9_decode_packets splits
 * each batch whose frames are all independent of one another (key frames
 * and error-resilient frames) between the host, which parses its first part
 * frame-parallel on its threads, and the device, which parses the rest
 * meanwhile; the split follows the two sides' measured times, so that both
 * end together. */
#define RV9_DEVICE_PARSE_SHARED 2
rv9_status rv9_decoder_set_device_parse(rv9_decoder* dec, int on, uint32_t window_frames);
/* Frames the device parser took, its boolean decodes, and the device time
 * of its batches (tile parse and work lists, CUDA events on its stream). */
void rv9_decoder_device_parse_stats(const rv9_decoder* dec, uint64_t* frames, uint64_t* bools, double* device_ms);

/* Failure detection (no counterpart in the reference, whose waits are host
 * threads joining; its abort model is src/decoder/loopfilter.rs:300-338).
 * Every device-side wait of the intra and loop-filter wavefronts is bounded:
 * after `polls` polls of an unready neighbour the kernel records a code in
 * the frame's error word, the other jobs of the frame give up as they next
 * wait, and the call that synchronises returns RV9_DEVICE. The decoder's
 * device state is then reset (cell maps, tickets) and stays usable; its
 * reference slots hold what the failed frames left, as after any error.
 * 0 restores the default (about a second of polling). */
void rv9_decoder_set_wait_limit(rv9_decoder* dec, uint32_t polls);
/* Failure injection for tests: bit 0 leaves the first intra job of every
 * frame untaken, bit 1 the first loop-filter row, so that the jobs that
 * depend on it wait until the wait limit runs out. Nothing faults and every
 * wait ends. 0 (the default) turns it off. */
void rv9_decoder_set_test_fault(rv9_decoder* dec, uint32_t mask);
uint64_t rv9_decoder_frames_decoded(const rv9_decoder* dec);
/* Message of the decoder's last error (valid until the next call). */
const char* rv9_last_error(const rv9_decoder* dec);
/* Why the last rv9_decoder_new failed. */
const char* rv9_last_global_error(void);

/* Decodes one packet (a frame or a superframe). Shown frames go to out[0..],
 * at most `cap`; *n_out receives how many the packet showed. */
rv9_status rv9_decode_all(rv9_decoder* dec, const uint8_t* packet, size_t len,
                          rv9_frame* out, size_t cap, size_t* n_out);
/* Decodes one packet; the last frame it shows goes to *out and *shown = 1. */
rv9_status rv9_decode(rv9_decoder* dec, const uint8_t* packet, size_t len,
                      rv9_frame* out, int* shown);
/* Frees a frame's data (from rv9_decode / rv9_decode_all). */
void rv9_frame_release(rv9_frame* frame);

/* Decodes `n` packets in order with host parsing overlapped with device
 * reconstruction, writing every shown frame's packed samples one after
 * another into `out` (`cap` bytes). *n_frames and *bytes receive the count
 * and size written. Frame geometry is that of rv9_decode_all's frames. */
rv9_status rv9_decode_packets(rv9_decoder* dec, const uint8_t* const* packets,
                              const size_t* lens, size_t n, uint8_t* out, size_t cap,
                              size_t* n_frames, size_t* bytes);

/* Timing of the device work since the last reset: reconstruction kernel
 * time (CUDA events on the decoder's stream), frames reconstructed, and the
 * algorithmic bytes of those frames (records read, reference samples
 * predicted from, samples written; 1 byte per sample at 8 bits, 2 above). */
typedef struct rv9_stats {
  double device_ms;
  double parse_ms;
  uint64_t frames;
  uint64_t algorithmic_bytes;
  uint64_t kernel_launches;
} rv9_stats;
void rv9_decoder_stats(rv9_decoder* dec, rv9_stats* out, int reset);

/* ---- Device-resident replay (the reconstruction engine on its own) ----
 *
 * A sequence is a stream's packets parsed on the host, with their records
 * and work lists copied to device memory once; rv9_sequence_run then
 * reconstructs every frame from those records (all kernels, no host work,
 * no copies), starting from empty reference slots. This measures the
 * reconstruction path with its inputs resident in HBM. */
typedef struct rv9_sequence rv9_sequence;
rv9_status rv9_sequence_load(rv9_decoder* dec, const uint8_t* const* packets, const size_t* lens, size_t n,
                             rv9_sequence** out);
/* Flags of rv9_sequence_run / rv9_sequences_run. */
#define RV9_RUN_PER_KERNEL 1 /* bracket each launch with events for rv9_kernel_stats */
#define RV9_RUN_GRAPH 2      /* replay the run as a CUDA graph, captured on first use
                                (after one ordinary run); per-kernel timing is off */
/* Reconstructs the sequence; *device_ms receives the CUDA-event time of the
 * run on the decoder's stream. */
rv9_status rv9_sequence_run(rv9_decoder* dec, rv9_sequence* seq, int flags, double* device_ms);
/* rv9_sequence_run without allocating. No counterpart in the reference
 * (whose decoder has no device and no replay): this entry point exists for
 * callers that must not allocate device memory while they decode — a
 * serving loop whose HBM is already reserved by its admission budget (a
 * cudaMalloc there can fail or take memory another stream was promised), or
 * a latency-bound loop that cannot take the device-wide synchronisation
 * cudaMalloc and cudaFree imply.
 *
 * It reconstructs the sequence exactly as rv9_sequence_run does (per_kernel
 * off), with two differences. The wavefront scratch (tickets, error word,
 * superblock done flags, per-8x8 loop-filter records) is a fixed static
 * device array of 1 MiB, not an allocation: a sequence with a frame needing
 * more (256 bytes + 4 per 64x64 superblock, rounded up to 256, + 4 per 8x8
 * block; e.g. 4096x2304 needs 0.57 MiB, 8192x4096 does not fit) is refused
 * with RV9_INVALID_INPUT before anything runs. And every frame buffer comes
 * from the decoder's pool: when the pool lacks a frame the run would take
 * (call rv9_sequence_run on the sequence once first to fill it), the call
 * returns RV9_INVALID_INPUT before anything runs.
 *
 * The first call on a device looks the array's address up with
 * cudaGetSymbolAddress; make that first call before any CUDA stream capture
 * begins. The address is kept for the life of the process, so the device's
 * primary context must stay alive (no cudaDeviceReset between calls). The
 * tickets and done flags must start at zero for each frame: the call clears
 * them with cudaMemsetAsync on the decoder's stream before each frame. The
 * error word is cleared once, before the call's first frame, so a wait that
 * gave up in any frame of the run is reported (RV9_DEVICE). The loop-filter
 * records are rewritten whole by each frame. All
 * calls on one device share the one array, so calls that overlap in time on
 * the same device (two decoders, or two host threads) race on it and must be
 * serialised by the caller. */
rv9_status rv9_sequence_run_noalloc(rv9_decoder* dec, rv9_sequence* seq, double* device_ms);
/* Reconstructs seqs[i] on decs[i] for all i at once: every decoder (all
 * distinct, on one device) runs its sequence on its own CUDA stream, frames
 * issued round-robin, so independent streams' kernels overlap on the GPU.
 * *device_ms receives the CUDA-event time from the common start to the last
 * stream's end. A multi-stream throughput form with no reference counterpart. */
rv9_status rv9_sequences_run(rv9_decoder* const* decs, rv9_sequence* const* seqs, size_t n, int flags,
                             double* device_ms);
/* The same reconstruction with one launch per stage for all sequences' next
 * frames: frame i of every sequence is in step i's launches (preparation,
 * inter prediction, residuals, the intra wavefront, the loop-filter
 * wavefront), 8-bit and deeper frames in separate launches. Each stage's
 * kernel walks a work list drawn from all of the step's frames; the
 * wavefront stages hand out each frame's rows from that frame's own tickets.
 * The decoders are split round-robin into `groups` groups (1 up to n), each
 * group's launches on its own CUDA stream, so that one group's loop filter
 * can run beside another's prediction. Frames are bit-identical to
 * rv9_sequences_run's. A multi-stream form with no reference counterpart. */
rv9_status rv9_sequences_run_batched(rv9_decoder* const* decs, rv9_sequence* const* seqs, size_t n, int groups,
                                     double* device_ms);
uint32_t rv9_sequence_frames(const rv9_sequence* seq);
uint64_t rv9_sequence_luma_samples(const rv9_sequence* seq);     /* visible luma of shown frames */
uint64_t rv9_sequence_algorithmic_bytes(const rv9_sequence* seq); /* per run */
uint64_t rv9_sequence_record_bytes(const rv9_sequence* seq);      /* device bytes held */
void rv9_sequence_free(rv9_decoder* dec, rv9_sequence* seq);
/* A device copy of `src` (its records and work lists) held by `dec`, without
 * parsing again: many decoders replaying the same content each read their
 * own records. */
rv9_status rv9_sequence_clone(rv9_decoder* dec, const rv9_sequence* src, rv9_sequence** out);

/* Autotuner (no counterpart in the reference): times the sequence with each
 * candidate launch shape, namely the intra wavefront's grain (its grid: a
 * quarter to four CTAs per SM), the CTA size of the large-region inter
 * kernel (64, 128 or 256 threads), and whether the small-region inter kernel
 * runs on a side stream beside it. It keeps the fastest for the geometry of
 * the sequence's frames, and this decoder then uses it for every frame of
 * that geometry. Results are bit-identical under every shape. */
typedef struct rv9_tune_result {
  int32_t intra_ctas_per_sm_x4; /* chosen grain: quarter CTAs per SM */
  int32_t inter_threads;        /* chosen CTA size */
  double best_ms;               /* the sequence's time with them */
  double default_ms;            /* ... and with the defaults (4, 128, fork on) */
  int32_t inter_fork;           /* 1: small inter regions on a side stream beside the large ones */
} rv9_tune_result;
rv9_status rv9_decoder_autotune(rv9_decoder* dec, rv9_sequence* seq, rv9_tune_result* out);
/* The same for sequences reconstructed together (rv9_sequences_run): each
 * candidate shape is applied to every decoder and the batch is timed as a
 * whole; every decoder keeps the fastest for its sequence's geometries. The
 * best shape for one stream alone (a wavefront grid sized to the whole GPU)
 * can crowd the other streams out when many share the device. Times are the
 * batch's; graphs captured before tuning keep their old shapes. */
rv9_status rv9_sequences_autotune(rv9_decoder* const* decs, rv9_sequence* const* seqs, size_t n,
                                  rv9_tune_result* out);
/* The autotuner for rv9_sequences_run_batched: times the batch with 1, 2, 4
 * and 8 groups (at most n) under each intra wavefront grain, keeps the
 * fastest grain on decs[0] (used by batched runs whose first decoder it is)
 * and returns it in *out with the fastest number of groups in *groups.
 * out->default_ms is one group with the default grain. */
rv9_status rv9_sequences_autotune_batched(rv9_decoder* const* decs, rv9_sequence* const* seqs, size_t n,
                                          int32_t* groups, rv9_tune_result* out);

/* A frame sink, for checking replays frame by frame (no counterpart in the
 * reference): while it is set, every frame the decoder shows — in
 * rv9_sequence_run (not graph replays), rv9_sequence_run_noalloc,
 * rv9_sequences_run, rv9_sequences_run_batched and the decode calls — is
 * copied, packed like rv9_frame data, into `buf` one after another. `buf`
 * may be host memory (pinned or not) or device memory of the decoder's
 * device; the copies are complete when the call that showed the frames
 * returns. Frames that would overrun `cap` bytes are not copied but counted.
 * buf == NULL turns the sink off; each set starts it empty. */
void rv9_decoder_set_frame_sink(rv9_decoder* dec, uint8_t* buf, size_t cap);
/* Frames and bytes the sink holds, and frames dropped for want of room. */
void rv9_decoder_frame_sink_state(const rv9_decoder* dec, uint64_t* frames, size_t* bytes, uint64_t* dropped);

/* On-device frame digests (no counterpart in the reference, whose tests hash
 * Frame::packed() on the host, tests/common/mod.rs:151): while on, the MD5 of
 * every frame the decoder shows — of the bytes rv9_frame data would hold — is
 * computed on the GPU from the frame's device planes, for up to `cap_frames`
 * frames, and nothing but the 16-byte digests is read back. Shown frames of
 * the same calls as the frame sink's are covered. 0 turns it off; each call
 * starts the list empty. The digest of a frame is a serial chain of 64-byte
 * blocks (about 40 ms for a 1080p 8-bit frame on one warp), so this is a
 * checking aid, not a throughput path. */
rv9_status rv9_decoder_set_frame_digests(rv9_decoder* dec, size_t cap_frames);
/* Copies the digests computed so far (16 bytes each, in show order) into
 * `out` (room for `cap` of them); returns how many there are. Call after the
 * decode or run call that showed the frames has returned. */
size_t rv9_decoder_frame_digests(rv9_decoder* dec, uint8_t* out, size_t cap);

/* The frame in reference slot `slot` (0..7), packed like rv9_frame data. */
rv9_status rv9_decoder_download_slot(rv9_decoder* dec, int slot, uint8_t* out, size_t cap, size_t* bytes);

typedef struct rv9_kernel_stat {
  char name[24];
  uint64_t launches;
  double ms;                  /* summed CUDA-event durations */
  uint64_t algorithmic_bytes; /* summed over the launches */
} rv9_kernel_stat;
/* Per-kernel timing of the per_kernel sequence runs; returns the count. */
size_t rv9_kernel_stats(rv9_decoder* dec, rv9_kernel_stat* out, size_t cap, int reset);
/* Which kernels per_kernel runs bracket with events: bit i for the i-th entry
 * of rv9_kernel_stats (default: all). Each pair of events costs the chain a
 * little time, so a run timed for one kernel's figures brackets only it. */
void rv9_decoder_set_event_mask(rv9_decoder* dec, uint32_t mask);

#ifdef __cplusplus
}
#endif

#endif /* RV9_H */

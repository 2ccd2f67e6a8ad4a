// The reconstruction engine: device frame buffers, the eight reference slots,
// and the per-frame launch of the reconstruction kernels from a parsed
// frame's records.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "../host/parser.h"
#include "engine_types.h"

namespace rv9g {

// Kernels of a frame, for per-kernel timing and byte accounting.
enum KernelId { K_PREP = 0, K_INTER, K_INTER_RES, K_INTRA, K_LF, K_COUNT };
extern const char* const kKernelNames[K_COUNT];

// Called around each launch when timing per kernel: phase 0 before, 1 after.
typedef void (*LaunchHook)(void* ctx, int kernel, int phase);

// Launch shapes the autotuner chooses per frame geometry: the intra
// wavefront's grain (its grid, in quarter CTAs per SM) and the CTA size of
// the large-region inter kernel.
struct TuneParams {
  int intra_ctas_per_sm_x4 = 4;  // 1, 2, 4, 8, 16: a quarter to four CTAs per SM
  int inter_threads = 128;       // 64, 128 or 256
  bool inter_fork = true;        // small inter regions on the side stream, beside the large ones
};
// A side stream of the engine's, and the events that fork work onto it and
// join it back (both launches of a frame then run side by side).
struct LaunchAux {
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};
cudaError_t launch_frame(const KFrame& k, int n_blocks, cudaStream_t s, int n_sm, int* launches, LaunchHook hook,
                         void* hook_ctx, const TuneParams& tune = TuneParams(), const LaunchAux* aux = nullptr);
cudaError_t upload_filters(const int16_t* f);

// On-device MD5 of frames (k_md5_frames): one job per frame, its packed
// planes read from the strided device planes, the 16-byte digest written to
// `out` (device memory). At most kMd5JobsPerLaunch jobs per launch.
struct Md5Job {
  const uint8_t* plane[3];
  int64_t stride[3];       // bytes
  uint32_t row_bytes[3];   // packed row: width x bytes per sample
  uint32_t rows[3];
  uint8_t* out;
};
constexpr int kMd5JobsPerLaunch = 32;
struct Md5Jobs {
  Md5Job job[kMd5JobsPerLaunch];
};
cudaError_t upload_md5_table();
cudaError_t launch_md5(const Md5Jobs& jobs, int n, cudaStream_t s);

// Per-device kernel set-up: the shared-memory opt-ins of the wavefront
// kernels and the batched launches' occupancy on that device. Once per
// device (thread-safe), with `device` current; Engine::init calls it.
struct DeviceKernels {
  std::atomic<bool> ready{false};
  int intra_batch_per_sm[2] = {1, 1};  // [8-bit, deeper]
  int lf_batch_per_sm[2] = {1, 1};
};
cudaError_t kernels_init_device(int device);
const DeviceKernels& device_kernels(int device);

// Batched launches: one launch per stage for frames of many streams (no
// frame of a batch may depend on another), all 8-bit or all above 8 bits.
// The batch's tables (the frames' KFrames, launch splits and CTA prefixes)
// are filled on the host by batch_fill into batch_table_bytes(n) bytes,
// copied to the device as they are, and launched from there.
struct BatchTotals {
  uint32_t ctas[4];     // preparation, small inter, large inter, residual
  uint32_t intra_jobs;  // over all frames
  uint32_t intra_ctas;  // the intra wavefront CTAs the frames would take each alone (with `tune`)
  uint32_t lf_rows;     // superblock rows of the frames with the loop filter on
};
size_t batch_table_bytes(int n);
void batch_fill(const KFrame* ks, const int* n_blocks, int n, uint8_t* host, BatchTotals* tot, int n_sm,
                const TuneParams& tune);
cudaError_t launch_batch(const uint8_t* dev, int n, const BatchTotals& tot, bool high, cudaStream_t s, int n_sm,
                         const TuneParams& tune, int* launches);

// The fixed wavefront scratch: a static device array of this many bytes.
// Layout: [0, 256) counters (the intra ticket, the loop-filter ticket, the
// error word), then the superblock done flags (4 bytes each, 256-byte
// aligned extent), then the per-8x8 loop-filter records (4 bytes each).
constexpr size_t kFixedScratchBytes = (size_t)1 << 20;
size_t fixed_scratch_need(uint32_t mi_cols, uint32_t mi_rows, uint32_t sb64_cols, uint32_t sb64_rows);
// Its device address on `device` (which must be current); the first call for
// a device looks it up with cudaGetSymbolAddress.
cudaError_t fixed_scratch_address(int device, void** ptr);

// A decoded frame in device memory: three SB-aligned planes of 1 byte per
// sample at 8 bits, 2 above, and the intra cell map.
struct DevFrame {
  uint32_t width = 0, height = 0, ss_x = 1, ss_y = 1, bit_depth = 8;
  uint32_t aw = 0, ah = 0;  // SB-aligned luma size
  void* base = nullptr;     // one allocation
  size_t bytes = 0;
  void* planes[3] = {nullptr, nullptr, nullptr};
  int32_t stride[3] = {0, 0, 0};   // samples
  int32_t pheight[3] = {0, 0, 0};  // SB-aligned rows
  uint8_t* cells[3] = {nullptr, nullptr, nullptr};
  int32_t cell_stride[3] = {0, 0, 0};
  int refs = 0;  // reference slots holding it
  int sim_refs = 0;  // scratch count of Engine::pool_covers
  uint8_t color_space = 1, color_range = 0;
  uint32_t render_w = 0, render_h = 0;
  size_t bps() const { return bit_depth > 8 ? 2 : 1; }
};

// One frame's work, staged in a byte buffer (host, then device): the records
// and the work lists built from them, at the given offsets.
struct FrameWork {
  rv9_frame_desc desc;
  bool show_existing = false, show_frame = false;
  int show_slot = 0;
  uint8_t refresh_mask = 0;
  int ref_slot[3] = {0, 0, 0};
  uint32_t n_blocks = 0, n_toks = 0, n_coefs = 0, n_units = 0, n_units_small = 0, n_res = 0, n_intra = 0,
           n_intra_jobs = 0;
  size_t o_blocks = 0, o_toks = 0, o_coefs = 0, o_units = 0, o_res = 0, o_intra = 0, o_intra_jobs = 0, bytes = 0;
  uint32_t n_res_by_size[4] = {0, 0, 0, 0};
  uint64_t kbytes[K_COUNT] = {0};  // algorithmic bytes per kernel
  uint64_t total_bytes = 0;        // algorithmic bytes of the frame
};

// Parsed frames resident in device memory, for repeated reconstruction.
struct DevFrame;
struct Sequence {
  std::vector<FrameWork> frames;
  uint8_t* d_data = nullptr;
  size_t bytes = 0;
  uint64_t luma_samples = 0;  // visible, shown frames
  // The whole run captured as a CUDA graph (Engine::sequence_graph), with
  // the launches it holds and the reference slots it leaves.
  mutable cudaGraphExec_t graph = nullptr;
  mutable uint64_t graph_launches = 0;
  mutable DevFrame* graph_slots[8] = {nullptr};
};

struct KernelStat {
  uint64_t launches = 0;
  double ms = 0;
  uint64_t bytes = 0;
};

class Engine {
 public:
  Engine() = default;
  ~Engine();
  // side_stream: a second CUDA stream that the large inter units of a frame
  // run on beside its small ones. Without it every launch of the engine is
  // on its one CUDA stream, which is what many engines on one device want:
  // the device has a fixed number of hardware queues, and CUDA streams
  // beyond them share queues, where one stream's long kernel holds up the
  // other's work.
  bool init(int device, std::string* err, bool side_stream = true);
  // Reconstructs a parsed frame (or handles show_existing); the frame to show
  // (or null) stays valid until the next call. Work is queued; errors of the
  // device waits surface at the next sync().
  rv9::Status recon(const rv9::ParsedFrame& pf, DevFrame** shown, std::string* err);
  // Reconstructs a frame whose records and work lists are already in device
  // memory at d_base (the device parser's output, complete before this
  // call), like recon().
  rv9::Status recon_resident(const FrameWork& fw, const uint8_t* d_base, DevFrame** shown, std::string* err) {
    return run_frame(fw, d_base, false, shown, err);
  }
  // Copies the visible planes of `f`, packed (the reference Frame layout),
  // into host memory `dst` on the engine's stream (queued).
  rv9::Status download_async(DevFrame* f, uint8_t* dst, std::string* err);
  rv9::Status sync(std::string* err);
  static size_t packed_bytes(const DevFrame* f);

  // Tries the launch shapes of TuneParams on `seq` (a few runs each), keeps
  // the fastest for the geometry of its frames and returns it with its time
  // and that of the defaults.
  rv9::Status autotune(const Sequence& seq, TuneParams* best, float* best_ms, float* default_ms, std::string* err);
  // Device-resident sequences.
  rv9::Status sequence_load(const std::vector<rv9::ParsedFrame>& frames, Sequence* seq, std::string* err);
  // Reconstructs every frame of `seq` from scratch (empty slots first);
  // returns the CUDA-event time of the whole run.
  rv9::Status sequence_run(const Sequence& seq, bool per_kernel, float* ms, std::string* err);
  // Captures `seq`'s run as a CUDA graph once (after one ordinary run, which
  // fills the frame pool and the scratch so that the capture allocates
  // nothing), then replays it: the steady state without per-launch host
  // work. The graph clears the loop filter's progress words before and
  // after the frames, so the epochs baked into it can repeat.
  rv9::Status sequence_graph(const Sequence& seq, std::string* err);
  rv9::Status sequence_replay(const Sequence& seq, float* ms, std::string* err);
  // Reconstructs several sequences at once, one per engine (all engines
  // distinct, on one device), each on its engine's own CUDA stream with
  // frames issued round-robin, so that the streams' kernels overlap on the
  // device. *ms is the CUDA-event time from the first launch to the last
  // completion, on engines[0]'s stream.
  static rv9::Status run_concurrent(Engine* const* engines, const Sequence* const* seqs, size_t n,
                                    bool per_kernel, float* ms, std::string* err, bool graphs = false);
  // Reconstructs several sequences at once (one per engine, all distinct, on
  // one device) with one launch per stage for the next frames of all of
  // them: frame i of every sequence goes in step i's launches, those of
  // 8-bit and of deeper sequences apart. The engines are split round-robin
  // into `groups` groups, each group's launches on its own CUDA stream (the
  // stream of its first engine), so that one group's loop filter can overlap
  // another's prediction. *ms is the CUDA-event time from the first launch
  // to the last completion.
  static rv9::Status run_batched(Engine* const* engines, const Sequence* const* seqs, size_t n, int groups,
                                 float* ms, std::string* err);
  // One launch per stage for one frame of each of engines[0..n) (all
  // distinct, on one device, frames independent of one another) on stream
  // s: each frame's records are at bases[q] in device memory (ordered before
  // on s). Frames are prepared, the batch tables filled at h_tables (pinned)
  // and copied to d_tables (at least step_table_bytes(n) bytes each, not in
  // use by earlier launches still running), the stages launched, the frames
  // committed to their engines' slots and each engine's error word queued
  // for copying back. shown[q] receives frame q's shown frame (or null); its
  // pixels are final in stream order on s.
  static rv9::Status launch_step(Engine* const* engines, const FrameWork* const* fws, const uint8_t* const* bases,
                                 size_t n, cudaStream_t s, const TuneParams& tune, uint8_t* h_tables,
                                 uint8_t* d_tables, size_t* table_bytes, DevFrame** shown, int* launches,
                                 std::string* err);
  static size_t step_table_bytes(size_t n);
  // The host side of recon() without the launches: the frame's work lists
  // built into this engine's pinned staging and copied to its device staging
  // on stream s (*d_base: their device address; null for a shown existing
  // frame). At most two frames staged this way may await their launches.
  rv9::Status stage(const rv9::ParsedFrame& pf, cudaStream_t s, FrameWork* fw, const uint8_t** d_base,
                    std::string* err);
  // Copies the visible planes of `f`, packed, to `dst` (host or device
  // memory) on stream `stream` (queued).
  rv9::Status download_on(DevFrame* f, uint8_t* dst, cudaStream_t stream, std::string* err);
  // The autotuner for run_batched: times the batch with each number of
  // groups (1, 2, 4, 8, at most n) and each intra wavefront grain, and keeps
  // the fastest grain on engines[0], which run_batched then uses for batches
  // led by it. *groups receives the fastest number of groups.
  static rv9::Status autotune_batched(Engine* const* engines, const Sequence* const* seqs, size_t n, int* groups,
                                      TuneParams* best, float* best_ms, float* default_ms, std::string* err);
  // The autotuner for sequences reconstructed together: times run_concurrent
  // with each candidate shape applied to every engine, and gives each engine
  // the fastest for its sequence's geometries. Shapes that suit one stream
  // alone (the whole GPU for one wavefront) can crowd the others out when
  // many streams share the device.
  static rv9::Status autotune_concurrent(Engine* const* engines, const Sequence* const* seqs, size_t n,
                                         TuneParams* best, float* best_ms, float* default_ms, std::string* err);
  int device() const { return device_; }
  // Polls before a wavefront wait gives up (0: the default, about a second
  // of polling), and failure injection for tests (KFrame::test_skip; 0 in
  // normal use). Both apply to frames launched after the call.
  void set_wait_limit(uint32_t polls) { wait_limit_ = polls ? (int32_t)std::min<uint32_t>(polls, 1u << 30) : kDefaultWaitLimit; }
  void set_test_skip(uint32_t mask) { test_skip_ = mask & 3; }
  // The device error word as last copied back (nonzero after a wavefront
  // wait gave up; sync() reports and clears it).
  int32_t error_word() const { return h_error_ ? *(volatile int32_t*)(h_error_ + 1) : 0; }
  // Device bytes one decoder of this geometry holds with `n_frames` pooled
  // frames and record staging of `stage_bytes` (per buffer, two buffers).
  static size_t footprint(uint32_t width, uint32_t height, uint32_t ss_x, uint32_t ss_y, uint32_t bit_depth,
                          int n_frames, size_t stage_bytes);
  // Allocates up front what decoding frames of this geometry takes: pooled
  // frames, record staging, loop-filter and wavefront scratch. Decoding such
  // frames then allocates nothing more.
  rv9::Status reserve(uint32_t width, uint32_t height, uint32_t ss_x, uint32_t ss_y, uint32_t bit_depth,
                      int n_frames, size_t stage_bytes, std::string* err);
  // Like sequence_run (per_kernel off), allocating nothing: the wavefront
  // scratch is the fixed static array, and every frame comes from the pool.
  // Fails before any launch when a frame of the sequence needs more scratch
  // than the array holds, or the pool lacks a frame the run would take.
  rv9::Status sequence_run_fixed(const Sequence& seq, float* ms, std::string* err);
  void sequence_free(Sequence* seq);
  // A device copy of `src` on this engine's device.
  rv9::Status sequence_clone(const Sequence& src, Sequence* seq, std::string* err);
  DevFrame* slot(int i) const { return slots_[i]; }
  // A frame sink: while it is set, every frame the engine shows (sequence
  // runs, concurrent and batched runs, the fixed-scratch run and recon();
  // not graph replays) is copied, packed like rv9_frame data, to `buf`, one
  // after another, queued on the stream of the frame's launches. `cap`
  // bytes; frames that would not fit are counted in sink_dropped and not
  // copied. Null turns it off. For checking what a run computed, frame by
  // frame.
  void set_sink(uint8_t* buf, size_t cap) {
    sink_ = buf;
    sink_cap_ = cap;
    sink_used_ = 0;
    sink_frames_ = 0;
    sink_dropped_ = 0;
  }
  size_t sink_used() const { return sink_used_; }
  // On-device digests: while on (cap > 0), the MD5 of every frame the
  // engine shows (as the sink would copy it) is computed on the GPU into a
  // device array of `cap` entries; digests() copies them out once the run
  // that showed them has returned.
  rv9::Status set_digests(size_t cap, std::string* err);
  size_t digests(uint8_t* out, size_t cap) const;
  uint64_t sink_frames() const { return sink_frames_; }
  uint64_t sink_dropped() const { return sink_dropped_; }

  // Stats.
  double device_ms = 0;
  uint64_t frames = 0, alg_bytes = 0, launches = 0;
  KernelStat kstats[K_COUNT];
  uint32_t event_mask = ~0u;  // kernels that per_kernel runs bracket with events
  cudaStream_t stream() const { return stream_; }

 private:
  // A frame of d's geometry from the pool, or a new one zeroed on `stream`.
  DevFrame* alloc_frame(const rv9_frame_desc& d, cudaStream_t stream);
  // Room for a frame's `n` staged bytes; *base receives their offset in the
  // buffer that the frame's offsets refer to. nullptr when it can't be had.
  using StageReserve = std::function<uint8_t*(size_t n, size_t* base)>;
  bool build_work(const rv9::ParsedFrame& pf, FrameWork* fw, const StageReserve& reserve);
  rv9::Status run_frame(const FrameWork& fw, const uint8_t* d_base, bool per_kernel, DevFrame** shown,
                        std::string* err);
  // The host side of a frame's reconstruction: its frame from the pool, the
  // scratch it uses (clears queued on `stream`) and the kernels' view of it
  // in *k. *cur is null for a shown existing frame. commit_frame then
  // updates the reference slots once the frame's launches are queued.
  rv9::Status prepare_frame(const FrameWork& fw, const uint8_t* d_base, cudaStream_t stream, KFrame* k,
                            DevFrame** cur, std::string* err);
  void commit_frame(const FrameWork& fw, DevFrame* cur, DevFrame** shown);
  // The shown frame's copy into the sink and its digest, when they are on
  // (queued on `stream`). With `jobs`, the digest joins those jobs (the
  // caller launches them); without, it is launched at once.
  rv9::Status sink_frame(DevFrame* shown, cudaStream_t stream, std::string* err, Md5Jobs* jobs = nullptr,
                         int* n_jobs = nullptr);
  // Loop-filter records and progress words for every frame of `seq`, so
  // that no frame of a run reallocates them.
  rv9::Status reserve_scratch(const Sequence& seq, std::string* err);
  void reset_slots();
  bool pool_covers(const Sequence& seq);
  static uint64_t geometry_key(const rv9_frame_desc& d) {
    return (uint64_t)d.sb64_cols | (uint64_t)d.sb64_rows << 16 | (uint64_t)d.bit_depth << 32 |
           (uint64_t)d.ss_x << 40 | (uint64_t)d.ss_y << 41;
  }
  std::map<uint64_t, TuneParams> tuned_;  // by frame geometry
  const TuneParams* tune_override_ = nullptr;
  static void hook(void* ctx, int kernel, int phase);
  void collect_kernel_events();

  static constexpr int32_t kDefaultWaitLimit = 1 << 22;
  int32_t wait_limit_ = kDefaultWaitLimit;
  uint32_t test_skip_ = 0;
  int device_ = 0;
  int n_sm_ = 148;
  cudaStream_t stream_ = nullptr;
  LaunchAux aux_;
  bool capturing_ = false;  // inside sequence_graph's capture
  std::vector<DevFrame*> pool_;
  DevFrame* slots_[8] = {nullptr};
  // Record staging for recon(): pinned host buffers (double-buffered),
  // which build_work writes into directly, and device buffers.
  uint8_t* h_stage_[2] = {nullptr, nullptr};
  size_t h_stage_cap_[2] = {0, 0};
  uint8_t* d_stage_[2] = {nullptr, nullptr};
  size_t stage_cap_[2] = {0, 0};
  cudaEvent_t stage_ev_[2] = {nullptr, nullptr};
  int stage_ = 0;
  uint32_t* d_lf_mi_ = nullptr;
  size_t lf_mi_cap_ = 0;
  uint32_t* d_sb_done_ = nullptr;
  size_t sb_cap_ = 0;
  int32_t* d_counters_ = nullptr;  // [0] intra, [1] lf, [2] error
  int32_t* h_error_ = nullptr;     // pinned copy of the error word
  uint32_t epoch_ = 0;
  uint8_t* fixed_ = nullptr;  // the fixed scratch, during sequence_run_fixed
  uint8_t* sink_ = nullptr;
  size_t sink_cap_ = 0, sink_used_ = 0;
  uint8_t* d_digest_ = nullptr;
  size_t digest_cap_ = 0, digest_n_ = 0;
  // Digest jobs of shown frames queued on a stream, launched together.
  void digest_add(DevFrame* f, Md5Jobs* jobs, int* n);
  uint64_t sink_frames_ = 0, sink_dropped_ = 0;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  // run_batched's launch shapes and tables (pinned host, device), on the
  // first engine of the batch.
  TuneParams batch_tune_;
  uint8_t* batch_h_ = nullptr;
  uint8_t* batch_d_ = nullptr;
  size_t batch_cap_ = 0;
  // Per-kernel timing.
  std::vector<cudaEvent_t> kev_;
  std::vector<int> kev_kernel_;
  size_t kev_used_ = 0;
  const FrameWork* cur_fw_ = nullptr;
  // Work lists of the frame being built.
  std::vector<InterUnit> units_small_, units_large_;
  std::vector<ResItem> res_by_size_[4];
  std::vector<IntraItem> intra_, sorted_intra_;
  std::vector<uint16_t> intra_diag_;
  std::vector<uint32_t> diag_start_;
  std::vector<uint32_t> intra_jobs_;
};

}  // namespace rv9g

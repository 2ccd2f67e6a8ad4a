// The reconstruction engine: device frame buffers, the eight reference slots,
// and the per-frame launch of the reconstruction kernels from a parsed
// frame's records.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../host/parser.h"
#include "engine_types.h"

namespace rv9g {

cudaError_t launch_frame(const KFrame& k, int n_blocks, cudaStream_t s, int n_sm, int* launches);
cudaError_t upload_filters(const int16_t* f);

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
  int refs = 0;             // reference slots holding it
  bool busy = false;        // being reconstructed or copied out
  // Output metadata.
  uint8_t color_space = 1, color_range = 0;
  uint32_t render_w = 0, render_h = 0;
  cudaEvent_t ready = nullptr;  // recorded when reconstruction is enqueued
  size_t bps() const { return bit_depth > 8 ? 2 : 1; }
};

struct HostFrameOut {
  DevFrame* f;
};

class Engine {
 public:
  Engine() = default;
  ~Engine();
  bool init(int device, std::string* err);
  // Reconstructs a parsed frame (or handles show_existing); returns the frame
  // to show (or null) — valid until the next call.
  rv9::Status recon(rv9::ParsedFrame& pf, DevFrame** shown, std::string* err);
  // Copies the visible planes of `f`, packed (the reference Frame layout),
  // into host memory `dst` (pinned or not) on the engine's stream; waits.
  rv9::Status download(DevFrame* f, uint8_t* dst, std::string* err);
  // Enqueues the packed copy of `f` into `dst` without waiting.
  rv9::Status download_async(DevFrame* f, uint8_t* dst, std::string* err);
  rv9::Status sync(std::string* err);
  static size_t packed_bytes(const DevFrame* f);

  // Stats.
  double device_ms = 0;
  uint64_t frames = 0, alg_bytes = 0, launches = 0;
  cudaStream_t stream() const { return stream_; }

 private:
  DevFrame* alloc_frame(const rv9_frame_desc& d);
  void release_ref(DevFrame* f);
  bool ensure_scratch(size_t bytes, std::string* err);
  void build_work(const rv9::ParsedFrame& pf);

  int device_ = 0;
  int n_sm_ = 148;
  cudaStream_t stream_ = nullptr;
  std::vector<DevFrame*> pool_;
  DevFrame* slots_[8] = {nullptr};
  // Device scratch for one frame's records and work lists, and its pinned
  // host staging copy.
  uint8_t* d_scratch_ = nullptr;
  uint8_t* h_scratch_ = nullptr;
  size_t scratch_cap_ = 0;
  uint32_t* d_lf_mi_ = nullptr;
  size_t lf_mi_cap_ = 0;
  uint32_t* d_sb_done_ = nullptr;
  size_t sb_cap_ = 0;
  int32_t* d_counters_ = nullptr;  // [0] intra, [1] lf, [2] error
  uint32_t epoch_ = 0;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  // Work lists of the current frame.
  std::vector<InterUnit> units_;
  std::vector<ResItem> res_;
  std::vector<IntraItem> intra_;
};

}  // namespace rv9g

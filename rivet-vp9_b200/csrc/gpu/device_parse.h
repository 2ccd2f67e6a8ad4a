// Device-side parsing of a batch of frames: the tile syntax on the GPU (one
// thread per tile column, every column of every frame of the batch at once;
// tile_parse.cuh), then one CTA per frame that gathers its columns' records
// and builds the reconstruction engine's work lists from them, in the exact
// order the host's Engine::build_work gives. The host keeps the frame headers
// (rv9::Parser::begin); a frame goes to the device when
// rv9::Parser::external_tiles admits it.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../host/parser.h"
#include "engine.h"
#include "tile_parse.cuh"

namespace rv9g {

// One frame's outcome as the build kernel leaves it (read back per batch).
struct BuildOut {
  int32_t err;  // tp::Error of the first failing tile in bitstream order, or 0
  uint32_t err_tile;
  uint32_t n_blocks, n_toks, n_coefs, n_units, n_units_small, n_res, n_intra, n_intra_jobs;
  uint32_t n_res_by_size[4];
  uint64_t kbytes[K_COUNT];
  uint64_t total_bytes;
  uint64_t bools;
};

// What the build kernel reads of a frame.
struct BuildFrame {
  uint32_t first_chain, n_chains;
  uint32_t mi_cols, mi_rows, sb64_cols, sb64_rows;
  uint32_t ss_x, ss_y, bit_depth, legacy_uv, lf_on;
  uint32_t cap_blocks, cap_items;
  uint64_t base;  // the frame's staged region in the batch's stage buffer (bytes)
  uint64_t o_blocks, o_toks, o_coefs, o_units, o_res, o_intra, o_jobs;  // within the region
  uint64_t scratch_at;  // the frame's per-block scratch (8 words per block)
};

// Kernel launches (parse_kernels.cu).
cudaError_t parse_tables(int device, const tp::Tables** out);
cudaError_t launch_parse_chains(const tp::Tables* T, const tp::FrameIn* frames, const tp::Chain* chains,
                                uint32_t first, uint32_t n, const tp::Span* spans, const uint8_t* data, tp::Mi* mi,
                                uint8_t* above, const tp::PrevMv* prev, rv9_block* blocks, rv9_tok* toks,
                                uint32_t* coefs, tp::ChainOut* outs, cudaStream_t s);
cudaError_t launch_mi_to_prev(const tp::Mi* mi, tp::PrevMv* prev, uint32_t n, cudaStream_t s);
cudaError_t launch_build_frames(const BuildFrame* frames, uint32_t n, const tp::Chain* chains,
                                const tp::ChainOut* outs, const rv9_block* blocks, const rv9_tok* toks,
                                const uint32_t* coefs, uint8_t* stage, uint32_t* scratch, BuildOut* results,
                                cudaStream_t s);

// A batch of frames for the device parser. Frames are added in decode order
// (add), then parsed and built together (launch, on one stream; frames that
// read the previous frame's motion vectors from a frame of the same batch go
// in a later wave of the parse), then read back (collect): each frame's
// status and FrameWork, whose offsets are relative to frame_base(i) in the
// batch's device stage buffer. The buffers grow as needed and are kept.
// Stage buffers alternate between batches, so that one batch is parsed while
// the frames of the one before reconstruct from the other buffer: after
// queuing a batch's reconstruction, the caller calls recon_queued with the
// reconstruction's stream, and a later batch that reuses that buffer waits
// for it.
class DeviceParser {
 public:
  DeviceParser() = default;
  ~DeviceParser();
  rv9::Status init(int device, std::string* err);
  void clear();
  size_t size() const { return frames_.size(); }
  // Adds a frame (its header and probabilities from the host parser, its
  // frame description for the engine). False when the frame's tile data
  // does not split into tiles (the caller leaves it to the host parser,
  // which reports the error).
  bool add(const rv9::Parser::ExternalTiles& x, const rv9_frame_desc& desc);
  // Queues the batch on `s` and returns once its tile columns are parsed
  // (its work lists are then being built on `s`).
  rv9::Status launch(cudaStream_t s, std::string* err);
  // Waits for the batch and reads back every frame's outcome.
  rv9::Status collect(cudaStream_t s, std::string* err);
  // Waits (asleep) for the work queued on `s` so far.
  rv9::Status wait_on(cudaStream_t s, std::string* err);
  // Frame i after collect: its tiles' status (and message), and its work.
  rv9::Status frame_status(size_t i, std::string* msg) const;
  void frame_work(size_t i, FrameWork* fw) const;  // counts, offsets and bytes (not the header fields)
  const uint8_t* frame_base(size_t i) const { return d_stage_[cur_] + fi_[i].base; }
  uint64_t frame_offset(size_t i) const { return fi_[i].base; }
  size_t stage_bytes() const { return stage_used_; }
  // The current batch's reconstruction is queued on `s`: its stage buffer
  // is free once `s` gets past this point. Switches to the other buffer.
  rv9::Status recon_queued(cudaStream_t s, std::string* err);
  // The last device-parsed frame's motion vectors (mi_rows x mi_cols
  // PrevMv), copied to the host, for a frame the host parser takes next.
  rv9::Status last_prev(std::vector<tp::PrevMv>* out, cudaStream_t s, std::string* err);
  bool have_last() const { return have_last_; }
  uint64_t bools() const { return bools_; }
  // Device bytes a parser holds for batches of `frames` frames of this size
  // at most: both stage buffers, the parse records, the frames' mode info
  // and motion vectors, and the build scratch, at the worst-case capacities
  // add() reserves (the compressed data and per-frame tables, which are
  // small beside them, excluded).
  static uint64_t footprint(uint32_t width, uint32_t height, uint32_t ss_x, uint32_t ss_y, uint32_t frames,
                            int stage_buffers = 2);
  // Allocates every buffer for batches of `frames` frames of this size at
  // the capacities footprint counts, so that such batches allocate nothing
  // (a device allocation or free waits for the whole device).
  rv9::Status reserve(uint32_t width, uint32_t height, uint32_t ss_x, uint32_t ss_y, uint32_t frames,
                      std::string* err);
  // One stage buffer instead of two, for a caller whose batch's
  // reconstruction has ended before it launches the next batch (a batch
  // reuses the buffer after waiting for the last one's reconstruction on
  // the device, as it would for the other buffer). Before reserve().
  void set_single_stage() { single_stage_ = true; }
  // Lets go of the current stage buffer: the caller owns it (cudaFree) and
  // a new one is allocated for the next batch that uses this slot.
  uint8_t* release_stage();

 private:
  struct FrameInfo {
    uint32_t first_chain, n_chains;
    uint64_t base, bytes;
    int wave;
    int prev_from;  // index of the batch frame it takes previous vectors from, -1 none
    bool prev_host; // previous vectors uploaded from the host
    uint64_t prev_host_at;
    uint64_t mi_at, prev_at;
  };
  template <class T>
  static rv9::Status grow(T** p, size_t* cap, size_t need, std::string* err);
  int device_ = 0;
  const tp::Tables* T_ = nullptr;
  std::vector<tp::FrameIn> fin_;
  std::vector<tp::Chain> chains_;
  std::vector<tp::Span> spans_;
  std::vector<uint8_t> data_;        // tile data
  std::vector<uint8_t> prev_host_;   // host-held previous vectors of frames that read them
  std::vector<FrameInfo> fi_;
  std::vector<BuildFrame> build_;
  std::vector<BuildOut> outs_;
  std::vector<rv9_frame_desc> frames_;
  uint64_t n_mi_ = 0, n_above_ = 0, n_prev_ = 0, n_blocks_ = 0, n_toks_ = 0, n_coefs_ = 0, stage_used_ = 0,
           scratch_used_ = 0;
  int last_frame_ = -1;       // the batch's last frame so far
  bool have_last_ = false;    // d_last_prev_ holds the last device-parsed frame's vectors
  uint32_t last_mi_len_ = 0;
  uint64_t bools_ = 0;
  // Device buffers.
  uint8_t* d_data_ = nullptr;
  size_t data_cap_ = 0;
  tp::FrameIn* d_fin_ = nullptr;
  size_t fin_cap_ = 0;
  tp::Chain* d_chains_ = nullptr;
  size_t chains_cap_ = 0;
  tp::Span* d_spans_ = nullptr;
  size_t spans_cap_ = 0;
  tp::ChainOut* d_outs_ = nullptr;
  size_t outs_cap_ = 0;
  tp::Mi* d_mi_ = nullptr;
  size_t mi_cap_ = 0;
  uint8_t* d_above_ = nullptr;
  size_t above_cap_ = 0;
  tp::PrevMv* d_prev_ = nullptr;
  size_t prev_cap_ = 0;
  rv9_block* d_blocks_ = nullptr;
  size_t blocks_cap_ = 0;
  rv9_tok* d_toks_ = nullptr;
  size_t toks_cap_ = 0;
  uint32_t* d_coefs_ = nullptr;
  size_t coefs_cap_ = 0;
  uint8_t* d_stage_[2] = {nullptr, nullptr};
  size_t stage_cap_[2] = {0, 0};
  cudaEvent_t stage_free_[2] = {nullptr, nullptr};
  cudaEvent_t collected_ = nullptr;  // the host's waits on the stream (blocking: the waiting thread sleeps)
  bool stage_pending_[2] = {false, false};  // stage_free_ recorded, not yet waited for
  int cur_ = 0;
  bool single_stage_ = false;
  uint32_t* d_scratch_ = nullptr;
  size_t scratch_cap_ = 0;
  BuildFrame* d_build_ = nullptr;
  size_t build_cap_ = 0;
  BuildOut* d_results_ = nullptr;
  size_t results_cap_ = 0;
  tp::PrevMv* d_last_prev_ = nullptr;  // the last device-parsed frame's vectors, between batches
  size_t last_prev_cap_ = 0;
  uint8_t* h_pinned_ = nullptr;  // host staging of the batch's inputs
  size_t pinned_cap_ = 0;
};

}  // namespace rv9g

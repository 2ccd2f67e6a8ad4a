// The host side of the decoder: frame headers, tile and block syntax, motion
// vector prediction, coefficient tokens and the decoder's frame-to-frame
// state (reference frame slots' sizes and formats, four frame contexts,
// previous motion vectors and segment ids). Everything of VP9 decoding except
// the samples: a parsed frame comes out as records (rv9_records.h) for a
// reconstruction engine.
//
// Follows the reference decoder's frame process (src/decoder/mod.rs:218-422)
// and its parse-only mode (src/decoder/block.rs:368-1715, mvpred.rs,
// header.rs, probs.rs), restated in C++.
#pragma once
#include <stdint.h>

#include <deque>
#include <functional>
#include <string>
#include <vector>

#include "../../../include/rv9_records.h"
#include "probs.h"

namespace rv9 {

enum Status : int {
  ST_OK = 0,
  ST_BITSTREAM = 1,
  ST_UNSUPPORTED = 2,
  ST_INVALID_INPUT = 3,
  ST_DEVICE = 4,
};

struct Mv {
  int32_t r, c;
  bool operator==(const Mv& o) const { return r == o.r && c == o.c; }
  bool operator!=(const Mv& o) const { return !(*this == o); }
};

// Per 8x8 position (the MiInfo of reference src/decoder/block.rs:19-31).
struct MiInfo {
  uint8_t mi_size;
  uint8_t skip;
  uint8_t tx_size;
  uint8_t y_mode;
  uint8_t sub_modes[4];
  uint8_t segment_id;
  int8_t ref_frame[2];
  uint8_t interp_filter;
  Mv mv[2][4];
};

// A parsed frame: what to do with the reference slots, and the records.
struct ParsedFrame {
  bool show_existing = false;  // show_existing_frame: output slot `show_slot`
  int show_slot = 0;
  bool show_frame = false;
  uint8_t refresh_mask = 0;    // slots that receive this frame
  int ref_slot[3] = {0, 0, 0}; // slots of LAST, GOLDEN, ALTREF (inter frames)
  rv9_frame_desc desc{};
  std::vector<rv9_block> blocks;
  std::vector<rv9_tok> toks;
  std::vector<uint32_t> coefs;
  double parse_seconds = 0;
};

struct SlotInfo {
  bool valid = false;
  uint32_t width = 0, height = 0;
  uint32_t ss_x = 1, ss_y = 1, bit_depth = 8;
};

namespace syn {
struct FrameHeader;
struct PrevMv;
}

class Parser {
 public:
  Parser();
  ~Parser();
  // 0: one thread per core (tile columns parse in parallel).
  void set_threads(int n) { threads_ = n; }
  void set_max_pixels(uint64_t p) { max_pixels_ = p; }
  uint64_t frames_decoded() const { return frames_; }
  // Parses one frame (not a superframe). On error returns the status and
  // fills `err`.
  Status parse_frame(const uint8_t* data, size_t len, ParsedFrame* out, std::string* err);

  // parse_frame in three steps, for frame-parallel parsing (FramePipeline):
  // begin parses the headers and applies what they decide; `after_header`
  // (may be empty) runs once the uncompressed header is read, before any
  // other state is touched. run parses the tiles (any thread; reads only the
  // job). finish applies what the tiles decide, in frame order, and hands out
  // the records. Every job ends with release.
  struct Job;
  using AfterHeader = std::function<void(const syn::FrameHeader&)>;
  Job* begin(const uint8_t* data, size_t len, const AfterHeader& after_header);
  void attach_work(Job* job);
  void run(Job* job);
  Status finish(Job* job, ParsedFrame* out, std::string* err);
  void release(Job* job);

  // Frames whose tiles another parser takes (the device tile parser): after
  // begin, external_tiles says whether the frame can be handed out (nothing
  // of it adapts probabilities, reads or writes segment ids, or needs the
  // legacy 4:4:4 probe) and what its tiles read; the other parser's outcome
  // comes back through finish_external, in frame order (ST_OK, or the
  // status and message of the first tile in bitstream order that failed).
  // The frame's motion vectors then stay with that parser: a later frame
  // parsed here that reads them (wants_external_prev) must be given them
  // first (provide_prev_mvs, in syn::PrevMv layout, mi_rows x mi_cols).
  // begin takes the previous frame's vectors as the state holds them then;
  // when frames were begun ahead of others that finish later, bind_prev
  // (after those finish) takes them again from the state.
  struct ExternalTiles {
    const syn::FrameHeader* h = nullptr;
    const Probs* probs = nullptr;
    const bool* ref_ok = nullptr;         // [3]
    const uint8_t* tiles = nullptr;       // the frame's tile data
    size_t tiles_len = 0;
    // Whether the frame reads the previous frame's motion vectors, as its
    // header and the last frame decide. Where they come from, as the state
    // was at begin (the right source when no frame begun before this one is
    // still unfinished; else the previous frame is one of those):
    // prev_external, held by the external parser; prev_host, held here; or
    // neither, in which case the frame reads none.
    bool use_prev = false;
    bool prev_external = false;
    const syn::PrevMv* prev_host = nullptr;
    const rv9_frame_desc* desc = nullptr;    // the records' frame description
  };
  bool external_tiles(const Job* job, ExternalTiles* out) const;
  // Whether the frame depends on nothing that frames before it decide at
  // finish (a key frame or an error-resilient one: contexts reset, no
  // previous motion vectors), so that it may parse while they do.
  bool independent(const Job* job) const;
  // attach_work, then run on a thread of the job's own; wait joins it
  // (finish and release need it joined; release joins it too).
  void run_async(Job* job);
  void wait(Job* job);
  Status finish_external(Job* job, Status tiles_st, const std::string& tiles_err, ParsedFrame* out,
                         std::string* err);
  void bind_prev(Job* job);
  bool wants_external_prev(const Job* job) const;
  void provide_prev_mvs(Job* job, const void* mvs, size_t n);

  struct Impl;

 private:
  Impl* impl_;
  int threads_ = 0;
  uint64_t max_pixels_ = 8192ull * 8192ull;
  uint64_t frames_ = 0;
};

// Parses the frames of one stream in order with several in flight at once.
// A frame whose parse may read what an earlier frame's tiles decide (adapted
// contexts, previous motion vectors or segment ids) waits for those frames;
// key frames and error-resilient frames do not, so streams made of them parse
// `depth` frames at a time. Results come out in order, identical to
// parse_frame's; after an error, the frames behind it are dropped and the
// parser's state is the failed frame's, as with parse_frame.
class FramePipeline {
 public:
  FramePipeline(Parser* parser, int depth);
  ~FramePipeline();
  // Starts a frame (its bytes must stay valid until it is popped).
  Status push(const uint8_t* data, size_t len);
  // The oldest frame's records (waits for its tiles).
  Status pop(ParsedFrame* out, std::string* err);
  size_t in_flight() const { return q_.size(); }
  int depth() const { return depth_; }

 private:
  void settle();
  Parser* p_;
  int depth_;
  std::deque<Parser::Job*> q_;
  bool failed_ = false;
};

// Annex B: splits a packet into its frames (reference src/superframe.rs:6-53).
void superframe_split(const uint8_t* pkt, size_t len, std::vector<std::pair<size_t, size_t>>* out);

}  // namespace rv9

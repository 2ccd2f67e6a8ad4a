// The tile, partition and block syntax of VP9 (spec 6.4), written once for
// both directions: TileCoder<DecCoder> parses (the host decoder), and
// TileCoder<EncCoder> writes the same syntax from an encoder's decisions (the
// stream generator). Every syntax element goes through the coder as
// `d.bit(prob, want)` or `d.tree(tree, probs, want)`; decoding ignores `want`.
//
// A C++ restatement of the reference decoder's tile and block syntax
// (src/decoder/block.rs:368-1715) and motion vector prediction
// (src/decoder/mvpred.rs), with the records of rv9_records.h as output.
#pragma once
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cstdlib>
#include <memory>
#include <vector>

#include "../../../include/rv9_records.h"
#include "../common/vp9_consts.h"
#include "../common/vp9_tables.h"
#include "bitreader.h"
#include "parser.h"
#include "probs.h"

namespace rv9 {
namespace syn {
using namespace vp9;

struct ParseError {
  Status st;
  const char* msg;
};

[[noreturn]] inline void bitstream_error(const char* m) { throw ParseError{ST_BITSTREAM, m}; }

struct LoopFilterParams {
  uint8_t level = 0, sharpness = 0;
  bool delta_enabled = true;
  int8_t ref_deltas[4] = {1, 0, -1, -1};
  int8_t mode_deltas[2] = {0, 0};
};

struct SegParams {
  bool enabled = false, update_map = false, temporal_update = false, abs_or_delta_update = false;
  uint8_t tree_probs[7] = {0};
  uint8_t pred_probs[3] = {0};
  bool feature_enabled[MAX_SEGMENTS][4] = {};
  int16_t feature_data[MAX_SEGMENTS][4] = {};
  bool active(int seg, int f) const { return enabled && feature_enabled[seg][f]; }
};

// State the uncompressed header reads and writes across frames
// (reference src/header.rs:58-84).
struct Persistent {
  LoopFilterParams lf;
  SegParams seg;
  uint32_t ref_w[8] = {0}, ref_h[8] = {0};
  uint8_t last_frame_type = KEY_FRAME;
  uint32_t bit_depth = 8, ss_x = 1, ss_y = 1;
  uint8_t color_space = 1;
  bool color_range = false;
};

// Everything the headers say about one frame (reference src/header.rs:88-146).
struct FrameHeader {
  uint8_t profile = 0;
  bool show_existing_frame = false;
  uint8_t frame_to_show_map_idx = 0;
  uint8_t frame_type = 0;
  uint8_t last_frame_type = 0;
  bool show_frame = false, error_resilient_mode = false, intra_only = false;
  uint8_t reset_frame_context = 0;
  uint32_t bit_depth = 8;
  uint8_t color_space = 1;
  bool color_range = false;
  uint32_t ss_x = 1, ss_y = 1;
  uint8_t refresh_frame_flags = 0;
  uint8_t ref_frame_idx[3] = {0, 0, 0};
  bool ref_frame_sign_bias[4] = {false, false, false, false};
  uint32_t width = 0, height = 0, render_width = 0, render_height = 0;
  bool allow_high_precision_mv = false;
  uint8_t interpolation_filter = 0;
  bool refresh_frame_context = false, frame_parallel_decoding_mode = false;
  uint8_t frame_context_idx = 0;
  int32_t base_q_idx = 0, delta_q_y_dc = 0, delta_q_uv_dc = 0, delta_q_uv_ac = 0;
  bool lossless = false;
  uint32_t tile_cols_log2 = 0, tile_rows_log2 = 0;
  uint32_t header_size_in_bytes = 0;
  size_t uncompressed_size = 0;
  bool past_independence = false;
  bool frame_is_intra = false;
  uint32_t mi_cols = 0, mi_rows = 0, sb64_cols = 0, sb64_rows = 0;
  uint8_t tx_mode = 0, reference_mode = 0;
  int8_t comp_fixed_ref = 0;
  int8_t comp_var_ref[2] = {0, 0};
  bool legacy_uv = false;

  void compute_image_size() {
    mi_cols = (width + 7) >> 3;
    mi_rows = (height + 7) >> 3;
    sb64_cols = (mi_cols + 7) >> 3;
    sb64_rows = (mi_rows + 7) >> 3;
  }
};

// get_tile_offset (spec 6.4.1).
inline uint32_t tile_offset(uint32_t tile_num, uint32_t mis, uint32_t log2) {
  uint32_t sbs = (mis + 7) >> 3;
  uint32_t off = ((tile_num * sbs) >> log2) << 3;
  return off < mis ? off : mis;
}

struct PrevMv {
  int8_t ref_frame[2];
  Mv mv[2];
};

// Probability of node `node` of the token tree (pareto, spec 9.3.2).
inline uint8_t pareto(int node, uint8_t prob) {
  if (node < 2) return prob;
  int x = ((prob < 1 ? 1 : prob) - 1) / 2;
  if (prob & 1) return vp9t_pareto_table[x][node - 2];
  int x1 = x + 1 < 127 ? x + 1 : 127;
  return (uint8_t)(((uint32_t)vp9t_pareto_table[x][node - 2] + vp9t_pareto_table[x1][node - 2]) >> 1);
}

// A growable array of plain values whose growth leaves the new elements
// uninitialised: the token loop reserves a block's worth of coefficient
// words, writes the nonzero ones and gives the rest back.
template <class T>
class PodVec {
 public:
  size_t size() const { return size_; }
  T* data() { return buf_.get(); }
  const T* data() const { return buf_.get(); }
  const T* begin() const { return buf_.get(); }
  const T* end() const { return buf_.get() + size_; }
  void clear() { size_ = 0; }
  void push_back(T v) { *grow(1) = v; }
  // `n` more elements at the end, uninitialised; returns the first.
  T* grow(size_t n) {
    if (size_ + n > cap_) {
      size_t cap = std::max(size_ + n, cap_ * 2 + 1024);
      std::unique_ptr<T[]> b(new T[cap]);
      if (size_) memcpy(b.get(), buf_.get(), size_ * sizeof(T));
      buf_ = std::move(b);
      cap_ = cap;
    }
    T* p = buf_.get() + size_;
    size_ += n;
    return p;
  }
  void shrink_to(size_t n) { size_ = n < size_ ? n : size_; }

 private:
  std::unique_ptr<T[]> buf_;
  size_t size_ = 0, cap_ = 0;
};

// pareto() for every probability value: row p holds the probabilities of
// token-tree nodes 2..9 when node 1's probability is p.
struct ParetoRows {
  uint8_t row[256][8];
  ParetoRows() {
    for (int p = 0; p < 256; ++p)
      for (int k = 2; k < 10; ++k) row[p][k - 2] = pareto(k, (uint8_t)p);
  }
};
inline const uint8_t* pareto_row(uint8_t prob) {
  static const ParetoRows rows;
  return rows.row[prob];
}

// The scan order of get_scan (spec 6.4.25).
inline const uint16_t* get_scan(int tx_sz, int tx_type) {
  switch (tx_sz) {
    case TX_4X4:
      return tx_type == ADST_DCT ? vp9t_row_scan_4x4 : tx_type == DCT_ADST ? vp9t_col_scan_4x4 : vp9t_default_scan_4x4;
    case TX_8X8:
      return tx_type == ADST_DCT ? vp9t_row_scan_8x8 : tx_type == DCT_ADST ? vp9t_col_scan_8x8 : vp9t_default_scan_8x8;
    case TX_16X16:
      return tx_type == ADST_DCT ? vp9t_row_scan_16x16
             : tx_type == DCT_ADST ? vp9t_col_scan_16x16
                                   : vp9t_default_scan_16x16;
    default:
      return vp9t_default_scan_32x32;
  }
}

// The two positions whose token energies give the context of the coefficient
// at each scan index (spec 6.4.24's above / left), per transform size and
// scan kind (reference src/decoder/block.rs:1656-1699).
struct NeighborTables {
  uint16_t nb[4][3][1024][2];
  NeighborTables() {
    const uint8_t types[3] = {DCT_DCT, DCT_ADST, ADST_DCT};
    for (int txs = 0; txs < 4; ++txs)
      for (int k = 0; k < 3; ++k) {
        int tx_type = types[k];
        int n = 4 << txs, log2n = 2 + txs, cnt = n * n;
        const uint16_t* sc = get_scan(txs, tx_type);
        for (int c = 0; c < cnt; ++c) {
          int pos = sc[c];
          int i = pos >> log2n, j = pos & (n - 1);
          int a, b;
          if (i > 0 && j > 0) {
            int up = (i - 1) * n + j, left = i * n + j - 1;
            if (tx_type == DCT_ADST) {
              a = b = up;
            } else if (tx_type == ADST_DCT) {
              a = b = left;
            } else {
              a = up;
              b = left;
            }
          } else if (i > 0) {
            a = b = (i - 1) * n + j;
          } else {
            a = b = j > 0 ? j - 1 : 0;
          }
          nb[txs][k][c][0] = (uint16_t)a;
          nb[txs][k][c][1] = (uint16_t)b;
        }
      }
  }
  const uint16_t (*get(int tx_sz, int tx_type) const)[2] {
    int k = tx_type == DCT_ADST ? 1 : tx_type == ADST_DCT ? 2 : 0;
    return nb[tx_sz][k];
  }
};

inline const NeighborTables& neighbor_tables() {
  static const NeighborTables t;
  return t;
}

inline bool use_mv_hp(const Mv& mv) {
  return (std::abs(mv.r) >> 3) < COMPANDED_MVREF_THRESH && (std::abs(mv.c) >> 3) < COMPANDED_MVREF_THRESH;
}

// The state of the block being decoded (reference src/decoder/block.rs:51-76).
struct BlockState {
  uint32_t mi_row, mi_col;
  uint8_t mi_size;
  bool avail_u, avail_l;
  uint8_t segment_id;
  bool skip;
  uint8_t tx_size;
  bool is_inter;
  uint8_t y_mode;
  uint8_t sub_modes[4];
  uint8_t uv_mode;
  int8_t ref_frame[2];
  uint8_t interp_filter;
  Mv block_mvs[2][4];
  const MiInfo* above;
  const MiInfo* left;
  uint8_t mode_context[4];
  Mv nearest_mv[2], near_mv[2], best_mv[2], mv[2];
};

// Shared, read-only inputs of a frame's tile decode.
struct FrameCtx {
  const FrameHeader* h;
  const SegParams* seg;
  const Probs* probs;
  const uint8_t* prev_seg_ids;
  size_t prev_seg_len;
  const PrevMv* prev_mvs;  // null unless UsePrevFrameMvs
  MiInfo* mi;              // frame-wide mode info, mi_rows x mi_cols
  uint8_t* above_nonzero[3];
  uint8_t* above_partition;
  uint8_t* above_seg_pred;
  bool ref_scale_ok[3];
  bool count_coefs;
};


// The boolean encoder: the exact inverse of BoolDecoder (spec 9.2). `low`
// accumulates the arithmetic code; whole bytes leave it with carries
// propagated into the bytes already written.
class BoolEncoder {
 public:
  void reset() {
    buf_.clear();
    low_ = 0;
    range_ = 255;
    count_ = -24;
  }
  void write(bool bit, int prob) {
    uint32_t split = 1 + (((range_ - 1) * (uint32_t)prob) >> 8);
    if (bit) {
      low_ += split;
      range_ -= split;
    } else {
      range_ = split;
    }
    int shift = __builtin_clz(range_) - 24;
    range_ <<= shift;
    count_ += shift;
    if (count_ >= 0) {
      int offset = shift - count_;
      if ((low_ << (offset - 1)) & 0x80000000u) {
        // Carry into the bytes already out.
        int x = (int)buf_.size() - 1;
        while (x >= 0 && buf_[x] == 0xff) {
          buf_[x] = 0;
          --x;
        }
        ++buf_[x];
      }
      buf_.push_back((uint8_t)(low_ >> (24 - offset)));
      low_ <<= offset;
      shift = count_;
      low_ &= 0xffffff;
      count_ -= 8;
    }
    low_ <<= shift;
  }
  void literal(uint32_t v, int n) {
    for (int i = n - 1; i >= 0; --i) write(((v >> i) & 1) != 0, 128);
  }
  // Pads with zero bits so that every written bit is decodable, and returns
  // the bytes.
  std::vector<uint8_t>& finish() {
    for (int i = 0; i < 32; ++i) write(false, 128);
    // A last byte that looks like a superframe marker would be misread.
    if (!buf_.empty() && (buf_.back() & 0xe0) == 0xc0) buf_.push_back(0);
    return buf_;
  }

 private:
  std::vector<uint8_t> buf_;
  uint32_t low_ = 0;
  uint32_t range_ = 255;
  int count_ = -24;
};

// Reading.
struct DecCoder {
  static constexpr bool kEncode = false;
  BoolDecoder bd;
  template <class F>
  inline bool bit(int prob, F&&) {
    return bd.read(prob);
  }
  template <class P, class F>
  inline int tree(const int8_t* t, P probs, F&&) {
    return bd.tree(t, probs);
  }
};

// Writing: each element's value is `want()`.
struct EncCoder {
  static constexpr bool kEncode = true;
  BoolEncoder be;
  template <class F>
  inline bool bit(int prob, F&& want) {
    bool v = want();
    be.write(v, prob);
    return v;
  }
  // Finds the path to leaf `v` and writes its branch bits.
  static bool path(const int8_t* t, int node, int v, int* nodes, int* bits, int* depth) {
    for (int br = 0; br < 2; ++br) {
      int nx = t[node + br];
      nodes[*depth] = node;
      bits[*depth] = br;
      ++*depth;
      if (nx <= 0) {
        if (-nx == v) return true;
      } else if (path(t, nx, v, nodes, bits, depth)) {
        return true;
      }
      --*depth;
    }
    return false;
  }
  template <class P, class F>
  inline int tree(const int8_t* t, P probs, F&& want) {
    int v = want();
    int nodes[16], bits[16], depth = 0;
    path(t, 0, v, nodes, bits, &depth);
    for (int i = 0; i < depth; ++i) be.write(bits[i] != 0, probs(nodes[i] >> 1));
    return v;
  }
};

// An encoder's decisions for the block being written.
struct EncBlock {
  uint8_t segment_id = 0;
  bool skip = false;
  uint8_t tx_size = 0;
  bool is_inter = false;
  uint8_t y_mode = 0, uv_mode = 0;
  uint8_t sub_modes[4] = {0, 0, 0, 0};
  int8_t ref_frame[2] = {0, -1};
  uint8_t interp_filter = 0;
  Mv mv[2] = {{0, 0}, {0, 0}};
};

// What TileCoder<EncCoder> asks the encoder.
struct EncHooks {
  virtual ~EncHooks() = default;
  // The partition of the bsize region at (r, c); SPLIT when neither half
  // fits, and HORZ/SPLIT or VERT/SPLIT at the frame's edges.
  virtual int partition(uint32_t r, uint32_t c, uint8_t bsize, bool has_rows, bool has_cols) = 0;
  // Decides, predicts, transforms, quantises and reconstructs a block.
  virtual void analyze(uint32_t r, uint32_t c, uint8_t bsize, EncBlock* out) = 0;
  // The inter mode that codes the block's motion vector, given the
  // candidates of b.
  virtual int inter_mode(const BlockState& b, const EncBlock* eb) = 0;
  // The quantised coefficients (raster order) of a transform block, and its
  // end of block in `scan`.
  virtual const int32_t* tx_coefs(const EncBlock* eb, int plane, uint32_t x, uint32_t y, int tx_sz,
                                  const uint16_t* scan, int* eob) = 0;
};

// The token of a coefficient magnitude (spec 9.3: ZERO .. DCT_VAL_CAT6).
inline int token_of(int32_t v) {
  uint32_t a = (uint32_t)(v < 0 ? -v : v);
  if (a <= 4) return (int)a;
  if (a <= 6) return 5;
  if (a <= 10) return 6;
  if (a <= 18) return 7;
  if (a <= 34) return 8;
  if (a <= 66) return 9;
  return 10;
}

// One tile column's syntax: its left contexts, counts and records. `C` reads
// (decoding) or writes (encoding) each syntax element; when writing, the
// values come from the encoder's decisions (`enc_`, `eb_`).
template <class C>
struct TileCoder {
  const FrameCtx* f;
  const FrameHeader* h;
  Counts counts;
  std::vector<rv9_block> blocks;
  std::vector<rv9_tok> toks;
  PodVec<uint32_t> coefs;
  std::vector<uint8_t> left_nonzero[3];
  std::vector<uint8_t> left_partition;
  std::vector<uint8_t> left_seg_pred;
  uint32_t mi_row_start = 0, mi_row_end = 0, mi_col_start = 0, mi_col_end = 0;
  uint32_t mi_cols = 0, mi_rows = 0;
  uint32_t ss_x = 0, ss_y = 0;
  BlockState b;
  EncHooks* enc_ = nullptr;  // encoding: the decisions
  EncBlock* eb_ = nullptr;
  uint32_t eob_total = 0;
  uint8_t token_cache[1024];
  bool padding_ok = true;
  // The frame's coefficient probabilities repacked: word k of a band holds
  // node k's probability for context c in byte c, so the token loop takes a
  // probability by shifting a word it fetched ahead, not by a load that
  // waits for the context.
  uint64_t coef_pk[4][2][2][6][3];

  void init(const FrameCtx* fc) {
    f = fc;
    h = fc->h;
    counts.clear();
    blocks.clear();
    toks.clear();
    coefs.clear();
    size_t n4h = h->sb64_rows * 16 + 16;
    for (int p = 0; p < 3; ++p) left_nonzero[p].assign(n4h, 0);
    left_partition.assign(h->sb64_rows * 8 + 8, 0);
    left_seg_pred.assign(h->sb64_rows * 8 + 8, 0);
    mi_cols = h->mi_cols;
    mi_rows = h->mi_rows;
    ss_x = h->ss_x;
    ss_y = h->ss_y;
    padding_ok = true;
    for (int t = 0; t < 4; ++t)
      for (int pt = 0; pt < 2; ++pt)
        for (int rt = 0; rt < 2; ++rt)
          for (int band = 0; band < 6; ++band)
            for (int k = 0; k < 3; ++k) {
              uint64_t w = 0;
              for (int cx = 0; cx < 6; ++cx) w |= (uint64_t)fc->probs->coef[t][pt][rt][band][cx][k] << (8 * cx);
              coef_pk[t][pt][rt][band][k] = w;
            }
  }

  MiInfo& mi_at(uint32_t r, uint32_t c) const { return f->mi[(size_t)r * mi_cols + c]; }

  void decode_tile(C& d) {
    for (uint32_t r = mi_row_start; r < mi_row_end; r += 8) {
      for (int p = 0; p < 3; ++p) std::fill(left_nonzero[p].begin(), left_nonzero[p].end(), 0);
      std::fill(left_partition.begin(), left_partition.end(), 0);
      std::fill(left_seg_pred.begin(), left_seg_pred.end(), 0);
      for (uint32_t c = mi_col_start; c < mi_col_end; c += 8) decode_partition(d, r, c, BLOCK_64X64);
    }
  }

  void decode_partition(C& d, uint32_t r, uint32_t c, uint8_t bsize) {
    if (r >= mi_rows || c >= mi_cols) return;
    uint32_t num8x8 = vp9t_num_8x8_wide[bsize];
    uint32_t half = num8x8 >> 1;
    bool has_rows = (r + half) < mi_rows;
    bool has_cols = (c + half) < mi_cols;
    uint32_t bsl = vp9t_mi_width_log2[bsize];
    uint32_t boffset = vp9t_mi_width_log2[BLOCK_64X64] - bsl;
    uint8_t above = 0, left = 0;
    for (uint32_t i = 0; i < num8x8; ++i) {
      above |= f->above_partition[c + i];
      left |= left_partition[(r + i)];
    }
    bool a = (above & (1 << boffset)) != 0;
    bool l = (left & (1 << boffset)) != 0;
    int ctx = (int)(bsl * 4 + (l ? 2 : 0) + (a ? 1 : 0));
    const uint8_t* probs = h->frame_is_intra ? vp9t_kf_partition_probs[ctx] : f->probs->partition[ctx];
    int partition;
    int want = 0;
    if (C::kEncode) want = enc_->partition(r, c, bsize, has_rows, has_cols);
    if (has_rows && has_cols)
      partition = d.tree(PARTITION_TREE, [&](int n) { return probs[n]; }, [&] { return want; });
    else if (has_cols)
      partition = d.bit(probs[1], [&] { return want == PARTITION_SPLIT; }) ? PARTITION_SPLIT : PARTITION_HORZ;
    else if (has_rows)
      partition = d.bit(probs[2], [&] { return want == PARTITION_SPLIT; }) ? PARTITION_SPLIT : PARTITION_VERT;
    else
      partition = PARTITION_SPLIT;
    if (!h->frame_is_intra) counts.partition[ctx][partition] += 1;
    uint8_t subsize = SUBSIZE_LOOKUP[partition][bsize];
    if (subsize == BLOCK_INVALID) bitstream_error("invalid partition");
    if (subsize < BLOCK_8X8 || partition == PARTITION_NONE) {
      decode_block(d, r, c, subsize);
    } else if (partition == PARTITION_HORZ) {
      decode_block(d, r, c, subsize);
      if (has_rows) decode_block(d, r + half, c, subsize);
    } else if (partition == PARTITION_VERT) {
      decode_block(d, r, c, subsize);
      if (has_cols) decode_block(d, r, c + half, subsize);
    } else {
      decode_partition(d, r, c, subsize);
      decode_partition(d, r, c + half, subsize);
      decode_partition(d, r + half, c, subsize);
      decode_partition(d, r + half, c + half, subsize);
    }
    if (bsize == BLOCK_8X8 || partition != PARTITION_SPLIT) {
      uint8_t av = (uint8_t)(15 >> vp9t_b_width_log2[subsize]);
      uint8_t lv = (uint8_t)(15 >> vp9t_b_height_log2[subsize]);
      for (uint32_t i = 0; i < num8x8; ++i) {
        f->above_partition[c + i] = av;
        left_partition[r + i] = lv;
      }
    }
  }

  void decode_block(C& d, uint32_t r, uint32_t c, uint8_t subsize) {
    if (ss_x + ss_y > 0 && subsize >= BLOCK_8X8) {
      if (SS_SIZE_LOOKUP[subsize][ss_x][ss_y] == BLOCK_INVALID)
        bitstream_error("block size invalid for the chroma subsampling");
    }
    BlockState& bb = b;
    memset(&bb, 0, sizeof bb);
    bb.mi_row = r;
    bb.mi_col = c;
    bb.mi_size = subsize;
    bb.avail_u = r > 0;
    bb.avail_l = c > mi_col_start;
    bb.above = bb.avail_u ? &mi_at(r - 1, c) : nullptr;
    bb.left = bb.avail_l ? &mi_at(r, c - 1) : nullptr;
    bb.ref_frame[0] = INTRA_FRAME;
    bb.ref_frame[1] = NONE_FRAME;
    if (C::kEncode) enc_->analyze(r, c, subsize, eb_);
    if (h->frame_is_intra)
      intra_frame_mode_info(d);
    else
      inter_frame_mode_info(d);
    eob_total = 0;
    size_t bi = blocks.size();
    blocks.emplace_back();
    uint32_t tok0 = (uint32_t)toks.size();
    bool coded_skip = bb.skip;
    residual(d);
    if (bb.is_inter && subsize >= BLOCK_8X8 && eob_total == 0) bb.skip = true;
    // Record.
    rv9_block& rb = blocks[bi];
    memset(&rb, 0, sizeof rb);
    rb.mi_row = (uint16_t)r;
    rb.mi_col = (uint16_t)c;
    rb.mi_size = subsize;
    rb.flags = (uint8_t)((bb.skip ? RV9_BLK_SKIP : 0) | (bb.is_inter ? RV9_BLK_INTER : 0) |
                         (bb.avail_l ? RV9_BLK_AVAIL_L : 0) | (bb.avail_u ? RV9_BLK_AVAIL_U : 0));
    rb.tx_size = bb.tx_size;
    rb.segment_id = bb.segment_id;
    rb.y_mode = bb.y_mode;
    rb.uv_mode = bb.uv_mode;
    rb.interp_filter = bb.interp_filter;
    rb.coded_skip = coded_skip ? 1 : 0;
    memcpy(rb.sub_modes, bb.sub_modes, 4);
    rb.ref_frame[0] = bb.ref_frame[0];
    rb.ref_frame[1] = bb.ref_frame[1];
    rb.tok_start = tok0;
    rb.n_tok = (uint16_t)(toks.size() - tok0);
    for (int l = 0; l < 2; ++l)
      for (int k = 0; k < 4; ++k) {
        rb.mv[l][k][0] = bb.block_mvs[l][k].r;
        rb.mv[l][k][1] = bb.block_mvs[l][k].c;
      }
    MiInfo info;
    info.mi_size = subsize;
    info.skip = bb.skip;
    info.tx_size = bb.tx_size;
    info.y_mode = bb.y_mode;
    memcpy(info.sub_modes, bb.sub_modes, 4);
    info.segment_id = bb.segment_id;
    info.ref_frame[0] = bb.ref_frame[0];
    info.ref_frame[1] = bb.ref_frame[1];
    info.interp_filter = bb.interp_filter;
    memcpy(info.mv, bb.block_mvs, sizeof info.mv);
    uint32_t bh = vp9t_num_8x8_high[subsize], bw = vp9t_num_8x8_wide[subsize];
    uint32_t ye = std::min(r + bh, mi_rows), xe = std::min(c + bw, mi_cols);
    for (uint32_t y = r; y < ye; ++y)
      for (uint32_t x = c; x < xe; ++x) mi_at(y, x) = info;
  }

  // ---- Mode info (spec 6.4.5 - 6.4.17) ----

  void intra_frame_mode_info(C& d) {
    const SegParams& seg = *f->seg;
    b.segment_id = (seg.enabled && seg.update_map)
                       ? (uint8_t)d.tree(SEGMENT_TREE, [&](int n) { return seg.tree_probs[n]; },
                                         [&] { return (int)eb_->segment_id; })
                       : 0;
    read_skip(d);
    read_tx_size(d, true);
    b.ref_frame[0] = INTRA_FRAME;
    b.ref_frame[1] = NONE_FRAME;
    b.is_inter = false;
    if (b.mi_size >= BLOCK_8X8) {
      uint8_t am = b.above ? b.above->sub_modes[2] : DC_PRED;
      uint8_t lm = b.left ? b.left->sub_modes[1] : DC_PRED;
      const uint8_t* p = vp9t_kf_y_mode_probs[am][lm];
      uint8_t mode = (uint8_t)d.tree(INTRA_MODE_TREE, [&](int n) { return p[n]; }, [&] { return (int)eb_->y_mode; });
      b.y_mode = mode;
      for (int i = 0; i < 4; ++i) b.sub_modes[i] = mode;
    } else {
      int n4w = vp9t_num_4x4_wide[b.mi_size], n4h = vp9t_num_4x4_high[b.mi_size];
      uint8_t mode = DC_PRED;
      for (int idy = 0; idy < 2; idy += n4h)
        for (int idx = 0; idx < 2; idx += n4w) {
          uint8_t am = idy > 0 ? b.sub_modes[idx] : (b.above ? b.above->sub_modes[2 + idx] : DC_PRED);
          uint8_t lm = idx > 0 ? b.sub_modes[idy * 2] : (b.left ? b.left->sub_modes[1 + idy * 2] : DC_PRED);
          const uint8_t* p = vp9t_kf_y_mode_probs[am][lm];
          mode = (uint8_t)d.tree(INTRA_MODE_TREE, [&](int n) { return p[n]; },
                                 [&] { return (int)eb_->sub_modes[idy * 2 + idx]; });
          for (int y2 = 0; y2 < n4h; ++y2)
            for (int x2 = 0; x2 < n4w; ++x2) b.sub_modes[(idy + y2) * 2 + idx + x2] = mode;
        }
      b.y_mode = mode;
    }
    const uint8_t* p = vp9t_kf_uv_mode_probs[b.y_mode];
    b.uv_mode = (uint8_t)d.tree(INTRA_MODE_TREE, [&](int n) { return p[n]; }, [&] { return (int)eb_->uv_mode; });
  }

  void read_skip(C& d) {
    if (f->seg->active(b.segment_id, SEG_LVL_SKIP)) {
      b.skip = true;
    } else {
      int ctx = (b.above ? b.above->skip : 0) + (b.left ? b.left->skip : 0);
      b.skip = d.bit(f->probs->skip[ctx], [&] { return eb_->skip; });
      counts.skip[ctx][b.skip ? 1 : 0] += 1;
    }
  }

  void read_tx_size(C& d, bool allow_select) {
    uint8_t max_tx = MAX_TXSIZE_LOOKUP[b.mi_size];
    if (allow_select && h->tx_mode == TX_MODE_SELECT && b.mi_size >= BLOCK_8X8) {
      uint8_t above = max_tx, left = max_tx;
      if (b.above && !b.above->skip) above = b.above->tx_size;
      if (b.left && !b.left->skip) left = b.left->tx_size;
      if (!b.avail_l) left = above;
      if (!b.avail_u) above = left;
      int ctx = (above + left) > max_tx ? 1 : 0;
      const uint8_t* p = f->probs->tx[max_tx][ctx];
      const int8_t* tree = max_tx == TX_32X32 ? TX_SIZE_32_TREE : max_tx == TX_16X16 ? TX_SIZE_16_TREE : TX_SIZE_8_TREE;
      int v = d.tree(tree, [&](int n) { return p[n]; }, [&] { return (int)eb_->tx_size; });
      counts.tx[max_tx][ctx][v] += 1;
      b.tx_size = (uint8_t)v;
    } else {
      uint8_t m = TX_MODE_TO_BIGGEST_TX_SIZE[h->tx_mode];
      b.tx_size = max_tx < m ? max_tx : m;
    }
  }

  void inter_frame_mode_info(C& d) {
    inter_segment_id(d);
    read_skip(d);
    read_is_inter(d);
    read_tx_size(d, !b.skip || !b.is_inter);
    if (b.is_inter)
      inter_block_mode_info(d);
    else
      intra_block_mode_info(d);
  }

  uint8_t get_segment_id() const {
    uint32_t bw = vp9t_num_8x8_wide[b.mi_size], bh = vp9t_num_8x8_high[b.mi_size];
    uint32_t xmis = std::min(mi_cols - b.mi_col, bw), ymis = std::min(mi_rows - b.mi_row, bh);
    uint8_t seg = 7;
    for (uint32_t y = 0; y < ymis; ++y)
      for (uint32_t x = 0; x < xmis; ++x) {
        size_t i = (size_t)(b.mi_row + y) * mi_cols + b.mi_col + x;
        uint8_t v = i < f->prev_seg_len ? f->prev_seg_ids[i] : 0;
        if (v < seg) seg = v;
      }
    return seg;
  }

  void inter_segment_id(C& d) {
    const SegParams& seg = *f->seg;
    if (!seg.enabled) {
      b.segment_id = 0;
      return;
    }
    uint8_t predicted = get_segment_id();
    if (!seg.update_map) {
      b.segment_id = predicted;
      return;
    }
    if (seg.temporal_update) {
      int ctx = left_seg_pred[b.mi_row] + f->above_seg_pred[b.mi_col];
      bool pred = d.bit(seg.pred_probs[ctx], [&] { return eb_->segment_id == predicted; });
      b.segment_id = pred ? predicted
                          : (uint8_t)d.tree(SEGMENT_TREE, [&](int n) { return seg.tree_probs[n]; },
                                            [&] { return (int)eb_->segment_id; });
      uint32_t bw = vp9t_num_8x8_wide[b.mi_size], bh = vp9t_num_8x8_high[b.mi_size];
      for (uint32_t i = 0; i < bw; ++i) f->above_seg_pred[b.mi_col + i] = pred;
      for (uint32_t i = 0; i < bh; ++i) left_seg_pred[b.mi_row + i] = pred;
    } else {
      b.segment_id = (uint8_t)d.tree(SEGMENT_TREE, [&](int n) { return seg.tree_probs[n]; },
                                     [&] { return (int)eb_->segment_id; });
    }
  }

  void left_ref(int8_t out[2]) const {
    if (b.left) {
      out[0] = b.left->ref_frame[0];
      out[1] = b.left->ref_frame[1];
    } else {
      out[0] = INTRA_FRAME;
      out[1] = NONE_FRAME;
    }
  }
  void above_ref(int8_t out[2]) const {
    if (b.above) {
      out[0] = b.above->ref_frame[0];
      out[1] = b.above->ref_frame[1];
    } else {
      out[0] = INTRA_FRAME;
      out[1] = NONE_FRAME;
    }
  }

  void read_is_inter(C& d) {
    const SegParams& seg = *f->seg;
    if (seg.active(b.segment_id, SEG_LVL_REF_FRAME)) {
      b.is_inter = seg.feature_data[b.segment_id][SEG_LVL_REF_FRAME] != INTRA_FRAME;
    } else {
      int8_t l[2], a[2];
      left_ref(l);
      above_ref(a);
      bool left_intra = l[0] <= INTRA_FRAME, above_intra = a[0] <= INTRA_FRAME;
      bool au = b.avail_u, al = b.avail_l;
      int ctx;
      if (au && al)
        ctx = (left_intra && above_intra) ? 3 : (left_intra || above_intra) ? 1 : 0;
      else if (au || al)
        ctx = 2 * (au ? above_intra : left_intra);
      else
        ctx = 0;
      b.is_inter = d.bit(f->probs->is_inter[ctx], [&] { return eb_->is_inter; });
      counts.is_inter[ctx][b.is_inter ? 1 : 0] += 1;
    }
  }

  void intra_block_mode_info(C& d) {
    b.ref_frame[0] = INTRA_FRAME;
    b.ref_frame[1] = NONE_FRAME;
    if (b.mi_size >= BLOCK_8X8) {
      int ctx = vp9t_size_group[b.mi_size];
      const uint8_t* p = f->probs->y_mode[ctx];
      uint8_t mode = (uint8_t)d.tree(INTRA_MODE_TREE, [&](int n) { return p[n]; }, [&] { return (int)eb_->y_mode; });
      counts.intra_mode[ctx][mode] += 1;
      b.y_mode = mode;
      for (int i = 0; i < 4; ++i) b.sub_modes[i] = mode;
    } else {
      int n4w = vp9t_num_4x4_wide[b.mi_size], n4h = vp9t_num_4x4_high[b.mi_size];
      const uint8_t* p = f->probs->y_mode[0];
      uint8_t mode = DC_PRED;
      for (int idy = 0; idy < 2; idy += n4h)
        for (int idx = 0; idx < 2; idx += n4w) {
          mode = (uint8_t)d.tree(INTRA_MODE_TREE, [&](int n) { return p[n]; },
                                 [&] { return (int)eb_->sub_modes[idy * 2 + idx]; });
          counts.intra_mode[0][mode] += 1;
          for (int y2 = 0; y2 < n4h; ++y2)
            for (int x2 = 0; x2 < n4w; ++x2) b.sub_modes[(idy + y2) * 2 + idx + x2] = mode;
        }
      b.y_mode = mode;
    }
    const uint8_t* p = f->probs->uv_mode[b.y_mode];
    uint8_t uv = (uint8_t)d.tree(INTRA_MODE_TREE, [&](int n) { return p[n]; }, [&] { return (int)eb_->uv_mode; });
    counts.uv_mode[b.y_mode][uv] += 1;
    b.uv_mode = uv;
  }

  void inter_block_mode_info(C& d) {
    read_ref_frames(d);
    for (int j = 0; j < 2; ++j)
      if (b.ref_frame[j] > INTRA_FRAME) find_best_ref_mvs(j);
    bool is_compound = b.ref_frame[1] > INTRA_FRAME;
    if (f->seg->active(b.segment_id, SEG_LVL_SKIP))
      b.y_mode = ZEROMV;
    else if (b.mi_size >= BLOCK_8X8)
      b.y_mode = (uint8_t)(NEARESTMV + read_inter_mode(d));
    if (h->interpolation_filter == SWITCHABLE) {
      int8_t l[2], a[2];
      left_ref(l);
      above_ref(a);
      int left_interp = (b.avail_l && l[0] > INTRA_FRAME) ? b.left->interp_filter : 3;
      int above_interp = (b.avail_u && a[0] > INTRA_FRAME) ? b.above->interp_filter : 3;
      int ctx;
      if (left_interp == above_interp)
        ctx = left_interp;
      else if (left_interp == 3 && above_interp != 3)
        ctx = above_interp;
      else if (left_interp != 3 && above_interp == 3)
        ctx = left_interp;
      else
        ctx = 3;
      const uint8_t* p = f->probs->interp_filter[ctx];
      int fl = d.tree(INTERP_FILTER_TREE, [&](int n) { return p[n]; }, [&] { return (int)eb_->interp_filter; });
      counts.interp_filter[ctx][fl] += 1;
      b.interp_filter = (uint8_t)fl;
    } else {
      b.interp_filter = h->interpolation_filter;
    }
    int nrefs = 1 + (is_compound ? 1 : 0);
    if (b.mi_size < BLOCK_8X8) {
      int n4w = vp9t_num_4x4_wide[b.mi_size], n4h = vp9t_num_4x4_high[b.mi_size];
      for (int idy = 0; idy < 2; idy += n4h)
        for (int idx = 0; idx < 2; idx += n4w) {
          b.y_mode = (uint8_t)(NEARESTMV + read_inter_mode(d));
          if (b.y_mode == NEARESTMV || b.y_mode == NEARMV)
            for (int j = 0; j < nrefs; ++j) append_sub8x8_mvs(idy * 2 + idx, j);
          assign_mv(d, is_compound);
          for (int y2 = 0; y2 < n4h; ++y2)
            for (int x2 = 0; x2 < n4w; ++x2) {
              int blk = (idy + y2) * 2 + idx + x2;
              for (int rl = 0; rl < nrefs; ++rl) b.block_mvs[rl][blk] = b.mv[rl];
            }
        }
    } else {
      assign_mv(d, is_compound);
      for (int rl = 0; rl < nrefs; ++rl)
        for (int k = 0; k < 4; ++k) b.block_mvs[rl][k] = b.mv[rl];
    }
  }

  int read_inter_mode(C& d) {
    int ctx = b.mode_context[b.ref_frame[0]];
    const uint8_t* p = f->probs->inter_mode[ctx];
    int v = d.tree(INTER_MODE_TREE, [&](int n) { return p[n]; }, [&] { return enc_->inter_mode(b, eb_) - NEARESTMV; });
    counts.inter_mode[ctx][v] += 1;
    return v;
  }

  void read_ref_frames(C& d) {
    const SegParams& seg = *f->seg;
    if (seg.active(b.segment_id, SEG_LVL_REF_FRAME)) {
      int rf = seg.feature_data[b.segment_id][SEG_LVL_REF_FRAME];
      if (rf < 1 || rf > 3) bitstream_error("segment reference feature names no inter frame");
      b.ref_frame[0] = (int8_t)rf;
      b.ref_frame[1] = NONE_FRAME;
      return;
    }
    int comp_mode;
    if (h->reference_mode == REFERENCE_MODE_SELECT) {
      int ctx = comp_mode_ctx();
      bool v = d.bit(f->probs->comp_mode[ctx], [&] { return eb_->ref_frame[1] > INTRA_FRAME; });
      counts.comp_mode[ctx][v ? 1 : 0] += 1;
      comp_mode = v ? COMPOUND_REFERENCE : SINGLE_REFERENCE;
    } else {
      comp_mode = h->reference_mode;
    }
    if (comp_mode == COMPOUND_REFERENCE) {
      int idx = h->ref_frame_sign_bias[h->comp_fixed_ref] ? 1 : 0;
      int ctx = comp_ref_ctx();
      bool v = d.bit(f->probs->comp_ref[ctx],
                     [&] { return eb_->ref_frame[1 - idx] == h->comp_var_ref[1]; });
      counts.comp_ref[ctx][v ? 1 : 0] += 1;
      b.ref_frame[idx] = h->comp_fixed_ref;
      b.ref_frame[1 - idx] = h->comp_var_ref[v ? 1 : 0];
    } else {
      int ctx = single_ref_p1_ctx();
      bool p1 = d.bit(f->probs->single_ref[ctx][0], [&] { return eb_->ref_frame[0] != LAST_FRAME; });
      counts.single_ref[ctx][0][p1 ? 1 : 0] += 1;
      if (p1) {
        int ctx2 = single_ref_p2_ctx();
        bool p2 = d.bit(f->probs->single_ref[ctx2][1], [&] { return eb_->ref_frame[0] == ALTREF_FRAME; });
        counts.single_ref[ctx2][1][p2 ? 1 : 0] += 1;
        b.ref_frame[0] = p2 ? ALTREF_FRAME : GOLDEN_FRAME;
      } else {
        b.ref_frame[0] = LAST_FRAME;
      }
      b.ref_frame[1] = NONE_FRAME;
    }
  }

  int comp_mode_ctx() const {
    bool au = b.avail_u, al = b.avail_l;
    int8_t a[2], l[2];
    above_ref(a);
    left_ref(l);
    bool a_single = a[1] <= NONE_FRAME, l_single = l[1] <= NONE_FRAME;
    bool a_intra = a[0] <= INTRA_FRAME, l_intra = l[0] <= INTRA_FRAME;
    int8_t fixed = h->comp_fixed_ref;
    if (au && al) {
      if (a_single && l_single) return (a[0] == fixed) ^ (l[0] == fixed);
      if (a_single) return 2 + (a[0] == fixed || a_intra);
      if (l_single) return 2 + (l[0] == fixed || l_intra);
      return 4;
    }
    if (au) return a_single ? (a[0] == fixed) : 3;
    if (al) return l_single ? (l[0] == fixed) : 3;
    return 1;
  }

  int comp_ref_ctx() const {
    bool au = b.avail_u, al = b.avail_l;
    int8_t a[2], l[2];
    above_ref(a);
    left_ref(l);
    bool a_single = a[1] <= NONE_FRAME, l_single = l[1] <= NONE_FRAME;
    bool a_intra = a[0] <= INTRA_FRAME, l_intra = l[0] <= INTRA_FRAME;
    int fix_ref_idx = h->ref_frame_sign_bias[h->comp_fixed_ref] ? 1 : 0;
    int var_ref_idx = 1 - fix_ref_idx;
    int8_t var1 = h->comp_var_ref[1], var0 = h->comp_var_ref[0], fixed = h->comp_fixed_ref;
    if (au && al) {
      if (a_intra && l_intra) return 2;
      if (l_intra) return a_single ? 1 + 2 * (a[0] != var1) : 1 + 2 * (a[var_ref_idx] != var1);
      if (a_intra) return l_single ? 1 + 2 * (l[0] != var1) : 1 + 2 * (l[var_ref_idx] != var1);
      int8_t vrfa = a_single ? a[0] : a[var_ref_idx];
      int8_t vrfl = l_single ? l[0] : l[var_ref_idx];
      if (vrfa == vrfl && var1 == vrfa) return 0;
      if (l_single && a_single) {
        if ((vrfa == fixed && vrfl == var0) || (vrfl == fixed && vrfa == var0)) return 4;
        if (vrfa == vrfl) return 3;
        return 1;
      }
      if (l_single || a_single) {
        int8_t vrfc = l_single ? vrfa : vrfl;
        int8_t rfs = a_single ? vrfa : vrfl;
        if (vrfc == var1 && rfs != var1) return 1;
        if (rfs == var1 && vrfc != var1) return 2;
        return 4;
      }
      if (vrfa == vrfl) return 4;
      return 2;
    }
    if (au) {
      if (a_intra) return 2;
      if (a_single) return 3 * (a[0] != var1);
      return 4 * (a[var_ref_idx] != var1);
    }
    if (al) {
      if (l_intra) return 2;
      if (l_single) return 3 * (l[0] != var1);
      return 4 * (l[var_ref_idx] != var1);
    }
    return 2;
  }

  int single_ref_p1_ctx() const {
    bool au = b.avail_u, al = b.avail_l;
    int8_t a[2], l[2];
    above_ref(a);
    left_ref(l);
    bool a_single = a[1] <= NONE_FRAME, l_single = l[1] <= NONE_FRAME;
    bool a_intra = a[0] <= INTRA_FRAME, l_intra = l[0] <= INTRA_FRAME;
    const int8_t LF = LAST_FRAME;
    if (au && al) {
      if (a_intra && l_intra) return 2;
      if (l_intra) return a_single ? 4 * (a[0] == LF) : 1 + (a[0] == LF || a[1] == LF);
      if (a_intra) return l_single ? 4 * (l[0] == LF) : 1 + (l[0] == LF || l[1] == LF);
      if (a_single && l_single) return 2 * (a[0] == LF) + 2 * (l[0] == LF);
      if (!a_single && !l_single) return 1 + (a[0] == LF || a[1] == LF || l[0] == LF || l[1] == LF);
      int8_t rfs = a_single ? a[0] : l[0];
      int8_t crf1 = a_single ? l[0] : a[0];
      int8_t crf2 = a_single ? l[1] : a[1];
      if (rfs == LF) return 3 + (crf1 == LF || crf2 == LF);
      return (crf1 == LF || crf2 == LF);
    }
    if (au) {
      if (a_intra) return 2;
      if (a_single) return 4 * (a[0] == LF);
      return 1 + (a[0] == LF || a[1] == LF);
    }
    if (al) {
      if (l_intra) return 2;
      if (l_single) return 4 * (l[0] == LF);
      return 1 + (l[0] == LF || l[1] == LF);
    }
    return 2;
  }

  int single_ref_p2_ctx() const {
    bool au = b.avail_u, al = b.avail_l;
    int8_t a[2], l[2];
    above_ref(a);
    left_ref(l);
    bool a_single = a[1] <= NONE_FRAME, l_single = l[1] <= NONE_FRAME;
    bool a_intra = a[0] <= INTRA_FRAME, l_intra = l[0] <= INTRA_FRAME;
    const int8_t LF = LAST_FRAME, GF = GOLDEN_FRAME, AF = ALTREF_FRAME;
    if (au && al) {
      if (a_intra && l_intra) return 2;
      if (l_intra) {
        if (a_single) return a[0] == LF ? 3 : 4 * (a[0] == GF);
        return 1 + 2 * (a[0] == GF || a[1] == GF);
      }
      if (a_intra) {
        if (l_single) return l[0] == LF ? 3 : 4 * (l[0] == GF);
        return 1 + 2 * (l[0] == GF || l[1] == GF);
      }
      if (a_single && l_single) {
        if (a[0] == LF && l[0] == LF) return 3;
        if (a[0] == LF) return 4 * (l[0] == GF);
        if (l[0] == LF) return 4 * (a[0] == GF);
        return 2 * (a[0] == GF) + 2 * (l[0] == GF);
      }
      if (!a_single && !l_single) {
        if (a[0] == l[0] && a[1] == l[1]) return 3 * (a[0] == GF || a[1] == GF);
        return 2;
      }
      int8_t rfs = a_single ? a[0] : l[0];
      int8_t crf1 = a_single ? l[0] : a[0];
      int8_t crf2 = a_single ? l[1] : a[1];
      if (rfs == GF) return 3 + (crf1 == GF || crf2 == GF);
      if (rfs == AF) return (crf1 == GF || crf2 == GF);
      return 1 + 2 * (crf1 == GF || crf2 == GF);
    }
    if (au) {
      if (a_intra || (a[0] == LF && a_single)) return 2;
      if (a_single) return 4 * (a[0] == GF);
      return 3 * (a[0] == GF || a[1] == GF);
    }
    if (al) {
      if (l_intra || (l[0] == LF && l_single)) return 2;
      if (l_single) return 4 * (l[0] == GF);
      return 3 * (l[0] == GF || l[1] == GF);
    }
    return 2;
  }

  void assign_mv(C& d, bool is_compound) {
    b.mv[1] = Mv{0, 0};
    for (int i = 0; i < 1 + (is_compound ? 1 : 0); ++i) {
      switch (b.y_mode) {
        case NEWMV: b.mv[i] = read_mv(d, i); break;
        case NEARESTMV: b.mv[i] = b.nearest_mv[i]; break;
        case NEARMV: b.mv[i] = b.near_mv[i]; break;
        default: b.mv[i] = Mv{0, 0}; break;
      }
    }
  }

  Mv read_mv(C& d, int r) {
    Mv best = b.best_mv[r];
    bool use_hp = h->allow_high_precision_mv && use_mv_hp(best);
    int32_t diff[2] = {0, 0};
    const uint8_t* p = f->probs->mv_joint;
    int32_t want[2] = {0, 0};
    if (C::kEncode) {
      want[0] = eb_->mv[r].r - best.r;
      want[1] = eb_->mv[r].c - best.c;
    }
    int joint = d.tree(MV_JOINT_TREE, [&](int n) { return p[n]; },
                       [&] { return (want[0] != 0 ? 2 : 0) | (want[1] != 0 ? 1 : 0); });
    counts.mv_joint[joint] += 1;
    if (joint == MV_JOINT_HZVNZ || joint == MV_JOINT_HNZVNZ) diff[0] = read_mv_component(d, 0, use_hp, want[0]);
    if (joint == MV_JOINT_HNZVZ || joint == MV_JOINT_HNZVNZ) diff[1] = read_mv_component(d, 1, use_hp, want[1]);
    return Mv{best.r + diff[0], best.c + diff[1]};
  }

  int32_t read_mv_component(C& d, int comp, bool use_hp, int32_t want) {
    const Probs& pr = *f->probs;
    // Encoding: the class, and the bits of the magnitude within it.
    int w_cls = 0, w_c0 = 0, w_fr = 0, w_hp = 0, w_dd = 0;
    if (C::kEncode) {
      int32_t z = (want < 0 ? -want : want) - 1;
      if (z < 16) {
        w_c0 = z >> 3;
        w_fr = (z >> 1) & 3;
        w_hp = z & 1;
      } else {
        w_cls = 1;
        while ((2 << (w_cls + 3)) <= z) ++w_cls;
        int32_t rem = z - (2 << (w_cls + 2));
        w_dd = rem >> 3;
        w_fr = (rem >> 1) & 3;
        w_hp = rem & 1;
      }
    }
    bool sign = d.bit(pr.mv_sign[comp], [&] { return want < 0; });
    counts.mv_sign[comp][sign ? 1 : 0] += 1;
    const uint8_t* pc = pr.mv_class[comp];
    int cls = d.tree(MV_CLASS_TREE, [&](int n) { return pc[n]; }, [&] { return w_cls; });
    counts.mv_class[comp][cls] += 1;
    int32_t mag;
    if (cls == 0) {
      int c0 = d.bit(pr.mv_class0_bit[comp], [&] { return w_c0 != 0; }) ? 1 : 0;
      counts.mv_class0_bit[comp][c0] += 1;
      const uint8_t* pf = pr.mv_class0_fr[comp][c0];
      int fr = d.tree(MV_FR_TREE, [&](int n) { return pf[n]; }, [&] { return w_fr; });
      counts.mv_class0_fr[comp][c0][fr] += 1;
      int hp = use_hp ? (d.bit(pr.mv_class0_hp[comp], [&] { return w_hp != 0; }) ? 1 : 0) : 1;
      counts.mv_class0_hp[comp][hp] += 1;
      mag = ((c0 << 3) | (fr << 1) | hp) + 1;
    } else {
      int32_t dd = 0;
      for (int i = 0; i < cls; ++i) {
        int bit = d.bit(pr.mv_bits[comp][i], [&] { return ((w_dd >> i) & 1) != 0; }) ? 1 : 0;
        counts.mv_bits[comp][i][bit] += 1;
        dd |= bit << i;
      }
      int32_t m0 = 2 << (cls + 2);
      const uint8_t* pf = pr.mv_fr[comp];
      int fr = d.tree(MV_FR_TREE, [&](int n) { return pf[n]; }, [&] { return w_fr; });
      counts.mv_fr[comp][fr] += 1;
      int hp = use_hp ? (d.bit(pr.mv_hp[comp], [&] { return w_hp != 0; }) ? 1 : 0) : 1;
      counts.mv_hp[comp][hp] += 1;
      mag = m0 + ((dd << 3) | (fr << 1) | hp) + 1;
    }
    return sign ? -mag : mag;
  }

  // ---- Motion vector prediction (spec 6.5; reference mvpred.rs) ----

  struct Search {
    int count;
    Mv list[2];
    Mv cand_mv[2];
    int8_t cand_frame[2];
    void add(int ref_list) {
      if (count >= 2) return;
      if (count > 0 && cand_mv[ref_list] == list[0]) return;
      list[count++] = cand_mv[ref_list];
    }
  };

  bool is_inside(int32_t r, int32_t c) const {
    return r >= 0 && r < (int32_t)mi_rows && c >= (int32_t)mi_col_start && c < (int32_t)mi_col_end;
  }

  void get_block_mv(Search& s, int32_t r, int32_t c, int ref_list, bool use_prev) const {
    if (use_prev) {
      size_t idx = (size_t)r * mi_cols + c;
      const PrevMv& p = f->prev_mvs[idx];
      s.cand_mv[ref_list] = p.mv[ref_list];
      s.cand_frame[ref_list] = p.ref_frame[ref_list];
    } else {
      const MiInfo& m = mi_at(r, c);
      s.cand_mv[ref_list] = m.mv[ref_list][3];
      s.cand_frame[ref_list] = m.ref_frame[ref_list];
    }
  }

  void if_same_ref_frame_add(Search& s, int32_t r, int32_t c, int8_t ref_frame, bool use_prev) const {
    for (int j = 0; j < 2; ++j) {
      get_block_mv(s, r, c, j, use_prev);
      if (s.cand_frame[j] == ref_frame) {
        s.add(j);
        return;
      }
    }
  }

  void scale_mv(Search& s, int ref_list, int8_t ref_frame) const {
    int8_t cand = s.cand_frame[ref_list];
    if (h->ref_frame_sign_bias[cand] != h->ref_frame_sign_bias[ref_frame]) {
      s.cand_mv[ref_list].r *= -1;
      s.cand_mv[ref_list].c *= -1;
    }
  }

  void if_diff_ref_frame_add(Search& s, int32_t r, int32_t c, int8_t ref_frame, bool use_prev) const {
    for (int j = 0; j < 2; ++j) get_block_mv(s, r, c, j, use_prev);
    bool mvs_same = s.cand_mv[0] == s.cand_mv[1];
    if (s.cand_frame[0] > INTRA_FRAME && s.cand_frame[0] != ref_frame) {
      scale_mv(s, 0, ref_frame);
      s.add(0);
    }
    if (s.cand_frame[1] > INTRA_FRAME && s.cand_frame[1] != ref_frame && !mvs_same) {
      scale_mv(s, 1, ref_frame);
      s.add(1);
    }
  }

  int32_t clamp_mv_row(int32_t v, int32_t border) const {
    int32_t bh = vp9t_num_8x8_high[b.mi_size];
    int32_t mi_row = (int32_t)b.mi_row;
    int32_t to_top = -((mi_row * 8) * 8);
    int32_t to_bottom = (((int32_t)mi_rows - bh - mi_row) * 8) * 8;
    int32_t lo = to_top - border, hi = to_bottom + border;
    return v < lo ? lo : (v > hi ? hi : v);
  }

  int32_t clamp_mv_col(int32_t v, int32_t border) const {
    int32_t bw = vp9t_num_8x8_wide[b.mi_size];
    int32_t mi_col = (int32_t)b.mi_col;
    int32_t to_left = -((mi_col * 8) * 8);
    int32_t to_right = (((int32_t)mi_cols - bw - mi_col) * 8) * 8;
    int32_t lo = to_left - border, hi = to_right + border;
    return v < lo ? lo : (v > hi ? hi : v);
  }

  // find_mv_refs( refFrame, block ) (spec 6.5.1).
  void find_mv_refs(int8_t ref_frame, int block, Mv out[2]) {
    Search s;
    s.count = 0;
    s.list[0] = s.list[1] = Mv{0, 0};
    s.cand_mv[0] = s.cand_mv[1] = Mv{0, 0};
    s.cand_frame[0] = s.cand_frame[1] = 0;
    int context_counter = 0;
    const int8_t(*search)[2] = vp9t_mv_ref_blocks[b.mi_size];
    int32_t mi_row = (int32_t)b.mi_row, mi_col = (int32_t)b.mi_col;
    for (int i = 0; i < 2; ++i) {
      int32_t r = mi_row + search[i][0], c = mi_col + search[i][1];
      if (is_inside(r, c)) {
        const MiInfo& m = mi_at(r, c);
        context_counter += vp9t_mode_2_counter[m.y_mode];
        for (int j = 0; j < 2; ++j) {
          if (m.ref_frame[j] == ref_frame) {
            int idx = block >= 0 ? vp9t_idx_n_column_to_subblock[block][search[i][1] == 0 ? 1 : 0] : 3;
            s.cand_mv[j] = m.mv[j][idx];
            s.add(j);
            break;
          }
        }
      }
    }
    for (int i = 2; i < 8; ++i) {
      int32_t r = mi_row + search[i][0], c = mi_col + search[i][1];
      if (is_inside(r, c)) if_same_ref_frame_add(s, r, c, ref_frame, false);
    }
    bool use_prev = f->prev_mvs != nullptr;
    if (use_prev) if_same_ref_frame_add(s, mi_row, mi_col, ref_frame, true);
    for (int i = 0; i < 8; ++i) {
      int32_t r = mi_row + search[i][0], c = mi_col + search[i][1];
      if (is_inside(r, c)) if_diff_ref_frame_add(s, r, c, ref_frame, false);
    }
    if (use_prev) if_diff_ref_frame_add(s, mi_row, mi_col, ref_frame, true);
    b.mode_context[ref_frame] = COUNTER_TO_CONTEXT[context_counter];
    for (int i = 0; i < 2; ++i) {
      s.list[i].r = clamp_mv_row(s.list[i].r, MV_BORDER);
      s.list[i].c = clamp_mv_col(s.list[i].c, MV_BORDER);
    }
    out[0] = s.list[0];
    out[1] = s.list[1];
  }

  // find_best_ref_mvs( refList ) (spec 6.5.12).
  void find_best_ref_mvs(int ref_list) {
    Mv list[2];
    find_mv_refs(b.ref_frame[ref_list], -1, list);
    int32_t border = (BORDERINPIXELS - INTERP_EXTEND) << 3;
    for (int i = 0; i < 2; ++i) {
      int32_t dr = list[i].r, dc = list[i].c;
      if (!h->allow_high_precision_mv || !use_mv_hp(list[i])) {
        if (dr & 1) dr += dr > 0 ? -1 : 1;
        if (dc & 1) dc += dc > 0 ? -1 : 1;
      }
      list[i].r = clamp_mv_row(dr, border);
      list[i].c = clamp_mv_col(dc, border);
    }
    b.nearest_mv[ref_list] = list[0];
    b.near_mv[ref_list] = list[1];
    b.best_mv[ref_list] = list[0];
  }

  // append_sub8x8_mvs( block, refList ) (spec 6.5.14).
  void append_sub8x8_mvs(int block, int ref_list) {
    Mv list[2];
    find_mv_refs(b.ref_frame[ref_list], block, list);
    Mv sub[2] = {{0, 0}, {0, 0}};
    int dst = 0;
    const Mv* bm = b.block_mvs[ref_list];
    if (block == 0) {
      sub[0] = list[0];
      sub[1] = list[1];
      dst = 2;
    } else if (block <= 2) {
      sub[dst++] = bm[0];
    } else {
      sub[dst++] = bm[2];
      for (int idx = 1; idx >= 0 && dst < 2; --idx) {
        if (bm[idx] != sub[0]) sub[dst++] = bm[idx];
      }
    }
    for (int n = 0; n < 2 && dst < 2; ++n) {
      if (list[n] != sub[0]) sub[dst++] = list[n];
    }
    if (dst < 2) sub[dst] = Mv{0, 0};
    b.nearest_mv[ref_list] = sub[0];
    b.near_mv[ref_list] = sub[1];
  }

  // ---- Residual (spec 6.4.21 - 6.4.26) ----

  uint8_t uv_tx_size() const {
    if (b.mi_size < BLOCK_8X8) return TX_4X4;
    int sx = h->legacy_uv ? 1 : (int)ss_x, sy = h->legacy_uv ? 1 : (int)ss_y;
    uint8_t uv = SS_SIZE_LOOKUP[b.mi_size][sx][sy];
    uint8_t m = MAX_TXSIZE_LOOKUP[uv];
    return b.tx_size < m ? b.tx_size : m;
  }

  uint8_t tx_type(int plane, int tx_sz, int block_idx) const {
    if (plane > 0 || tx_sz == TX_32X32) return DCT_DCT;
    if (tx_sz == TX_4X4) {
      if (h->lossless || b.is_inter) return DCT_DCT;
      return MODE2TXFM_MAP[b.mi_size < BLOCK_8X8 ? b.sub_modes[block_idx] : b.y_mode];
    }
    return MODE2TXFM_MAP[b.y_mode];
  }

  void check_refs() const {
    int n = 1 + (b.ref_frame[1] > INTRA_FRAME ? 1 : 0);
    for (int i = 0; i < n; ++i) {
      int rf = b.ref_frame[i];
      if (!f->ref_scale_ok[rf - LAST_FRAME]) bitstream_error("reference frame scaled beyond 2:1 / 1:16");
    }
  }

  void residual(C& d) {
    uint8_t bsize = b.mi_size < BLOCK_8X8 ? BLOCK_8X8 : b.mi_size;
    for (int plane = 0; plane < 3; ++plane) {
      int tx_sz = plane > 0 ? uv_tx_size() : b.tx_size;
      int step = 1 << tx_sz;
      int sx = plane > 0 ? (int)ss_x : 0, sy = plane > 0 ? (int)ss_y : 0;
      uint8_t plane_sz = SS_SIZE_LOOKUP[bsize][sx][sy];
      if (plane_sz == BLOCK_INVALID) bitstream_error("invalid chroma block size");
      int n4w = vp9t_num_4x4_wide[plane_sz], n4h = vp9t_num_4x4_high[plane_sz];
      uint32_t base_x = (b.mi_col * 8) >> sx, base_y = (b.mi_row * 8) >> sy;
      if (b.is_inter && plane == 0) check_refs();
      uint32_t max_x = (mi_cols * 8) >> sx, max_y = (mi_rows * 8) >> sy;
      int block_idx = 0;
      uint8_t* an = f->above_nonzero[plane];
      uint8_t* ln = left_nonzero[plane].data();
      for (int y = 0; y < n4h; y += step) {
        for (int x = 0; x < n4w; x += step) {
          uint32_t start_x = base_x + 4 * x, start_y = base_y + 4 * y;
          bool nonzero = false;
          if (start_x < max_x && start_y < max_y) {
            if (!b.skip) {
              int eob = tokens(d, plane, start_x, start_y, tx_sz, block_idx);
              nonzero = eob > 0;
            }
          }
          for (int i = 0; i < step; ++i) {
            an[(start_x >> 2) + i] = nonzero;
            ln[(start_y >> 2) + i] = nonzero;
          }
          ++block_idx;
        }
      }
    }
  }

  // `want` (encoding): the magnitude to write.
  static int32_t read_coef(C& d, int token, uint32_t bit_depth, int32_t want) {
    int cat = EXTRA_BITS[token][0], num_extra = EXTRA_BITS[token][1];
    int32_t coef = EXTRA_BITS[token][2];
    const int32_t rem = want - coef;
    if (token == DCT_VAL_CAT6) {
      for (int e = 0; e < (int)bit_depth - 8; ++e) {
        const int sh = 5 + (int)bit_depth - e;
        int32_t high = d.bit(255, [&] { return ((rem >> sh) & 1) != 0; }) ? 1 : 0;
        coef += high << sh;
      }
    }
    const uint8_t* probs = CAT_PROBS[cat];
    for (int e = 0; e < num_extra; ++e) {
      const int sh = num_extra - 1 - e;
      int32_t bit = d.bit(probs[e], [&] { return ((rem >> sh) & 1) != 0; }) ? 1 : 0;
      coef += bit << sh;
    }
    return coef;
  }

  // The token loop of tokens() for decoding, with the bool decoder's state
  // in locals and the coefficient words written through a raw pointer;
  // returns the end of block.
  int tokens_dec(BoolDecoder& bdec, int tx_sz, int ptype, int ref_type, int ctx, const uint16_t* scan,
                 const uint16_t (*nb)[2], const uint8_t* bands, const uint64_t (*pk)[3], bool count, int seg_eob,
                 uint32_t bit_depth) {
    BoolDecoder::State r = bdec.save();
    const size_t base = coefs.size();
    uint32_t* out = coefs.grow(seg_eob);
    uint32_t n_out = 0;
    uint8_t* tc = token_cache;
    int c = 0;
    // The context as a shift into the band's words `w`.
    int sh = ctx * 8;
    const uint64_t* w = pk[bands[0]];
    while (true) {
      // more_coefs: read at the start and after every nonzero token.
      {
        const bool more = BoolDecoder::read(r, (uint8_t)(w[0] >> sh));
        if (count) counts.more_coefs[tx_sz][ptype][ref_type][bands[c]][sh >> 3][more ? 1 : 0] += 1;
        if (!more) break;
      }
      // A run of zero tokens; after a zero token no more_coefs is read.
      while (!BoolDecoder::read(r, (uint8_t)(w[1] >> sh))) {
        if (count) counts.token[tx_sz][ptype][ref_type][bands[c]][sh >> 3][0] += 1;
        tc[scan[c]] = 0;
        if (++c == seg_eob) goto done;
        w = pk[bands[c]];
        sh = ((1 + tc[nb[c][0]] + tc[nb[c][1]]) >> 1) * 8;
      }
      {
        const int pos = scan[c];
        int token;
        int32_t coef;
        const uint8_t p2 = (uint8_t)(w[2] >> sh);
        if (!BoolDecoder::read(r, p2)) {
          token = 1;  // ONE_TOKEN
          coef = 1;
          tc[pos] = 1;
        } else {
          // The rest of the token tree, its probabilities from one pareto row.
          const uint8_t* pp = pareto_row(p2);
          int n = 4;
          do {
            n = TOKEN_TREE[n + (int)BoolDecoder::read(r, pp[(n >> 1) - 2])];
          } while (n > 0);
          token = -n;
          tc[pos] = vp9t_energy_class[token];
          coef = EXTRA_BITS[token][2];
          const int num_extra = EXTRA_BITS[token][1];
          if (num_extra) {
            if (token == DCT_VAL_CAT6)
              for (int e = 0; e < (int)bit_depth - 8; ++e)
                coef += (int32_t)BoolDecoder::read(r, 255) << (5 + (int)bit_depth - e);
            const uint8_t* cat = CAT_PROBS[EXTRA_BITS[token][0]];
            for (int e = 0; e < num_extra; ++e) coef += (int32_t)BoolDecoder::read(r, cat[e]) << (num_extra - 1 - e);
          }
        }
        if (count) counts.token[tx_sz][ptype][ref_type][bands[c]][sh >> 3][token < 2 ? token : 2] += 1;
        const bool sign = BoolDecoder::read(r, 128);
        out[n_out++] = RV9_COEF_PACK(pos, sign ? -coef : coef);
      }
      if (++c == seg_eob) break;
      w = pk[bands[c]];
      sh = ((1 + tc[nb[c][0]] + tc[nb[c][1]]) >> 1) * 8;
    }
  done:
    coefs.shrink_to(base + n_out);
    bdec.load(r);
    return c;
  }

  // tokens() (spec 6.4.24): records the nonzero coefficients; returns eob.
  int tokens(C& d, int plane, uint32_t start_x, uint32_t start_y, int tx_sz, int block_idx) {
    int seg_eob = 16 << (tx_sz << 1);
    int ttype = tx_type(plane, tx_sz, block_idx);
    const uint16_t* scan = get_scan(tx_sz, ttype);
    int ref_type = b.is_inter ? 1 : 0;
    int ptype = plane > 0 ? 1 : 0;
    int sx = plane > 0 ? (int)ss_x : 0, sy = plane > 0 ? (int)ss_y : 0;
    uint32_t max_x4 = (2 * mi_cols) >> sx, max_y4 = (2 * mi_rows) >> sy;
    uint32_t x4 = start_x >> 2, y4 = start_y >> 2;
    uint8_t above = 0, left = 0;
    const uint8_t* an = f->above_nonzero[plane];
    const uint8_t* ln = left_nonzero[plane].data();
    for (int i = 0; i < (1 << tx_sz); ++i) {
      if (x4 + i < max_x4) above |= an[x4 + i];
      if (y4 + i < max_y4) left |= ln[y4 + i];
    }
    int ctx = above + left;
    const uint16_t(*nb)[2] = neighbor_tables().get(tx_sz, ttype);
    const uint8_t* bands = tx_sz == TX_4X4 ? vp9t_coefband_4x4 : vp9t_coefband_8x8plus;
    const uint8_t(*cp)[6][3] = f->probs->coef[tx_sz][ptype][ref_type];
    bool count = f->count_coefs;
    bool check_eob = true;
    int c = 0;
    uint32_t bd = h->bit_depth;
    rv9_tok t;
    t.x = (uint16_t)start_x;
    t.y = (uint16_t)start_y;
    t.plane = (uint8_t)plane;
    t.tx_size = (uint8_t)tx_sz;
    t.tx_type = (uint8_t)ttype;
    t.reserved = 0;
    t.coef_start = (uint32_t)coefs.size();
    // Encoding: the block's quantised coefficients (raster order) and eob.
    const int32_t* wc = nullptr;
    int w_eob = 0;
    if (C::kEncode) wc = enc_->tx_coefs(eb_, plane, start_x, start_y, tx_sz, scan, &w_eob);
    if constexpr (!C::kEncode) {
      c = tokens_dec(d.bd, tx_sz, ptype, ref_type, ctx, scan, nb, bands, coef_pk[tx_sz][ptype][ref_type], count,
                     seg_eob, bd);
    } else {
    for (; c < seg_eob; ++c) {
      int pos = scan[c];
      int band = bands[c];
      if (c > 0) ctx = (1 + token_cache[nb[c][0]] + token_cache[nb[c][1]]) >> 1;
      const uint8_t* probs = cp[band][ctx];
      if (check_eob) {
        bool more = d.bit(probs[0], [&] { return c < w_eob; });
        if (count) counts.more_coefs[tx_sz][ptype][ref_type][band][ctx][more ? 1 : 0] += 1;
        if (!more) break;
      }
      int token = d.tree(TOKEN_TREE, [&](int node) { return pareto(node, probs[(1 + node) < 2 ? (1 + node) : 2]); },
                         [&] { return token_of(wc[pos]); });
      if (count) counts.token[tx_sz][ptype][ref_type][band][ctx][token < 2 ? token : 2] += 1;
      token_cache[pos] = vp9t_energy_class[token];
      if (token == ZERO_TOKEN) {
        check_eob = false;
      } else {
        int32_t coef = read_coef(d, token, bd, wc ? (wc[pos] < 0 ? -wc[pos] : wc[pos]) : 0);
        bool sign = d.bit(128, [&] { return wc[pos] < 0; });
        coefs.push_back(RV9_COEF_PACK(pos, sign ? -coef : coef));
        check_eob = true;
      }
    }
    }
    if (c > 0) ++eob_total;
    t.eob = (uint16_t)c;
    t.n_coef = (uint16_t)(coefs.size() - t.coef_start);
    toks.push_back(t);
    return c;
  }
};


}  // namespace syn
}  // namespace rv9

// VP9 frame parsing: uncompressed and compressed headers, tiles, partitions,
// mode info, motion vector prediction and coefficient tokens, producing the
// records of rv9_records.h. A C++ restatement of the reference decoder's
// parse path: src/header.rs (headers), src/decoder/block.rs (tile, partition,
// block and token syntax), src/decoder/mvpred.rs (motion vector prediction),
// src/decoder/mod.rs:218-422 (the frame process and its state).
#include "parser.h"

#include <string.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <functional>
#include <memory>
#include <thread>

#include "../common/vp9_consts.h"
#include "../common/vp9_tables.h"
#include "bitreader.h"
#include "syntax.h"

namespace rv9 {
using namespace vp9;

namespace {
using namespace syn;

enum ResetKind { RESET_NONE, RESET_ALL, RESET_ONE };

void frame_sync_code(BitReader& r) {
  uint32_t a = r.f(8), b = r.f(8), c = r.f(8);
  if (a != 0x49 || b != 0x83 || c != 0x42) bitstream_error("invalid frame sync code");
}

void color_config(BitReader& r, FrameHeader& h) {
  h.bit_depth = h.profile >= 2 ? (r.flag() ? 12 : 10) : 8;
  h.color_space = (uint8_t)r.f(3);
  if (h.color_space != 7) {  // not sRGB
    h.color_range = r.flag();
    if (h.profile == 1 || h.profile == 3) {
      h.ss_x = r.f(1);
      h.ss_y = r.f(1);
      if (r.flag()) bitstream_error("reserved_zero is not zero");
      if (h.ss_x == 1 && h.ss_y == 1) bitstream_error("4:2:0 is not allowed in profiles 1 and 3");
    } else {
      h.ss_x = h.ss_y = 1;
    }
  } else {
    h.color_range = true;
    if (h.profile == 1 || h.profile == 3) {
      h.ss_x = h.ss_y = 0;
      if (r.flag()) bitstream_error("reserved_zero is not zero");
    } else {
      bitstream_error("sRGB is not allowed in profiles 0 and 2");
    }
  }
}

void frame_size(BitReader& r, FrameHeader& h) {
  h.width = r.f(16) + 1;
  h.height = r.f(16) + 1;
  h.compute_image_size();
}

void render_size(BitReader& r, FrameHeader& h) {
  if (r.flag()) {
    h.render_width = r.f(16) + 1;
    h.render_height = r.f(16) + 1;
  } else {
    h.render_width = h.width;
    h.render_height = h.height;
  }
}

int32_t read_delta_q(BitReader& r) { return r.flag() ? r.s(4) : 0; }
uint8_t read_prob(BitReader& r) { return r.flag() ? (uint8_t)r.f(8) : 255; }

// uncompressed_header() and trailing_bits() (reference src/header.rs:245-463).
FrameHeader parse_uncompressed(const uint8_t* data, size_t len, Persistent& st, ResetKind* reset,
                               int* reset_idx) {
  BitReader r(data, len);
  FrameHeader h;
  *reset = RESET_NONE;
  if (r.f(2) != 2) bitstream_error("frame_marker is not 2");
  uint32_t lo = r.f(1), hi = r.f(1);
  h.profile = (uint8_t)((hi << 1) + lo);
  if (h.profile == 3 && r.flag()) bitstream_error("reserved_zero is not zero");
  h.show_existing_frame = r.flag();
  if (h.show_existing_frame) {
    h.frame_to_show_map_idx = (uint8_t)r.f(3);
    r.byte_align();
    h.uncompressed_size = r.position() / 8;
    return h;
  }
  uint8_t last_frame_type = st.last_frame_type;
  h.frame_type = (uint8_t)r.f(1);
  h.show_frame = r.flag();
  h.error_resilient_mode = r.flag();
  h.last_frame_type = last_frame_type;
  st.last_frame_type = h.frame_type;
  h.bit_depth = st.bit_depth;
  h.ss_x = st.ss_x;
  h.ss_y = st.ss_y;
  h.color_space = st.color_space;
  h.color_range = st.color_range;
  if (h.frame_type == KEY_FRAME) {
    frame_sync_code(r);
    color_config(r, h);
    frame_size(r, h);
    render_size(r, h);
    h.refresh_frame_flags = 0xff;
    h.frame_is_intra = true;
  } else {
    h.intra_only = !h.show_frame ? r.flag() : false;
    h.frame_is_intra = h.intra_only;
    h.reset_frame_context = !h.error_resilient_mode ? (uint8_t)r.f(2) : 0;
    if (h.intra_only) {
      frame_sync_code(r);
      if (h.profile > 0) {
        color_config(r, h);
      } else {
        h.color_space = 1;
        h.ss_x = h.ss_y = 1;
        h.bit_depth = 8;
      }
      h.refresh_frame_flags = (uint8_t)r.f(8);
      frame_size(r, h);
      render_size(r, h);
    } else {
      h.refresh_frame_flags = (uint8_t)r.f(8);
      for (int i = 0; i < 3; ++i) {
        h.ref_frame_idx[i] = (uint8_t)r.f(3);
        h.ref_frame_sign_bias[LAST_FRAME + i] = r.flag();
      }
      bool found = false;
      for (int i = 0; i < 3; ++i) {
        if (r.flag()) {
          uint32_t w = st.ref_w[h.ref_frame_idx[i]], ht = st.ref_h[h.ref_frame_idx[i]];
          if (w == 0) bitstream_error("frame size taken from an empty reference slot");
          h.width = w;
          h.height = ht;
          found = true;
          break;
        }
      }
      if (!found)
        frame_size(r, h);
      else
        h.compute_image_size();
      render_size(r, h);
      h.allow_high_precision_mv = r.flag();
      h.interpolation_filter = r.flag() ? SWITCHABLE : LITERAL_TO_TYPE[r.f(2)];
    }
  }
  st.bit_depth = h.bit_depth;
  st.ss_x = h.ss_x;
  st.ss_y = h.ss_y;
  st.color_space = h.color_space;
  st.color_range = h.color_range;
  if (!h.error_resilient_mode) {
    h.refresh_frame_context = r.flag();
    h.frame_parallel_decoding_mode = r.flag();
  } else {
    h.refresh_frame_context = false;
    h.frame_parallel_decoding_mode = true;
  }
  h.frame_context_idx = (uint8_t)r.f(2);
  if (h.frame_is_intra || h.error_resilient_mode) {
    // setup_past_independence()
    h.past_independence = true;
    memset(st.seg.feature_data, 0, sizeof st.seg.feature_data);
    memset(st.seg.feature_enabled, 0, sizeof st.seg.feature_enabled);
    st.seg.abs_or_delta_update = false;
    st.lf.delta_enabled = true;
    st.lf.ref_deltas[0] = 1;
    st.lf.ref_deltas[1] = 0;
    st.lf.ref_deltas[2] = -1;
    st.lf.ref_deltas[3] = -1;
    st.lf.mode_deltas[0] = st.lf.mode_deltas[1] = 0;
    if (h.frame_type == KEY_FRAME || h.error_resilient_mode || h.reset_frame_context == 3)
      *reset = RESET_ALL;
    else if (h.reset_frame_context == 2)
      *reset = RESET_ONE;  // the context h.frame_context_idx, before it is zeroed
    *reset_idx = h.frame_context_idx;
    h.frame_context_idx = 0;
  }
  // loop_filter_params()
  st.lf.level = (uint8_t)r.f(6);
  st.lf.sharpness = (uint8_t)r.f(3);
  st.lf.delta_enabled = r.flag();
  if (st.lf.delta_enabled && r.flag()) {
    for (int i = 0; i < 4; ++i)
      if (r.flag()) st.lf.ref_deltas[i] = (int8_t)r.s(6);
    for (int i = 0; i < 2; ++i)
      if (r.flag()) st.lf.mode_deltas[i] = (int8_t)r.s(6);
  }
  // quantization_params()
  h.base_q_idx = (int32_t)r.f(8);
  h.delta_q_y_dc = read_delta_q(r);
  h.delta_q_uv_dc = read_delta_q(r);
  h.delta_q_uv_ac = read_delta_q(r);
  h.lossless = h.base_q_idx == 0 && h.delta_q_y_dc == 0 && h.delta_q_uv_dc == 0 && h.delta_q_uv_ac == 0;
  // segmentation_params()
  SegParams& seg = st.seg;
  seg.enabled = r.flag();
  seg.update_map = false;
  seg.temporal_update = false;
  if (seg.enabled) {
    seg.update_map = r.flag();
    if (seg.update_map) {
      for (int i = 0; i < 7; ++i) seg.tree_probs[i] = read_prob(r);
      seg.temporal_update = r.flag();
      for (int i = 0; i < 3; ++i) seg.pred_probs[i] = seg.temporal_update ? read_prob(r) : 255;
    }
    if (r.flag()) {
      seg.abs_or_delta_update = r.flag();
      for (int i = 0; i < MAX_SEGMENTS; ++i)
        for (int j = 0; j < 4; ++j) {
          int16_t v = 0;
          bool en = r.flag();
          seg.feature_enabled[i][j] = en;
          if (en) {
            v = (int16_t)r.f(vp9t_segmentation_feature_bits[j]);
            if (vp9t_segmentation_feature_signed[j] == 1 && r.flag()) v = (int16_t)-v;
          }
          seg.feature_data[i][j] = v;
        }
    }
  }
  // tile_info()
  uint32_t min_log2 = 0;
  while ((MAX_TILE_WIDTH_B64 << min_log2) < h.sb64_cols) ++min_log2;
  uint32_t max_log2 = 1;
  while ((h.sb64_cols >> max_log2) >= MIN_TILE_WIDTH_B64) ++max_log2;
  --max_log2;
  h.tile_cols_log2 = min_log2;
  while (h.tile_cols_log2 < max_log2) {
    if (r.flag())
      ++h.tile_cols_log2;
    else
      break;
  }
  h.tile_rows_log2 = r.f(1);
  if (h.tile_rows_log2 == 1) h.tile_rows_log2 += r.f(1);
  h.header_size_in_bytes = r.f(16);
  r.byte_align();
  h.uncompressed_size = r.position() / 8;
  return h;
}

// decode_term_subexp (spec 6.3.4).
uint32_t decode_term_subexp(BoolDecoder& d) {
  if (d.literal(1) == 0) return d.literal(4);
  if (d.literal(1) == 0) return d.literal(4) + 16;
  if (d.literal(1) == 0) return d.literal(5) + 32;
  uint32_t v = d.literal(7);
  if (v < 65) return v + 64;
  uint32_t bit = d.literal(1);
  return (v << 1) - 1 + bit;
}

int32_t inv_recenter_nonneg(int32_t v, int32_t m) {
  if (v > 2 * m) return v;
  if (v & 1) return m - ((v + 1) >> 1);
  return m + (v >> 1);
}

// inv_remap_prob (spec 6.3.5).
uint8_t inv_remap_prob(uint32_t delta, uint8_t prob) {
  int32_t v = vp9t_inv_map_table[delta < 254 ? delta : 254];
  int32_t m = (int32_t)prob - 1;
  int32_t r;
  if ((m << 1) <= 255)
    r = 1 + inv_recenter_nonneg(v, m);
  else
    r = 255 - inv_recenter_nonneg(v, 255 - 1 - m);
  return (uint8_t)(r < 1 ? 1 : (r > 255 ? 255 : r));
}

void diff_update_prob(BoolDecoder& d, uint8_t* p) {
  if (d.read(252)) {
    uint32_t delta = decode_term_subexp(d);
    *p = inv_remap_prob(delta, *p);
  }
}

void update_mv_prob(BoolDecoder& d, uint8_t* p) {
  if (d.read(252)) *p = (uint8_t)((d.literal(7) << 1) | 1);
}

// compressed_header() (reference src/header.rs:525-679).
void parse_compressed(const uint8_t* data, size_t len, FrameHeader& h, Probs& probs) {
  BoolDecoder d;
  if (len == 0) bitstream_error("boolean-coded partition of size 0");
  if (!d.init(data, len)) bitstream_error("boolean decoder marker bit is not 0");
  if (h.lossless) {
    h.tx_mode = ONLY_4X4;
  } else {
    h.tx_mode = (uint8_t)d.literal(2);
    if (h.tx_mode == ALLOW_32X32) h.tx_mode += (uint8_t)d.literal(1);
  }
  if (h.tx_mode == TX_MODE_SELECT) {
    for (int i = 0; i < 2; ++i) diff_update_prob(d, &probs.tx[1][i][0]);
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) diff_update_prob(d, &probs.tx[2][i][j]);
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 3; ++j) diff_update_prob(d, &probs.tx[3][i][j]);
  }
  int max_tx = TX_MODE_TO_BIGGEST_TX_SIZE[h.tx_mode];
  for (int tx = 0; tx <= max_tx; ++tx) {
    if (d.literal(1) == 1) {
      for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
          for (int k = 0; k < 6; ++k) {
            int max_l = k == 0 ? 3 : 6;
            for (int l = 0; l < max_l; ++l)
              for (int m = 0; m < 3; ++m) diff_update_prob(d, &probs.coef[tx][i][j][k][l][m]);
          }
    }
  }
  for (int i = 0; i < 3; ++i) diff_update_prob(d, &probs.skip[i]);
  h.reference_mode = SINGLE_REFERENCE;
  if (!h.frame_is_intra) {
    for (int i = 0; i < 7; ++i)
      for (int j = 0; j < 3; ++j) diff_update_prob(d, &probs.inter_mode[i][j]);
    if (h.interpolation_filter == SWITCHABLE)
      for (int j = 0; j < 4; ++j)
        for (int i = 0; i < 2; ++i) diff_update_prob(d, &probs.interp_filter[j][i]);
    for (int i = 0; i < 4; ++i) diff_update_prob(d, &probs.is_inter[i]);
    const bool* sb = h.ref_frame_sign_bias;
    bool compound_allowed = sb[2] != sb[1] || sb[3] != sb[1];
    if (compound_allowed) {
      if (d.literal(1) == 0) {
        h.reference_mode = SINGLE_REFERENCE;
      } else {
        h.reference_mode = d.literal(1) == 0 ? COMPOUND_REFERENCE : REFERENCE_MODE_SELECT;
        // setup_compound_reference_mode()
        if (sb[LAST_FRAME] == sb[GOLDEN_FRAME]) {
          h.comp_fixed_ref = ALTREF_FRAME;
          h.comp_var_ref[0] = LAST_FRAME;
          h.comp_var_ref[1] = GOLDEN_FRAME;
        } else if (sb[LAST_FRAME] == sb[ALTREF_FRAME]) {
          h.comp_fixed_ref = GOLDEN_FRAME;
          h.comp_var_ref[0] = LAST_FRAME;
          h.comp_var_ref[1] = ALTREF_FRAME;
        } else {
          h.comp_fixed_ref = LAST_FRAME;
          h.comp_var_ref[0] = GOLDEN_FRAME;
          h.comp_var_ref[1] = ALTREF_FRAME;
        }
      }
    }
    if (h.reference_mode == REFERENCE_MODE_SELECT)
      for (int i = 0; i < 5; ++i) diff_update_prob(d, &probs.comp_mode[i]);
    if (h.reference_mode != COMPOUND_REFERENCE)
      for (int i = 0; i < 5; ++i) {
        diff_update_prob(d, &probs.single_ref[i][0]);
        diff_update_prob(d, &probs.single_ref[i][1]);
      }
    if (h.reference_mode != SINGLE_REFERENCE)
      for (int i = 0; i < 5; ++i) diff_update_prob(d, &probs.comp_ref[i]);
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 9; ++j) diff_update_prob(d, &probs.y_mode[i][j]);
    for (int i = 0; i < 16; ++i)
      for (int j = 0; j < 3; ++j) diff_update_prob(d, &probs.partition[i][j]);
    for (int j = 0; j < 3; ++j) update_mv_prob(d, &probs.mv_joint[j]);
    for (int i = 0; i < 2; ++i) {
      update_mv_prob(d, &probs.mv_sign[i]);
      for (int j = 0; j < 10; ++j) update_mv_prob(d, &probs.mv_class[i][j]);
      update_mv_prob(d, &probs.mv_class0_bit[i]);
      for (int j = 0; j < 10; ++j) update_mv_prob(d, &probs.mv_bits[i][j]);
    }
    for (int i = 0; i < 2; ++i) {
      for (int j = 0; j < 2; ++j)
        for (int k = 0; k < 3; ++k) update_mv_prob(d, &probs.mv_class0_fr[i][j][k]);
      for (int k = 0; k < 3; ++k) update_mv_prob(d, &probs.mv_fr[i][k]);
    }
    if (h.allow_high_precision_mv)
      for (int i = 0; i < 2; ++i) {
        update_mv_prob(d, &probs.mv_class0_hp[i]);
        update_mv_prob(d, &probs.mv_hp[i]);
      }
  }
}

struct TileSpan {
  uint32_t row, col;
  const uint8_t* data;
  size_t size;
};

struct TileResult {
  Status st = ST_OK;
  std::string err;
  int failed_tile = -1;
  bool padding_ok = true;
};

// Working memory of one frame's tile parse.
struct TileWork {
  std::vector<MiInfo> mi;
  std::vector<uint8_t> above_nonzero[3];
  std::vector<uint8_t> above_partition, above_seg_pred;
  std::vector<TileCoder<DecCoder>> tile_decs;

  // Decodes all tiles of a frame into `tile_decs` (one per tile column).
  TileResult decode_tiles(const FrameHeader& h, const SegParams& seg, const Probs& probs, const PrevMv* prev,
                          const std::vector<uint8_t>* prev_seg, const bool ref_ok[3], const uint8_t* data,
                          size_t len, int threads) {
    TileResult res;
    size_t mi_len = (size_t)h.mi_rows * h.mi_cols;
    if (mi.size() < mi_len) mi.resize(mi_len);
    size_t n4w = h.sb64_cols * 16 + 16;
    for (int p = 0; p < 3; ++p) above_nonzero[p].assign(n4w, 0);
    above_partition.assign(h.sb64_cols * 8 + 8, 0);
    above_seg_pred.assign(h.sb64_cols * 8 + 8, 0);
    FrameCtx fc;
    fc.h = &h;
    fc.seg = &seg;
    fc.probs = &probs;
    fc.prev_seg_ids = prev_seg ? prev_seg->data() : nullptr;
    fc.prev_seg_len = prev_seg ? prev_seg->size() : 0;
    fc.prev_mvs = prev;
    fc.mi = mi.data();
    for (int p = 0; p < 3; ++p) fc.above_nonzero[p] = above_nonzero[p].data();
    fc.above_partition = above_partition.data();
    fc.above_seg_pred = above_seg_pred.data();
    for (int i = 0; i < 3; ++i) fc.ref_scale_ok[i] = ref_ok[i];
    fc.count_coefs = !h.error_resilient_mode && !h.frame_parallel_decoding_mode;
    // Split tiles (reference src/decoder/block.rs:1726-1763).
    uint32_t tile_cols = 1u << h.tile_cols_log2, tile_rows = 1u << h.tile_rows_log2;
    std::vector<TileSpan> tiles;
    size_t pos = 0;
    const char* size_err = nullptr;
    for (uint32_t row = 0; row < tile_rows && !size_err; ++row)
      for (uint32_t col = 0; col < tile_cols; ++col) {
        bool last = row == tile_rows - 1 && col == tile_cols - 1;
        size_t size;
        if (last) {
          size = len - pos;
        } else {
          if (pos + 4 > len) {
            size_err = "tile size runs past the end of the frame";
            break;
          }
          size = ((size_t)data[pos] << 24) | ((size_t)data[pos + 1] << 16) | ((size_t)data[pos + 2] << 8) | data[pos + 3];
          pos += 4;
        }
        if (pos + size > len) {
          size_err = "tile runs past the end of the frame";
          break;
        }
        tiles.push_back(TileSpan{row, col, data + pos, size});
        pos += size;
      }
    if (tile_decs.size() < tile_cols) tile_decs.resize(tile_cols);
    for (uint32_t c = 0; c < tile_cols; ++c) tile_decs[c].init(&fc);
    std::vector<TileResult> col_res(tile_cols);
    auto run_col = [&](uint32_t col) {
      TileCoder<DecCoder>& td = tile_decs[col];
      for (size_t i = 0; i < tiles.size(); ++i) {
        const TileSpan& t = tiles[i];
        if (t.col != col) continue;
        td.mi_row_start = tile_offset(t.row, h.mi_rows, h.tile_rows_log2);
        td.mi_row_end = tile_offset(t.row + 1, h.mi_rows, h.tile_rows_log2);
        td.mi_col_start = tile_offset(t.col, h.mi_cols, h.tile_cols_log2);
        td.mi_col_end = tile_offset(t.col + 1, h.mi_cols, h.tile_cols_log2);
        try {
          DecCoder d;
          if (t.size == 0) bitstream_error("boolean-coded partition of size 0");
          if (!d.bd.init(t.data, t.size)) bitstream_error("boolean decoder marker bit is not 0");
          td.decode_tile(d);
          td.padding_ok &= d.bd.padding_is_zero();
        } catch (const ParseError& e) {
          col_res[col].st = e.st;
          col_res[col].err = e.msg;
          col_res[col].failed_tile = (int)i;
          return;
        }
      }
    };
    int workers = threads;
    if (workers <= 0) workers = (int)std::thread::hardware_concurrency();
    if (workers > (int)tile_cols) workers = (int)tile_cols;
    if (workers > 1) {
      std::vector<std::thread> th;
      for (int w = 0; w < workers; ++w)
        th.emplace_back([&, w]() {
          for (uint32_t col = (uint32_t)w; col < tile_cols; col += (uint32_t)workers) run_col(col);
        });
      for (auto& t : th) t.join();
    } else {
      for (uint32_t col = 0; col < tile_cols; ++col) run_col(col);
    }
    // The first error in bitstream order wins.
    int first = -1;
    for (uint32_t c = 0; c < tile_cols; ++c)
      if (col_res[c].st != ST_OK && (first < 0 || col_res[c].failed_tile < col_res[first].failed_tile)) first = (int)c;
    if (first >= 0) return col_res[first];
    if (size_err) {
      res.st = ST_BITSTREAM;
      res.err = size_err;
      return res;
    }
    for (uint32_t c = 0; c < tile_cols; ++c) res.padding_ok &= tile_decs[c].padding_ok;
    return res;
  }
};

}  // namespace

// ---------------------------------------------------------------------------

// The decoder's frame-to-frame state. The previous frame's segment ids and
// motion vectors are shared, never written in place, so that a frame still
// parsing keeps reading the ones it started with.
struct FrameState {
  Persistent st;
  Probs contexts[4];
  SlotInfo slots[8];
  std::shared_ptr<std::vector<uint8_t>> prev_segment_ids = std::make_shared<std::vector<uint8_t>>();
  std::shared_ptr<std::vector<PrevMv>> prev_mvs = std::make_shared<std::vector<PrevMv>>();
  bool prev_external = false;  // the last frame's vectors are held by an external tile parser
  bool have_last_size = false;
  uint32_t last_w = 0, last_h = 0;
  bool last_show_frame = false;
  bool legacy_uv = false;
  FrameState() {
    for (auto& c : contexts) c.set_default();
  }
};

// One frame between its header (begin) and its state update (finish).
struct Parser::Job {
  Status st = ST_OK;  // of the header, then of the tiles
  std::string err;
  bool show_existing = false;
  FrameHeader h;
  SegParams seg;
  Probs probs;  // after the compressed header
  Probs pre;    // the context before it (the base of adaptation)
  bool ref_ok[3] = {true, true, true};
  std::shared_ptr<std::vector<uint8_t>> prev_seg;
  std::shared_ptr<std::vector<PrevMv>> prev_mvs;  // set when the frame uses them
  bool use_prev = false;       // the frame reads the previous frame's vectors
  bool use_prev_hdr = false;   // ... as its header and the last frame's decide (before the vectors' size check)
  bool prev_external = false;  // ... and an external tile parser holds them
  bool external = false;       // the tiles were parsed outside (finish_external)
  const uint8_t* tiles = nullptr;
  size_t tiles_len = 0;
  bool non420 = false;
  bool late_ctx = false;  // adapts and refreshes a context at finish
  FrameState snap;        // the state to restore if the tiles fail
  ParsedFrame out;
  std::unique_ptr<TileWork> work;
  TileResult tr;
  std::thread th;
  bool running = false;
  double seconds = 0;
  // A frame settled early by the pipeline keeps its result here.
  bool settled = false;
  Status settled_status = ST_OK;
  std::string settled_err;
  ParsedFrame settled_out;
};

struct Parser::Impl {
  FrameState s;
  std::vector<std::unique_ptr<TileWork>> spare;  // reusable working memory

  std::unique_ptr<TileWork> take_work() {
    if (spare.empty()) return std::unique_ptr<TileWork>(new TileWork);
    std::unique_ptr<TileWork> w = std::move(spare.back());
    spare.pop_back();
    return w;
  }
};

Parser::Parser() : impl_(new Impl) {}
Parser::~Parser() { delete impl_; }

static void fill_desc(const FrameHeader& h, const Persistent& st, const SlotInfo* slots, rv9_frame_desc* d) {
  memset(d, 0, sizeof *d);
  d->width = h.width;
  d->height = h.height;
  d->mi_cols = h.mi_cols;
  d->mi_rows = h.mi_rows;
  d->sb64_cols = h.sb64_cols;
  d->sb64_rows = h.sb64_rows;
  d->ss_x = (uint8_t)h.ss_x;
  d->ss_y = (uint8_t)h.ss_y;
  d->bit_depth = (uint8_t)h.bit_depth;
  d->lossless = h.lossless;
  d->legacy_uv = h.legacy_uv;
  d->frame_is_intra = h.frame_is_intra;
  d->show_frame = h.show_frame;
  d->tile_cols_log2 = (uint8_t)h.tile_cols_log2;
  d->base_q_idx = h.base_q_idx;
  d->delta_q_y_dc = h.delta_q_y_dc;
  d->delta_q_uv_dc = h.delta_q_uv_dc;
  d->delta_q_uv_ac = h.delta_q_uv_ac;
  d->lf_level = st.lf.level;
  d->lf_sharpness = st.lf.sharpness;
  d->lf_delta_enabled = st.lf.delta_enabled;
  memcpy(d->lf_ref_deltas, st.lf.ref_deltas, 4);
  memcpy(d->lf_mode_deltas, st.lf.mode_deltas, 2);
  d->seg.enabled = st.seg.enabled;
  d->seg.update_map = st.seg.update_map;
  d->seg.temporal_update = st.seg.temporal_update;
  d->seg.abs_or_delta_update = st.seg.abs_or_delta_update;
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 4; ++j) {
      d->seg.feature_enabled[i][j] = st.seg.feature_enabled[i][j];
      d->seg.feature_data[i][j] = st.seg.feature_data[i][j];
    }
  if (!h.frame_is_intra)
    for (int i = 0; i < 3; ++i) {
      d->ref_width[i] = slots[h.ref_frame_idx[i]].width;
      d->ref_height[i] = slots[h.ref_frame_idx[i]].height;
    }
  d->color_space = h.color_space;
  d->color_range = h.color_range;
  d->render_width = h.render_width;
  d->render_height = h.render_height;
}

// The frame process (reference src/decoder/mod.rs:218-422), without samples,
// in three steps: begin (headers and everything the frame's header decides,
// including the reference slots it refreshes), run (the tiles), finish (what
// the tiles decide for later frames: adapted contexts, previous motion
// vectors and segment ids, the legacy 4:4:4 layout). On a tile error the
// state goes back to what the header left, as if the frame had been parsed
// on its own.

Parser::Job* Parser::begin(const uint8_t* data, size_t len, const AfterHeader& after_header) {
  Impl& I = *impl_;
  FrameState& S = I.s;
  Job* job = new Job;
  job->out.blocks.clear();
  try {
    if (len == 0) bitstream_error("empty frame");
    uint8_t saved_last_type = S.st.last_frame_type;
    ResetKind reset;
    int reset_idx = 0;
    FrameHeader h;
    try {
      h = parse_uncompressed(data, len, S.st, &reset, &reset_idx);
    } catch (const HeaderError& e) {
      throw ParseError{ST_BITSTREAM, e.msg};
    }
    // What this frame reads of earlier frames' tile results; the pipeline
    // settles those frames first.
    if (after_header) after_header(h);
    if (h.show_existing_frame) {
      S.st.last_frame_type = saved_last_type;
      if (!S.slots[h.frame_to_show_map_idx].valid) bitstream_error("show_existing_frame of an empty slot");
      job->show_existing = true;
      job->out.show_existing = true;
      job->out.show_slot = h.frame_to_show_map_idx;
      job->out.show_frame = true;
      job->out.refresh_mask = 0;
      return job;
    }
    if ((uint64_t)h.width * h.height > max_pixels_) throw ParseError{ST_UNSUPPORTED, "frame size is above the decoder's limit"};
    if (h.header_size_in_bytes == 0) bitstream_error("compressed header of size 0");
    if (h.profile >= 4) throw ParseError{ST_UNSUPPORTED, "profile above 3"};
    if (!h.frame_is_intra) {
      for (int i = 0; i < 3; ++i) {
        const SlotInfo& s = S.slots[h.ref_frame_idx[i]];
        if (!s.valid) bitstream_error("reference to an empty slot");
        if (s.ss_x != h.ss_x || s.ss_y != h.ss_y || s.bit_depth != h.bit_depth)
          bitstream_error("reference frame of another format");
        // inter_scale's bounds (reference src/decoder/mod.rs:503-511).
        job->ref_ok[i] = !(2 * h.width < s.width || 2 * h.height < s.height || h.width > 16 * s.width ||
                           h.height > 16 * s.height);
      }
    }
    // compute_image_size() semantics (7.2.6).
    bool first = !S.have_last_size;
    bool same_size = S.have_last_size && S.last_w == h.width && S.last_h == h.height;
    size_t mi_len = (size_t)h.mi_rows * h.mi_cols;
    bool use_prev = !first && same_size && S.last_show_frame && !h.error_resilient_mode && !h.frame_is_intra;
    if (!same_size) S.prev_segment_ids = std::make_shared<std::vector<uint8_t>>(mi_len, 0);
    S.have_last_size = true;
    S.last_w = h.width;
    S.last_h = h.height;
    S.last_show_frame = h.show_frame;
    if (h.past_independence) S.prev_segment_ids = std::make_shared<std::vector<uint8_t>>(S.prev_segment_ids->size(), 0);
    if (reset == RESET_ALL) {
      for (auto& c : S.contexts) c.set_default();
    } else if (reset == RESET_ONE) {
      S.contexts[reset_idx].set_default();
    }
    job->pre = S.contexts[h.frame_context_idx];
    job->probs = job->pre;
    size_t comp_start = h.uncompressed_size;
    size_t comp_end = comp_start + h.header_size_in_bytes;
    if (comp_end > len) bitstream_error("compressed header runs past the end of the frame");
    parse_compressed(data + comp_start, h.header_size_in_bytes, h, job->probs);
    job->seg = S.st.seg;
    job->prev_seg = S.prev_segment_ids;
    job->prev_external = S.prev_external;
    job->use_prev_hdr = use_prev;
    job->use_prev = use_prev && (S.prev_external || S.prev_mvs->size() >= mi_len);
    if (job->use_prev && !S.prev_external) job->prev_mvs = S.prev_mvs;
    job->tiles = data + comp_end;
    job->tiles_len = len - comp_end;
    job->non420 = !(h.ss_x == 1 && h.ss_y == 1);
    h.legacy_uv = job->non420 && !h.frame_is_intra && S.legacy_uv;
    bool adapts = !h.error_resilient_mode && !h.frame_parallel_decoding_mode;
    job->late_ctx = adapts && h.refresh_frame_context;
    // The state a tile error returns to.
    job->snap = S;
    // Header-decided updates: a context refreshed without adaptation, the
    // reference slots, the records' frame description.
    if (h.refresh_frame_context && !adapts) S.contexts[h.frame_context_idx] = job->probs;
    fill_desc(h, S.st, S.slots, &job->out.desc);
    job->out.show_frame = h.show_frame;
    job->out.refresh_mask = h.refresh_frame_flags;
    for (int i = 0; i < 3; ++i) job->out.ref_slot[i] = h.ref_frame_idx[i];
    for (int i = 0; i < 8; ++i)
      if ((h.refresh_frame_flags >> i) & 1) {
        SlotInfo& sl = S.slots[i];
        sl.valid = true;
        sl.width = h.width;
        sl.height = h.height;
        sl.ss_x = h.ss_x;
        sl.ss_y = h.ss_y;
        sl.bit_depth = h.bit_depth;
        S.st.ref_w[i] = h.width;
        S.st.ref_h[i] = h.height;
      }
    job->h = h;
  } catch (const ParseError& e) {
    job->st = e.st;
    job->err = e.msg ? e.msg : "bitstream error";
  }
  return job;
}

void Parser::run(Job* job) {
  if (job->st != ST_OK || job->show_existing) return;
  if (job->use_prev && !job->prev_mvs) {
    // The previous frame's vectors are held by an external parser and were
    // not handed over (provide_prev_mvs).
    job->tr.st = ST_INVALID_INPUT;
    job->tr.err = "previous motion vectors held by the device parser were not provided";
    return;
  }
  auto t0 = std::chrono::steady_clock::now();
  const FrameHeader& h = job->h;
  TileWork& W = *job->work;
  const PrevMv* prev = job->prev_mvs ? job->prev_mvs->data() : nullptr;
  TileResult tr = W.decode_tiles(h, job->seg, job->probs, prev, job->prev_seg.get(), job->ref_ok, job->tiles,
                                 job->tiles_len, threads_);
  if (h.frame_is_intra && job->non420 && !(tr.st == ST_OK && tr.padding_ok)) {
    // Legacy 4:4:4 layout probe (reference README quirk): decode again with
    // the 4:2:0 chroma layout; keep it if it parses cleanly.
    FrameHeader legacy = h;
    legacy.legacy_uv = true;
    std::vector<TileCoder<DecCoder>> saved;
    saved.swap(W.tile_decs);
    TileResult retry = W.decode_tiles(legacy, job->seg, job->probs, prev, job->prev_seg.get(), job->ref_ok,
                                      job->tiles, job->tiles_len, threads_);
    if (retry.st == ST_OK && retry.padding_ok) {
      tr = retry;
      job->h.legacy_uv = true;
      job->out.desc.legacy_uv = 1;
    } else {
      W.tile_decs.swap(saved);
      // The mode info of the first attempt is lost: decode it once more.
      if (tr.st == ST_OK)
        tr = W.decode_tiles(h, job->seg, job->probs, prev, job->prev_seg.get(), job->ref_ok, job->tiles,
                            job->tiles_len, threads_);
    }
  }
  job->tr = tr;
  if (tr.st == ST_OK) {
    // Records in bitstream order of tile columns (tile rows within a column
    // stay in order; a column reads nothing of another).
    uint32_t tile_cols = 1u << h.tile_cols_log2;
    size_t nb = 0, nt = 0, nc = 0;
    for (uint32_t c = 0; c < tile_cols; ++c) {
      nb += W.tile_decs[c].blocks.size();
      nt += W.tile_decs[c].toks.size();
      nc += W.tile_decs[c].coefs.size();
    }
    ParsedFrame& out = job->out;
    out.blocks.clear();
    out.toks.clear();
    out.coefs.clear();
    out.blocks.reserve(nb);
    out.toks.reserve(nt);
    out.coefs.reserve(nc);
    for (uint32_t c = 0; c < tile_cols; ++c) {
      TileCoder<DecCoder>& td = W.tile_decs[c];
      uint32_t tok_base = (uint32_t)out.toks.size(), coef_base = (uint32_t)out.coefs.size();
      for (rv9_block b : td.blocks) {
        b.tok_start += tok_base;
        out.blocks.push_back(b);
      }
      for (rv9_tok t : td.toks) {
        t.coef_start += coef_base;
        out.toks.push_back(t);
      }
      out.coefs.insert(out.coefs.end(), td.coefs.begin(), td.coefs.end());
    }
  }
  job->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

Status Parser::finish(Job* job, ParsedFrame* out, std::string* err) {
  Impl& I = *impl_;
  FrameState& S = I.s;
  if (job->st != ST_OK) {
    *err = job->err;
    return job->st;
  }
  if (job->show_existing) {
    out->blocks.clear();
    out->toks.clear();
    out->coefs.clear();
    out->show_existing = true;
    out->show_slot = job->out.show_slot;
    out->show_frame = true;
    out->refresh_mask = 0;
    ++frames_;
    return ST_OK;
  }
  const FrameHeader& h = job->h;
  if (h.frame_is_intra) {
    // The layout the probe settled on carries to the inter frames that
    // follow, whether or not the tiles parsed.
    job->snap.legacy_uv = job->h.legacy_uv;
  }
  if (job->tr.st != ST_OK) {
    // Back to what this frame's header left. Frames before it may have
    // finished since (the pipeline): their previous motion vectors and
    // legacy layout stay; nothing else of theirs can be pending then.
    FrameState now = S;
    S = job->snap;
    S.prev_mvs = now.prev_mvs;
    S.prev_external = now.prev_external;
    if (!h.frame_is_intra) S.legacy_uv = now.legacy_uv;
    *err = job->tr.err.empty() ? "bitstream error" : job->tr.err;
    return job->tr.st;
  }
  if (h.frame_is_intra) S.legacy_uv = job->h.legacy_uv;
  size_t mi_len = (size_t)h.mi_rows * h.mi_cols;
  if (job->external) {
    // Nothing of the frame adapts or segments (external_tiles); its motion
    // vectors stay with the external parser.
    S.prev_mvs = std::make_shared<std::vector<PrevMv>>();
    S.prev_external = true;
    out->show_existing = false;
    out->show_frame = job->out.show_frame;
    out->refresh_mask = job->out.refresh_mask;
    for (int i = 0; i < 3; ++i) out->ref_slot[i] = job->out.ref_slot[i];
    out->desc = job->out.desc;
    out->blocks.clear();
    out->toks.clear();
    out->coefs.clear();
    out->parse_seconds = 0;
    ++frames_;
    return ST_OK;
  }
  TileWork& W = *job->work;
  // Backward adaptation (refresh_probs, 6.1.2).
  if (job->late_ctx) {
    Counts counts;
    counts.clear();
    uint32_t tile_cols = 1u << h.tile_cols_log2;
    for (uint32_t c = 0; c < tile_cols; ++c) counts.add(W.tile_decs[c].counts);
    Probs adapted = job->probs;
    adapted.load_except_tx_skip(job->pre);
    adapt_coef_probs(adapted, counts, h.frame_is_intra, h.last_frame_type == KEY_FRAME);
    if (!h.frame_is_intra) {
      adapted.load_tx_skip(job->pre);
      adapt_noncoef_probs(adapted, counts, h.interpolation_filter == SWITCHABLE, h.tx_mode == TX_MODE_SELECT,
                          h.allow_high_precision_mv);
    }
    S.contexts[h.frame_context_idx] = adapted;
  }
  // Segmentation map for the next frame (8.1 step 3).
  if (job->seg.enabled && job->seg.update_map) {
    auto ids = std::make_shared<std::vector<uint8_t>>(mi_len);
    for (size_t i = 0; i < mi_len; ++i) (*ids)[i] = W.mi[i].segment_id;
    S.prev_segment_ids = ids;
  }
  // PrevMvs / PrevRefFrames (8.10 step 2).
  auto mvs = std::make_shared<std::vector<PrevMv>>(mi_len);
  for (size_t i = 0; i < mi_len; ++i) {
    const MiInfo& m = W.mi[i];
    PrevMv& p = (*mvs)[i];
    p.ref_frame[0] = m.ref_frame[0];
    p.ref_frame[1] = m.ref_frame[1];
    p.mv[0] = m.mv[0][3];
    p.mv[1] = m.mv[1][3];
  }
  S.prev_mvs = mvs;
  S.prev_external = false;
  out->show_existing = false;
  out->show_frame = job->out.show_frame;
  out->refresh_mask = job->out.refresh_mask;
  for (int i = 0; i < 3; ++i) out->ref_slot[i] = job->out.ref_slot[i];
  out->desc = job->out.desc;
  out->blocks.swap(job->out.blocks);
  out->toks.swap(job->out.toks);
  out->coefs.swap(job->out.coefs);
  out->parse_seconds = job->seconds;
  ++frames_;
  return ST_OK;
}

void Parser::attach_work(Job* job) { job->work = impl_->take_work(); }

bool Parser::external_tiles(const Job* job, ExternalTiles* out) const {
  if (job->st != ST_OK || job->show_existing || job->late_ctx || job->seg.enabled) return false;
  if (job->h.frame_is_intra && job->non420) return false;  // the legacy 4:4:4 probe
  out->h = &job->h;
  out->probs = &job->probs;
  out->ref_ok = job->ref_ok;
  out->tiles = job->tiles;
  out->tiles_len = job->tiles_len;
  out->use_prev = job->use_prev_hdr;
  out->prev_external = job->use_prev && job->prev_external;
  out->prev_host = job->use_prev && !job->prev_external ? job->prev_mvs->data() : nullptr;
  out->desc = &job->out.desc;
  return true;
}

Status Parser::finish_external(Job* job, Status tiles_st, const std::string& tiles_err, ParsedFrame* out,
                               std::string* err) {
  if (job->st == ST_OK && !job->show_existing) {
    job->external = true;
    job->tr.st = tiles_st;
    job->tr.err = tiles_err;
  }
  return finish(job, out, err);
}

bool Parser::independent(const Job* job) const {
  return job->st == ST_OK && !job->show_existing && !job->use_prev &&
         (job->h.error_resilient_mode || job->h.frame_type == KEY_FRAME);
}

void Parser::run_async(Job* job) {
  attach_work(job);
  if (job->st != ST_OK || job->show_existing) return;
  job->running = true;
  job->th = std::thread([this, job]() { run(job); });
}

void Parser::wait(Job* job) {
  if (job->th.joinable()) job->th.join();
  job->running = false;
}

void Parser::bind_prev(Job* job) {
  if (job->st != ST_OK || job->show_existing || !job->use_prev_hdr) return;
  const FrameState& S = impl_->s;
  // begin's rule, against the state as it is now: host-held vectors of
  // another size are not used.
  job->prev_external = S.prev_external;
  job->use_prev = S.prev_external || S.prev_mvs->size() >= (size_t)job->h.mi_rows * job->h.mi_cols;
  job->prev_mvs = job->use_prev && !S.prev_external ? S.prev_mvs : nullptr;
}

bool Parser::wants_external_prev(const Job* job) const {
  return job->st == ST_OK && !job->show_existing && job->use_prev && job->prev_external && !job->prev_mvs;
}

void Parser::provide_prev_mvs(Job* job, const void* mvs, size_t n) {
  auto v = std::make_shared<std::vector<PrevMv>>(n);
  if (n) memcpy(v->data(), mvs, n * sizeof(PrevMv));
  job->prev_mvs = v;
}

void Parser::release(Job* job) {
  if (!job) return;
  if (job->th.joinable()) job->th.join();
  if (job->work) impl_->spare.push_back(std::move(job->work));
  delete job;
}

Status Parser::parse_frame(const uint8_t* data, size_t len, ParsedFrame* out, std::string* err) {
  Job* job = begin(data, len, nullptr);
  if (job->st == ST_OK && !job->show_existing) {
    attach_work(job);
    run(job);
  }
  Status st = finish(job, out, err);
  release(job);
  return st;
}

// ---------------------------------------------------------------------------
// Frame-parallel parsing.

FramePipeline::FramePipeline(Parser* p, int depth) : p_(p), depth_(depth < 1 ? 1 : depth) {}

FramePipeline::~FramePipeline() {
  for (Parser::Job* j : q_) p_->release(j);
}

void FramePipeline::settle() {
  // Finishes every frame in flight, in order (their results wait in q_).
  for (Parser::Job* j : q_) {
    if (j->running) {
      j->th.join();
      j->running = false;
    }
    if (!j->settled) {
      j->settled_status = p_->finish(j, &j->settled_out, &j->settled_err);
      j->settled = true;
      if (j->settled_status != ST_OK) {
        failed_ = true;
        return;
      }
    }
  }
}

Status FramePipeline::push(const uint8_t* data, size_t len) {
  if (failed_) return ST_INVALID_INPUT;
  // The new frame's header runs against the state that the frames before it
  // leave. Those still in flight settle first, unless the new frame cannot
  // depend on what they decide at finish: it is a key frame or error
  // resilient (contexts reset, no previous motion vectors or segment ids),
  // and no frame in flight adapts a context, carries a segment map or probes
  // the legacy 4:4:4 layout that this frame would read.
  bool pending = false, pending_intra_non420 = false;
  for (Parser::Job* j : q_)
    if (!j->settled && j->st == ST_OK && !j->show_existing) {
      pending |= j->late_ctx || (j->seg.enabled && j->seg.update_map);
      pending_intra_non420 |= j->h.frame_is_intra && j->non420;
    }
  Parser::Job* job = p_->begin(data, len, [&](const FrameHeader& h) {
    bool fresh = h.error_resilient_mode || h.frame_type == KEY_FRAME;
    bool non420 = !(h.ss_x == 1 && h.ss_y == 1);
    if (pending || !fresh || h.show_existing_frame || (non420 && pending_intra_non420)) {
      settle();
      if (failed_) throw ParseError{ST_INVALID_INPUT, "an earlier frame failed"};
    }
  });
  q_.push_back(job);
  if (failed_) return ST_OK;  // an earlier frame failed: pop() reports it first
  if (job->st == ST_OK && !job->show_existing) {
    p_->attach_work(job);
    job->running = true;
    Parser* p = p_;
    job->th = std::thread([p, job]() { p->run(job); });
  }
  return ST_OK;
}

Status FramePipeline::pop(ParsedFrame* out, std::string* err) {
  if (q_.empty()) {
    *err = "no frame in flight";
    return ST_INVALID_INPUT;
  }
  Parser::Job* j = q_.front();
  q_.pop_front();
  Status st;
  if (j->settled) {
    st = j->settled_status;
    if (st == ST_OK) {
      *out = std::move(j->settled_out);
    } else {
      *err = j->settled_err;
    }
  } else {
    if (j->running) {
      j->th.join();
      j->running = false;
    }
    st = p_->finish(j, out, err);
  }
  p_->release(j);
  if (st != ST_OK) {
    // Frames after a failed one are dropped (the state is the failed
    // frame's, as the sequential parse leaves it).
    for (Parser::Job* k : q_) p_->release(k);
    q_.clear();
    failed_ = true;
  }
  return st;
}

void superframe_split(const uint8_t* pkt, size_t len, std::vector<std::pair<size_t, size_t>>* out) {
  out->clear();
  if (len > 0) {
    uint8_t last = pkt[len - 1];
    if ((last & 0xe0) == 0xc0) {
      size_t sz_bytes = ((last >> 3) & 3) + 1;
      size_t frames = (last & 7) + 1;
      size_t index_len = 2 + frames * sz_bytes;
      if (len >= index_len && pkt[len - index_len] == last) {
        size_t p = len - index_len + 1;
        std::vector<size_t> sizes;
        size_t total = 0;
        for (size_t f = 0; f < frames; ++f) {
          size_t s = 0;
          for (size_t b = 0; b < sz_bytes; ++b) s |= (size_t)pkt[p + b] << (8 * b);
          p += sz_bytes;
          total += s;
          sizes.push_back(s);
        }
        if (total <= len - index_len) {
          size_t pos = 0;
          for (size_t s : sizes) {
            if (s == 0) continue;
            out->emplace_back(pos, s);
            pos += s;
          }
          return;
        }
      }
    }
  }
  out->emplace_back(0, len);
}

}  // namespace rv9

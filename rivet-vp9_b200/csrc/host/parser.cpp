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
#include <thread>

#include "../common/vp9_consts.h"
#include "../common/vp9_tables.h"
#include "bitreader.h"

namespace rv9 {
using namespace vp9;

namespace {

struct ParseError {
  Status st;
  const char* msg;
};

[[noreturn]] void bitstream_error(const char* m) { throw ParseError{ST_BITSTREAM, m}; }

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

// get_tile_offset (spec 6.4.1).
uint32_t tile_offset(uint32_t tile_num, uint32_t mis, uint32_t log2) {
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

// The scan order of get_scan (spec 6.4.25).
const uint16_t* get_scan(int tx_sz, int tx_type) {
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

const NeighborTables& neighbor_tables() {
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

// One tile column's decoder: its left contexts, counts and records.
struct TileDec {
  const FrameCtx* f;
  const FrameHeader* h;
  Counts counts;
  std::vector<rv9_block> blocks;
  std::vector<rv9_tok> toks;
  std::vector<uint32_t> coefs;
  std::vector<uint8_t> left_nonzero[3];
  std::vector<uint8_t> left_partition;
  std::vector<uint8_t> left_seg_pred;
  uint32_t mi_row_start = 0, mi_row_end = 0, mi_col_start = 0, mi_col_end = 0;
  uint32_t mi_cols = 0, mi_rows = 0;
  uint32_t ss_x = 0, ss_y = 0;
  BlockState b;
  uint32_t eob_total = 0;
  uint8_t token_cache[1024];
  bool padding_ok = true;

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
  }

  MiInfo& mi_at(uint32_t r, uint32_t c) const { return f->mi[(size_t)r * mi_cols + c]; }

  void decode_tile(BoolDecoder& d) {
    for (uint32_t r = mi_row_start; r < mi_row_end; r += 8) {
      for (int p = 0; p < 3; ++p) std::fill(left_nonzero[p].begin(), left_nonzero[p].end(), 0);
      std::fill(left_partition.begin(), left_partition.end(), 0);
      std::fill(left_seg_pred.begin(), left_seg_pred.end(), 0);
      for (uint32_t c = mi_col_start; c < mi_col_end; c += 8) decode_partition(d, r, c, BLOCK_64X64);
    }
  }

  void decode_partition(BoolDecoder& d, uint32_t r, uint32_t c, uint8_t bsize) {
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
    if (has_rows && has_cols)
      partition = d.tree(PARTITION_TREE, [&](int n) { return probs[n]; });
    else if (has_cols)
      partition = d.read(probs[1]) ? PARTITION_SPLIT : PARTITION_HORZ;
    else if (has_rows)
      partition = d.read(probs[2]) ? PARTITION_SPLIT : PARTITION_VERT;
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

  void decode_block(BoolDecoder& d, uint32_t r, uint32_t c, uint8_t subsize) {
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

  void intra_frame_mode_info(BoolDecoder& d) {
    const SegParams& seg = *f->seg;
    b.segment_id = (seg.enabled && seg.update_map)
                       ? (uint8_t)d.tree(SEGMENT_TREE, [&](int n) { return seg.tree_probs[n]; })
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
      uint8_t mode = (uint8_t)d.tree(INTRA_MODE_TREE, [&](int n) { return p[n]; });
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
          mode = (uint8_t)d.tree(INTRA_MODE_TREE, [&](int n) { return p[n]; });
          for (int y2 = 0; y2 < n4h; ++y2)
            for (int x2 = 0; x2 < n4w; ++x2) b.sub_modes[(idy + y2) * 2 + idx + x2] = mode;
        }
      b.y_mode = mode;
    }
    const uint8_t* p = vp9t_kf_uv_mode_probs[b.y_mode];
    b.uv_mode = (uint8_t)d.tree(INTRA_MODE_TREE, [&](int n) { return p[n]; });
  }

  void read_skip(BoolDecoder& d) {
    if (f->seg->active(b.segment_id, SEG_LVL_SKIP)) {
      b.skip = true;
    } else {
      int ctx = (b.above ? b.above->skip : 0) + (b.left ? b.left->skip : 0);
      b.skip = d.read(f->probs->skip[ctx]);
      counts.skip[ctx][b.skip ? 1 : 0] += 1;
    }
  }

  void read_tx_size(BoolDecoder& d, bool allow_select) {
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
      int v = d.tree(tree, [&](int n) { return p[n]; });
      counts.tx[max_tx][ctx][v] += 1;
      b.tx_size = (uint8_t)v;
    } else {
      uint8_t m = TX_MODE_TO_BIGGEST_TX_SIZE[h->tx_mode];
      b.tx_size = max_tx < m ? max_tx : m;
    }
  }

  void inter_frame_mode_info(BoolDecoder& d) {
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

  void inter_segment_id(BoolDecoder& d) {
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
      bool pred = d.read(seg.pred_probs[ctx]);
      b.segment_id = pred ? predicted : (uint8_t)d.tree(SEGMENT_TREE, [&](int n) { return seg.tree_probs[n]; });
      uint32_t bw = vp9t_num_8x8_wide[b.mi_size], bh = vp9t_num_8x8_high[b.mi_size];
      for (uint32_t i = 0; i < bw; ++i) f->above_seg_pred[b.mi_col + i] = pred;
      for (uint32_t i = 0; i < bh; ++i) left_seg_pred[b.mi_row + i] = pred;
    } else {
      b.segment_id = (uint8_t)d.tree(SEGMENT_TREE, [&](int n) { return seg.tree_probs[n]; });
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

  void read_is_inter(BoolDecoder& d) {
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
      b.is_inter = d.read(f->probs->is_inter[ctx]);
      counts.is_inter[ctx][b.is_inter ? 1 : 0] += 1;
    }
  }

  void intra_block_mode_info(BoolDecoder& d) {
    b.ref_frame[0] = INTRA_FRAME;
    b.ref_frame[1] = NONE_FRAME;
    if (b.mi_size >= BLOCK_8X8) {
      int ctx = vp9t_size_group[b.mi_size];
      const uint8_t* p = f->probs->y_mode[ctx];
      uint8_t mode = (uint8_t)d.tree(INTRA_MODE_TREE, [&](int n) { return p[n]; });
      counts.intra_mode[ctx][mode] += 1;
      b.y_mode = mode;
      for (int i = 0; i < 4; ++i) b.sub_modes[i] = mode;
    } else {
      int n4w = vp9t_num_4x4_wide[b.mi_size], n4h = vp9t_num_4x4_high[b.mi_size];
      const uint8_t* p = f->probs->y_mode[0];
      uint8_t mode = DC_PRED;
      for (int idy = 0; idy < 2; idy += n4h)
        for (int idx = 0; idx < 2; idx += n4w) {
          mode = (uint8_t)d.tree(INTRA_MODE_TREE, [&](int n) { return p[n]; });
          counts.intra_mode[0][mode] += 1;
          for (int y2 = 0; y2 < n4h; ++y2)
            for (int x2 = 0; x2 < n4w; ++x2) b.sub_modes[(idy + y2) * 2 + idx + x2] = mode;
        }
      b.y_mode = mode;
    }
    const uint8_t* p = f->probs->uv_mode[b.y_mode];
    uint8_t uv = (uint8_t)d.tree(INTRA_MODE_TREE, [&](int n) { return p[n]; });
    counts.uv_mode[b.y_mode][uv] += 1;
    b.uv_mode = uv;
  }

  void inter_block_mode_info(BoolDecoder& d) {
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
      int fl = d.tree(INTERP_FILTER_TREE, [&](int n) { return p[n]; });
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

  int read_inter_mode(BoolDecoder& d) {
    int ctx = b.mode_context[b.ref_frame[0]];
    const uint8_t* p = f->probs->inter_mode[ctx];
    int v = d.tree(INTER_MODE_TREE, [&](int n) { return p[n]; });
    counts.inter_mode[ctx][v] += 1;
    return v;
  }

  void read_ref_frames(BoolDecoder& d) {
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
      bool v = d.read(f->probs->comp_mode[ctx]);
      counts.comp_mode[ctx][v ? 1 : 0] += 1;
      comp_mode = v ? COMPOUND_REFERENCE : SINGLE_REFERENCE;
    } else {
      comp_mode = h->reference_mode;
    }
    if (comp_mode == COMPOUND_REFERENCE) {
      int idx = h->ref_frame_sign_bias[h->comp_fixed_ref] ? 1 : 0;
      int ctx = comp_ref_ctx();
      bool v = d.read(f->probs->comp_ref[ctx]);
      counts.comp_ref[ctx][v ? 1 : 0] += 1;
      b.ref_frame[idx] = h->comp_fixed_ref;
      b.ref_frame[1 - idx] = h->comp_var_ref[v ? 1 : 0];
    } else {
      int ctx = single_ref_p1_ctx();
      bool p1 = d.read(f->probs->single_ref[ctx][0]);
      counts.single_ref[ctx][0][p1 ? 1 : 0] += 1;
      if (p1) {
        int ctx2 = single_ref_p2_ctx();
        bool p2 = d.read(f->probs->single_ref[ctx2][1]);
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

  void assign_mv(BoolDecoder& d, bool is_compound) {
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

  Mv read_mv(BoolDecoder& d, int r) {
    Mv best = b.best_mv[r];
    bool use_hp = h->allow_high_precision_mv && use_mv_hp(best);
    int32_t diff[2] = {0, 0};
    const uint8_t* p = f->probs->mv_joint;
    int joint = d.tree(MV_JOINT_TREE, [&](int n) { return p[n]; });
    counts.mv_joint[joint] += 1;
    if (joint == MV_JOINT_HZVNZ || joint == MV_JOINT_HNZVNZ) diff[0] = read_mv_component(d, 0, use_hp);
    if (joint == MV_JOINT_HNZVZ || joint == MV_JOINT_HNZVNZ) diff[1] = read_mv_component(d, 1, use_hp);
    return Mv{best.r + diff[0], best.c + diff[1]};
  }

  int32_t read_mv_component(BoolDecoder& d, int comp, bool use_hp) {
    const Probs& pr = *f->probs;
    bool sign = d.read(pr.mv_sign[comp]);
    counts.mv_sign[comp][sign ? 1 : 0] += 1;
    const uint8_t* pc = pr.mv_class[comp];
    int cls = d.tree(MV_CLASS_TREE, [&](int n) { return pc[n]; });
    counts.mv_class[comp][cls] += 1;
    int32_t mag;
    if (cls == 0) {
      int c0 = d.read(pr.mv_class0_bit[comp]) ? 1 : 0;
      counts.mv_class0_bit[comp][c0] += 1;
      const uint8_t* pf = pr.mv_class0_fr[comp][c0];
      int fr = d.tree(MV_FR_TREE, [&](int n) { return pf[n]; });
      counts.mv_class0_fr[comp][c0][fr] += 1;
      int hp = use_hp ? (d.read(pr.mv_class0_hp[comp]) ? 1 : 0) : 1;
      counts.mv_class0_hp[comp][hp] += 1;
      mag = ((c0 << 3) | (fr << 1) | hp) + 1;
    } else {
      int32_t dd = 0;
      for (int i = 0; i < cls; ++i) {
        int bit = d.read(pr.mv_bits[comp][i]) ? 1 : 0;
        counts.mv_bits[comp][i][bit] += 1;
        dd |= bit << i;
      }
      int32_t m0 = 2 << (cls + 2);
      const uint8_t* pf = pr.mv_fr[comp];
      int fr = d.tree(MV_FR_TREE, [&](int n) { return pf[n]; });
      counts.mv_fr[comp][fr] += 1;
      int hp = use_hp ? (d.read(pr.mv_hp[comp]) ? 1 : 0) : 1;
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

  void residual(BoolDecoder& d) {
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

  static int32_t read_coef(BoolDecoder& d, int token, uint32_t bit_depth) {
    int cat = EXTRA_BITS[token][0], num_extra = EXTRA_BITS[token][1];
    int32_t coef = EXTRA_BITS[token][2];
    if (token == DCT_VAL_CAT6) {
      for (int e = 0; e < (int)bit_depth - 8; ++e) {
        int32_t high = d.read(255) ? 1 : 0;
        coef += high << (5 + (int)bit_depth - e);
      }
    }
    const uint8_t* probs = CAT_PROBS[cat];
    for (int e = 0; e < num_extra; ++e) {
      int32_t bit = d.read(probs[e]) ? 1 : 0;
      coef += bit << (num_extra - 1 - e);
    }
    return coef;
  }

  // tokens() (spec 6.4.24): records the nonzero coefficients; returns eob.
  int tokens(BoolDecoder& d, int plane, uint32_t start_x, uint32_t start_y, int tx_sz, int block_idx) {
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
    for (; c < seg_eob; ++c) {
      int pos = scan[c];
      int band = bands[c];
      if (c > 0) ctx = (1 + token_cache[nb[c][0]] + token_cache[nb[c][1]]) >> 1;
      const uint8_t* probs = cp[band][ctx];
      if (check_eob) {
        bool more = d.read(probs[0]);
        if (count) counts.more_coefs[tx_sz][ptype][ref_type][band][ctx][more ? 1 : 0] += 1;
        if (!more) break;
      }
      int token = d.tree(TOKEN_TREE, [&](int node) { return pareto(node, probs[(1 + node) < 2 ? (1 + node) : 2]); });
      if (count) counts.token[tx_sz][ptype][ref_type][band][ctx][token < 2 ? token : 2] += 1;
      token_cache[pos] = vp9t_energy_class[token];
      if (token == ZERO_TOKEN) {
        check_eob = false;
      } else {
        int32_t coef = read_coef(d, token, bd);
        bool sign = d.read(128);
        coefs.push_back(RV9_COEF_PACK(pos, sign ? -coef : coef));
        check_eob = true;
      }
    }
    if (c > 0) ++eob_total;
    t.eob = (uint16_t)c;
    t.n_coef = (uint16_t)(coefs.size() - t.coef_start);
    toks.push_back(t);
    return c;
  }
};

struct TileSpan {
  uint32_t row, col;
  const uint8_t* data;
  size_t size;
};

}  // namespace

// ---------------------------------------------------------------------------

struct Parser::Impl {
  Persistent st;
  Probs contexts[4];
  SlotInfo slots[8];
  std::vector<uint8_t> prev_segment_ids;
  std::vector<PrevMv> prev_mvs;
  bool have_last_size = false;
  uint32_t last_w = 0, last_h = 0;
  bool last_show_frame = false;
  bool legacy_uv = false;
  // Frame working memory.
  std::vector<MiInfo> mi;
  std::vector<uint8_t> above_nonzero[3];
  std::vector<uint8_t> above_partition, above_seg_pred;
  std::vector<TileDec> tile_decs;

  Impl() {
    for (auto& c : contexts) c.set_default();
  }

  struct TileResult {
    Status st = ST_OK;
    std::string err;
    int failed_tile = -1;
    bool padding_ok = true;
  };

  // Decodes all tiles of a frame into `tile_decs` (one per tile column).
  TileResult decode_tiles(const FrameHeader& h, const SegParams& seg, const Probs& probs,
                          const PrevMv* prev, const bool ref_ok[3], const uint8_t* data, size_t len,
                          int threads) {
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
    fc.prev_seg_ids = prev_segment_ids.data();
    fc.prev_seg_len = prev_segment_ids.size();
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
      TileDec& td = tile_decs[col];
      for (size_t i = 0; i < tiles.size(); ++i) {
        const TileSpan& t = tiles[i];
        if (t.col != col) continue;
        td.mi_row_start = tile_offset(t.row, h.mi_rows, h.tile_rows_log2);
        td.mi_row_end = tile_offset(t.row + 1, h.mi_rows, h.tile_rows_log2);
        td.mi_col_start = tile_offset(t.col, h.mi_cols, h.tile_cols_log2);
        td.mi_col_end = tile_offset(t.col + 1, h.mi_cols, h.tile_cols_log2);
        try {
          BoolDecoder d;
          if (t.size == 0) bitstream_error("boolean-coded partition of size 0");
          if (!d.init(t.data, t.size)) bitstream_error("boolean decoder marker bit is not 0");
          td.decode_tile(d);
          td.padding_ok &= d.padding_is_zero();
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

// The frame process (reference src/decoder/mod.rs:218-422), without samples.
Status Parser::parse_frame(const uint8_t* data, size_t len, ParsedFrame* out, std::string* err) {
  auto t0 = std::chrono::steady_clock::now();
  Impl& I = *impl_;
  out->blocks.clear();
  out->toks.clear();
  out->coefs.clear();
  out->show_existing = false;
  if (len == 0) {
    *err = "empty frame";
    return ST_BITSTREAM;
  }
  try {
    uint8_t saved_last_type = I.st.last_frame_type;
    ResetKind reset;
    int reset_idx = 0;
    FrameHeader h;
    try {
      h = parse_uncompressed(data, len, I.st, &reset, &reset_idx);
    } catch (const HeaderError& e) {
      throw ParseError{ST_BITSTREAM, e.msg};
    }
    if (h.show_existing_frame) {
      I.st.last_frame_type = saved_last_type;
      if (!I.slots[h.frame_to_show_map_idx].valid) bitstream_error("show_existing_frame of an empty slot");
      out->show_existing = true;
      out->show_slot = h.frame_to_show_map_idx;
      out->show_frame = true;
      out->refresh_mask = 0;
      ++frames_;
      return ST_OK;
    }
    if ((uint64_t)h.width * h.height > max_pixels_) throw ParseError{ST_UNSUPPORTED, "frame size is above the decoder's limit"};
    if (h.header_size_in_bytes == 0) bitstream_error("compressed header of size 0");
    if (h.profile >= 4) throw ParseError{ST_UNSUPPORTED, "profile above 3"};
    bool ref_ok[3] = {true, true, true};
    if (!h.frame_is_intra) {
      for (int i = 0; i < 3; ++i) {
        const SlotInfo& s = I.slots[h.ref_frame_idx[i]];
        if (!s.valid) bitstream_error("reference to an empty slot");
        if (s.ss_x != h.ss_x || s.ss_y != h.ss_y || s.bit_depth != h.bit_depth)
          bitstream_error("reference frame of another format");
        // inter_scale's bounds (reference src/decoder/mod.rs:503-511).
        ref_ok[i] = !(2 * h.width < s.width || 2 * h.height < s.height || h.width > 16 * s.width ||
                      h.height > 16 * s.height);
      }
    }
    // compute_image_size() semantics (7.2.6).
    bool first = !I.have_last_size;
    bool same_size = I.have_last_size && I.last_w == h.width && I.last_h == h.height;
    size_t mi_len = (size_t)h.mi_rows * h.mi_cols;
    bool use_prev = !first && same_size && I.last_show_frame && !h.error_resilient_mode && !h.frame_is_intra;
    if (!same_size) I.prev_segment_ids.assign(mi_len, 0);
    I.have_last_size = true;
    I.last_w = h.width;
    I.last_h = h.height;
    I.last_show_frame = h.show_frame;
    if (h.past_independence) std::fill(I.prev_segment_ids.begin(), I.prev_segment_ids.end(), 0);
    if (reset == RESET_ALL) {
      for (auto& c : I.contexts) c.set_default();
    } else if (reset == RESET_ONE) {
      I.contexts[reset_idx].set_default();
    }
    Probs probs = I.contexts[h.frame_context_idx];
    size_t comp_start = h.uncompressed_size;
    size_t comp_end = comp_start + h.header_size_in_bytes;
    if (comp_end > len) bitstream_error("compressed header runs past the end of the frame");
    parse_compressed(data + comp_start, h.header_size_in_bytes, h, probs);
    SegParams seg = I.st.seg;
    const PrevMv* prev = use_prev && I.prev_mvs.size() >= mi_len ? I.prev_mvs.data() : nullptr;
    const uint8_t* tiles = data + comp_end;
    size_t tiles_len = len - comp_end;
    bool non420 = !(h.ss_x == 1 && h.ss_y == 1);
    h.legacy_uv = non420 && !h.frame_is_intra && I.legacy_uv;
    Impl::TileResult tr = I.decode_tiles(h, seg, probs, prev, ref_ok, tiles, tiles_len, threads_);
    if (h.frame_is_intra) {
      if (non420 && !(tr.st == ST_OK && tr.padding_ok)) {
        FrameHeader legacy = h;
        legacy.legacy_uv = true;
        // Keep the first attempt's records in case the retry fails too.
        std::vector<TileDec> saved;
        saved.swap(I.tile_decs);
        Impl::TileResult retry = I.decode_tiles(legacy, seg, probs, prev, ref_ok, tiles, tiles_len, threads_);
        if (retry.st == ST_OK && retry.padding_ok) {
          tr = retry;
          h = legacy;
        } else {
          I.tile_decs.swap(saved);
          // The mode info of the first attempt is lost; only its status matters now.
          if (tr.st == ST_OK) {
            // Re-run the first attempt so the records and mode info are its own.
            tr = I.decode_tiles(h, seg, probs, prev, ref_ok, tiles, tiles_len, threads_);
          }
        }
      }
      I.legacy_uv = h.legacy_uv;
    }
    if (tr.st != ST_OK) throw ParseError{tr.st, nullptr};
    // Gather records in bitstream order of tile columns (tile rows within a
    // column stay in order; a column reads nothing of another).
    uint32_t tile_cols = 1u << h.tile_cols_log2;
    Counts counts;
    counts.clear();
    size_t nb = 0, nt = 0, nc = 0;
    for (uint32_t c = 0; c < tile_cols; ++c) {
      nb += I.tile_decs[c].blocks.size();
      nt += I.tile_decs[c].toks.size();
      nc += I.tile_decs[c].coefs.size();
    }
    out->blocks.reserve(nb);
    out->toks.reserve(nt);
    out->coefs.reserve(nc);
    for (uint32_t c = 0; c < tile_cols; ++c) {
      TileDec& td = I.tile_decs[c];
      uint32_t tok_base = (uint32_t)out->toks.size(), coef_base = (uint32_t)out->coefs.size();
      for (rv9_block b : td.blocks) {
        b.tok_start += tok_base;
        out->blocks.push_back(b);
      }
      for (rv9_tok t : td.toks) {
        t.coef_start += coef_base;
        out->toks.push_back(t);
      }
      out->coefs.insert(out->coefs.end(), td.coefs.begin(), td.coefs.end());
      counts.add(td.counts);
    }
    // Backward adaptation (refresh_probs, 6.1.2).
    if (!h.error_resilient_mode && !h.frame_parallel_decoding_mode) {
      const Probs& pre = I.contexts[h.frame_context_idx];
      Probs adapted = probs;
      adapted.load_except_tx_skip(pre);
      adapt_coef_probs(adapted, counts, h.frame_is_intra, h.last_frame_type == KEY_FRAME);
      if (!h.frame_is_intra) {
        adapted.load_tx_skip(pre);
        adapt_noncoef_probs(adapted, counts, h.interpolation_filter == SWITCHABLE, h.tx_mode == TX_MODE_SELECT,
                            h.allow_high_precision_mv);
      }
      probs = adapted;
    }
    if (h.refresh_frame_context) I.contexts[h.frame_context_idx] = probs;
    // Segmentation map for the next frame (8.1 step 3).
    if (seg.enabled && seg.update_map) {
      I.prev_segment_ids.resize(mi_len);
      for (size_t i = 0; i < mi_len; ++i) I.prev_segment_ids[i] = I.mi[i].segment_id;
    }
    // PrevMvs / PrevRefFrames (8.10 step 2).
    I.prev_mvs.resize(mi_len);
    for (size_t i = 0; i < mi_len; ++i) {
      const MiInfo& m = I.mi[i];
      PrevMv& p = I.prev_mvs[i];
      p.ref_frame[0] = m.ref_frame[0];
      p.ref_frame[1] = m.ref_frame[1];
      p.mv[0] = m.mv[0][3];
      p.mv[1] = m.mv[1][3];
    }
    fill_desc(h, I.st, I.slots, &out->desc);
    out->show_frame = h.show_frame;
    out->refresh_mask = h.refresh_frame_flags;
    for (int i = 0; i < 3; ++i) out->ref_slot[i] = h.ref_frame_idx[i];
    // Reference update (8.10 step 1).
    for (int i = 0; i < 8; ++i)
      if ((h.refresh_frame_flags >> i) & 1) {
        SlotInfo& s = I.slots[i];
        s.valid = true;
        s.width = h.width;
        s.height = h.height;
        s.ss_x = h.ss_x;
        s.ss_y = h.ss_y;
        s.bit_depth = h.bit_depth;
        I.st.ref_w[i] = h.width;
        I.st.ref_h[i] = h.height;
      }
    ++frames_;
  } catch (const ParseError& e) {
    *err = e.msg ? e.msg : "bitstream error";
    return e.st;
  }
  out->parse_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return ST_OK;
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

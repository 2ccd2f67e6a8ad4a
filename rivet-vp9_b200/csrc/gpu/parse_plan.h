// The host side of the device tile parser (tile_parse.cuh): its tables, one
// frame's inputs from the host parser's headers, and the split of a frame's
// tile data into tile-column chains. Plain host code (no CUDA calls), shared
// by the engine and the CPU test of the device parser.
#pragma once
#include <stdint.h>
#include <string.h>

#include <vector>

#include "../host/parser.h"
#include "../host/syntax.h"
#include "tile_parse.cuh"

namespace rv9g {
namespace tp {

static_assert(sizeof(Mi) == sizeof(rv9::MiInfo), "mode info layouts differ");
static_assert(sizeof(PrevMv) == sizeof(rv9::syn::PrevMv), "previous motion vector layouts differ");

// The tables, from the specification tables the host parser uses.
inline void fill_tables(Tables* t) {
  using namespace rv9::syn;
  using namespace vp9;
  memset(t, 0, sizeof *t);
  const NeighborTables& nbt = neighbor_tables();
  const uint8_t kinds[3] = {DCT_DCT, DCT_ADST, ADST_DCT};
  for (int tx = 0; tx < 4; ++tx)
    for (int k = 0; k < 3; ++k) {
      const uint16_t* scan = get_scan(tx, kinds[k]);
      const uint16_t(*nb)[2] = nbt.get(tx, kinds[k]);
      const uint8_t* bands = tx == TX_4X4 ? vp9t_coefband_4x4 : vp9t_coefband_8x8plus;
      const int cnt = 16 << (tx << 1);
      for (int c = 0; c < cnt; ++c) t->scan[tx][k][c] = ScanEnt{scan[c], nb[c][0], nb[c][1], bands[c], 0};
    }
  for (int p = 0; p < 256; ++p) memcpy(t->pareto[p], pareto_row((uint8_t)p), 8);
  memcpy(t->energy, vp9t_energy_class, sizeof t->energy);
  memcpy(t->kf_partition, vp9t_kf_partition_probs, sizeof t->kf_partition);
  memcpy(t->kf_y_mode, vp9t_kf_y_mode_probs, sizeof t->kf_y_mode);
  memcpy(t->kf_uv_mode, vp9t_kf_uv_mode_probs, sizeof t->kf_uv_mode);
  memcpy(t->mv_ref_blocks, vp9t_mv_ref_blocks, sizeof t->mv_ref_blocks);
  memcpy(t->mode_2_counter, vp9t_mode_2_counter, sizeof t->mode_2_counter);
  memcpy(t->idx_n_col_to_sub, vp9t_idx_n_column_to_subblock, sizeof t->idx_n_col_to_sub);
  memcpy(t->b_wl2, vp9t_b_width_log2, 13);
  memcpy(t->b_hl2, vp9t_b_height_log2, 13);
  memcpy(t->n4w, vp9t_num_4x4_wide, 13);
  memcpy(t->n4h, vp9t_num_4x4_high, 13);
  memcpy(t->mi_wl2, vp9t_mi_width_log2, 13);
  memcpy(t->n8w, vp9t_num_8x8_wide, 13);
  memcpy(t->n8h, vp9t_num_8x8_high, 13);
  memcpy(t->size_group, vp9t_size_group, 13);
  memcpy(t->subsize, SUBSIZE_LOOKUP, sizeof t->subsize);
  memcpy(t->ss_size, SS_SIZE_LOOKUP, sizeof t->ss_size);
  memcpy(t->max_tx, MAX_TXSIZE_LOOKUP, sizeof t->max_tx);
  memcpy(t->tx_mode_biggest, TX_MODE_TO_BIGGEST_TX_SIZE, sizeof t->tx_mode_biggest);
  memcpy(t->mode2txfm, MODE2TXFM_MAP, sizeof t->mode2txfm);
  memcpy(t->counter_to_ctx, COUNTER_TO_CONTEXT, sizeof t->counter_to_ctx);
  for (int i = 0; i < 11; ++i)
    for (int j = 0; j < 3; ++j) t->extra_bits[i][j] = (int16_t)EXTRA_BITS[i][j];
  memcpy(t->cat_probs, CAT_PROBS, sizeof t->cat_probs);
  memcpy(t->partition_tree, PARTITION_TREE, sizeof t->partition_tree);
  memcpy(t->intra_mode_tree, INTRA_MODE_TREE, sizeof t->intra_mode_tree);
  memcpy(t->tx32_tree, TX_SIZE_32_TREE, sizeof t->tx32_tree);
  memcpy(t->tx16_tree, TX_SIZE_16_TREE, sizeof t->tx16_tree);
  memcpy(t->tx8_tree, TX_SIZE_8_TREE, sizeof t->tx8_tree);
  memcpy(t->inter_mode_tree, INTER_MODE_TREE, sizeof t->inter_mode_tree);
  memcpy(t->interp_tree, INTERP_FILTER_TREE, sizeof t->interp_tree);
  memcpy(t->mv_joint_tree, MV_JOINT_TREE, sizeof t->mv_joint_tree);
  memcpy(t->mv_class_tree, MV_CLASS_TREE, sizeof t->mv_class_tree);
  memcpy(t->mv_fr_tree, MV_FR_TREE, sizeof t->mv_fr_tree);
  memcpy(t->token_tree, TOKEN_TREE, sizeof t->token_tree);
}

// One frame's inputs from its headers and probabilities.
inline void fill_frame_in(const rv9::Parser::ExternalTiles& x, FrameIn* f) {
  const rv9::syn::FrameHeader& h = *x.h;
  memset(f, 0, sizeof *f);
  f->mi_cols = h.mi_cols;
  f->mi_rows = h.mi_rows;
  f->sb64_cols = h.sb64_cols;
  f->sb64_rows = h.sb64_rows;
  f->ss_x = (uint8_t)h.ss_x;
  f->ss_y = (uint8_t)h.ss_y;
  f->bit_depth = (uint8_t)h.bit_depth;
  f->frame_is_intra = h.frame_is_intra;
  f->tx_mode = h.tx_mode;
  f->reference_mode = h.reference_mode;
  f->interp_filter = h.interpolation_filter;
  f->allow_hp = h.allow_high_precision_mv;
  f->comp_fixed_ref = h.comp_fixed_ref;
  f->comp_var_ref[0] = h.comp_var_ref[0];
  f->comp_var_ref[1] = h.comp_var_ref[1];
  for (int i = 0; i < 4; ++i) f->sign_bias[i] = h.ref_frame_sign_bias[i];
  f->lossless = h.lossless;
  f->legacy_uv = h.legacy_uv;
  f->tile_cols_log2 = (uint8_t)h.tile_cols_log2;
  f->tile_rows_log2 = (uint8_t)h.tile_rows_log2;
  for (int i = 0; i < 3; ++i) f->ref_ok[i] = x.ref_ok[i];
  f->use_prev = x.use_prev;
  f->probs = *x.probs;
  for (int t = 0; t < 4; ++t)
    for (int pt = 0; pt < 2; ++pt)
      for (int rt = 0; rt < 2; ++rt)
        for (int band = 0; band < 6; ++band)
          for (int k = 0; k < 3; ++k) {
            uint64_t w = 0;
            for (int cx = 0; cx < 6; ++cx) w |= (uint64_t)x.probs->coef[t][pt][rt][band][cx][k] << (8 * cx);
            f->coef_pk[t][pt][rt][band][k] = w;
          }
}

// A frame's tile data split into tiles (reference src/decoder/block.rs:
// 1726-1763) and grouped into one chain per tile column, its tiles in row
// order. `data_off` is where the frame's tile data sits in the batch's
// bytes. Returns null, or the host parser's message for a tile size that
// runs past the data (the caller then leaves the frame to the host parser,
// which reports it in its order).
inline const char* plan_frame(const rv9::syn::FrameHeader& h, const uint8_t* data, size_t len, uint64_t data_off,
                              uint32_t frame, std::vector<Span>* spans, std::vector<Chain>* chains) {
  const uint32_t tile_cols = 1u << h.tile_cols_log2, tile_rows = 1u << h.tile_rows_log2;
  const size_t span0 = spans->size();
  size_t pos = 0;
  for (uint32_t row = 0; row < tile_rows; ++row)
    for (uint32_t col = 0; col < tile_cols; ++col) {
      const bool last = row == tile_rows - 1 && col == tile_cols - 1;
      size_t size;
      if (last) {
        size = len - pos;
      } else {
        if (pos + 4 > len) return "tile size runs past the end of the frame";
        size = ((size_t)data[pos] << 24) | ((size_t)data[pos + 1] << 16) | ((size_t)data[pos + 2] << 8) | data[pos + 3];
        pos += 4;
      }
      if (pos + size > len) return "tile runs past the end of the frame";
      Span s;
      s.off = data_off + pos;
      s.size = (uint32_t)size;
      s.mi_row_start = rv9::syn::tile_offset(row, h.mi_rows, h.tile_rows_log2);
      s.mi_row_end = rv9::syn::tile_offset(row + 1, h.mi_rows, h.tile_rows_log2);
      s.index = row * tile_cols + col;
      spans->push_back(s);
      pos += size;
    }
  // Chains: column c's spans are span0 + row * tile_cols + c; gather them
  // contiguous per column.
  std::vector<Span> byrow(spans->begin() + span0, spans->end());
  spans->resize(span0);
  for (uint32_t col = 0; col < tile_cols; ++col) {
    Chain ch;
    memset(&ch, 0, sizeof ch);
    ch.frame = frame;
    ch.first_span = (uint32_t)spans->size();
    ch.n_spans = tile_rows;
    ch.mi_col_start = rv9::syn::tile_offset(col, h.mi_cols, h.tile_cols_log2);
    ch.mi_col_end = rv9::syn::tile_offset(col + 1, h.mi_cols, h.tile_cols_log2);
    for (uint32_t row = 0; row < tile_rows; ++row) spans->push_back(byrow[row * tile_cols + col]);
    chain_caps(ch.mi_col_end - ch.mi_col_start, h.mi_rows, h.ss_x, h.ss_y, &ch.blocks_cap, &ch.toks_cap,
               &ch.coefs_cap);
    chains->push_back(ch);
  }
  return nullptr;
}

}  // namespace tp
}  // namespace rv9g

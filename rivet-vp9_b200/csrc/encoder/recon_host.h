// Host reconstruction for the stream generator's closed loop: the same
// per-sample arithmetic as the CUDA kernels (dsp_math.cuh), sequenced on the
// CPU. The encoder predicts from what a decoder will reconstruct, so every
// function here mirrors the decoding process exactly (inverse transforms,
// intra edges and predictors, inter prediction with motion vector clamping and
// reference scaling, the loop filter).
#pragma once
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../../include/rv9_records.h"
#include "../common/vp9_consts.h"
#include "../common/vp9_tables.h"
#include "../gpu/dsp_math.cuh"

namespace rv9enc {

struct Plane16 {
  std::vector<uint16_t> d;
  int stride = 0, height = 0;
  uint16_t* row(int y) { return d.data() + (size_t)y * stride; }
  const uint16_t* row(int y) const { return d.data() + (size_t)y * stride; }
};

struct Picture16 {
  Plane16 p[3];
  int width = 0, height = 0;  // luma, visible
  int ss_x = 1, ss_y = 1, bit_depth = 8;
  void alloc(int w, int h, int ssx, int ssy, int bd) {
    width = w;
    height = h;
    ss_x = ssx;
    ss_y = ssy;
    bit_depth = bd;
    int aw = ((w + 63) / 64) * 64, ah = ((h + 63) / 64) * 64;
    for (int i = 0; i < 3; ++i) {
      p[i].stride = i ? aw >> ssx : aw;
      p[i].height = i ? ah >> ssy : ah;
      p[i].d.assign((size_t)p[i].stride * p[i].height, 0);
    }
  }
  int pw(int i) const { return i ? (width + ss_x) >> ss_x : width; }
  int ph(int i) const { return i ? (height + ss_y) >> ss_y : height; }
};

// The dequantised inverse transform of `coefs` (raster, n0 x n0) added to dst.
inline void itx_add(const int32_t* coefs, int n, int tx_type, int eob, int bd, uint16_t* dst, int stride) {
  using namespace rv9g;
  const int maxv = (1 << bd) - 1, n0 = 1 << n;
  auto run = [&](auto lane) {
    using V = decltype(lane);
    if (eob == 1 && tx_type == 0) {
      int shift = (n + 2) < 6 ? (n + 2) : 6;
      V v = V::load(coefs[0]).mul(11585).rshift(14);
      int res = v.mul(11585).rshift(14).rshift(shift).residual();
      for (int i = 0; i < n0; ++i)
        for (int j = 0; j < n0; ++j) {
          int x = dst[i * stride + j] + res;
          dst[i * stride + j] = (uint16_t)(x < 0 ? 0 : (x > maxv ? maxv : x));
        }
      return;
    }
    typename V::store_t s[32][32];
    for (int r = 0; r < n0; ++r)
      for (int c = 0; c < n0; ++c) s[r][c] = coefs[r * n0 + c];
    int row_kind = (tx_type == 0 || tx_type == 1) ? 0 : 1;
    int col_kind = (tx_type == 0 || tx_type == 2) ? 0 : 1;
    auto pass = [&](V* t, int kind) {
      switch (n) {
        case 2: tx1d<2>(t, kind, 0); break;
        case 3: tx1d<3>(t, kind, 0); break;
        case 4: tx1d<4>(t, kind, 0); break;
        default: tx1d<5>(t, kind, 0); break;
      }
    };
    for (int r = 0; r < n0; ++r) {
      bool nz = false;
      for (int c = 0; c < n0; ++c) nz |= s[r][c] != 0;
      if (!nz) continue;
      V t[32];
      for (int c = 0; c < n0; ++c) t[c] = V::load(s[r][c]);
      pass(t, row_kind);
      for (int c = 0; c < n0; ++c) s[r][c] = t[c].v;
    }
    int shift = (n + 2) < 6 ? (n + 2) : 6;
    for (int c = 0; c < n0; ++c) {
      V t[32];
      for (int i = 0; i < n0; ++i) t[i] = V::load(s[i][c]);
      pass(t, col_kind);
      for (int i = 0; i < n0; ++i) {
        int x = dst[i * stride + c] + t[i].rshift(shift).residual();
        dst[i * stride + c] = (uint16_t)(x < 0 ? 0 : (x > maxv ? maxv : x));
      }
    }
  };
  if (bd > 8)
    run(rv9g::L64{0});
  else
    run(rv9g::L32{0});
}

// Intra prediction of one transform block in place (the decoding process's
// edge assembly, spec 8.5.1.1, with the predictors of dsp_math.cuh).
inline void intra_pred(Plane16& buf, int mode, int x, int y, int tx_sz, bool have_left, bool have_above,
                       bool not_on_right, int max_x, int max_y, int bd) {
  const int log2 = tx_sz + 2, size = 1 << log2;
  const int base = 1 << (bd - 1);
  int32_t above[66], left[32];
  if (have_above) {
    const uint16_t* row = buf.row(y - 1);
    for (int i = 0; i < 2 * size; ++i) {
      int xx = (i < size || (not_on_right && tx_sz == 0)) ? x + i : x + size - 1;
      above[1 + i] = row[std::min(max_x, xx)];
    }
    above[0] = have_left ? row[std::min(max_x, x - 1)] : base + 1;
  } else {
    for (int i = 0; i <= 2 * size; ++i) above[i] = base - 1;
  }
  for (int i = 0; i < size; ++i) left[i] = have_left ? buf.row(std::min(max_y, y + i))[x - 1] : base + 1;
  int32_t sa = 0, sl = 0;
  for (int i = 0; i < size; ++i) {
    sa += above[1 + i];
    sl += left[i];
  }
  int32_t dc = rv9g::intra_dc(log2, sa, sl, have_left, have_above, bd);
  for (int i = 0; i < size; ++i) {
    uint16_t* d = buf.row(y + i) + x;
    for (int j = 0; j < size; ++j)
      d[j] = (uint16_t)rv9g::intra_pixel(mode, i, j, size, above, left, dc, (1 << bd) - 1);
  }
}

// Block-to-reference geometry of inter prediction (spec 8.5.2.2-8.5.2.3):
// the clamped motion vector of a w x h region at (x, y) of `plane` of a
// block, scaled into the reference.
struct RefPos {
  int start_x, start_y, step_x, step_y;
};

inline RefPos ref_position(int mv_r, int mv_c, int plane, int x, int y, int mi_row, int mi_col, int mi_size,
                           int mi_rows, int mi_cols, int ss_x, int ss_y, int64_t xs, int64_t ys) {
  int sx = plane ? ss_x : 0, sy = plane ? ss_y : 0;
  int bh = vp9t_num_8x8_high[mi_size], bw = vp9t_num_8x8_wide[mi_size];
  int to_top = -((mi_row * 8) * 16) >> sy;
  int to_bottom = (((mi_rows - bh - mi_row) * 8) * 16) >> sy;
  int to_left = -((mi_col * 8) * 16) >> sx;
  int to_right = (((mi_cols - bw - mi_col) * 8) * 16) >> sx;
  int spel_left = (4 + ((bw * 8) >> sx)) << 4;
  int spel_top = (4 + ((bh * 8) >> sy)) << 4;
  int c0 = std::min(std::max((2 * mv_r) >> sy, to_top - spel_top), to_bottom + spel_top - 16);
  int c1 = std::min(std::max((2 * mv_c) >> sx, to_left - spel_left), to_right + spel_left - 16);
  int64_t base_x = ((int64_t)x * xs) >> 14, base_y = ((int64_t)y * ys) >> 14;
  int64_t luma_x = plane ? ((int64_t)x << ss_x) : x, luma_y = plane ? ((int64_t)y << ss_y) : y;
  int64_t frac_x = ((16 * luma_x * xs) >> 14) & 15, frac_y = ((16 * luma_y * ys) >> 14) & 15;
  RefPos p;
  p.step_x = (int)((16 * xs) >> 14);
  p.step_y = (int)((16 * ys) >> 14);
  p.start_x = (int)((base_x << 4) + (((int64_t)c1 * xs) >> 14) + frac_x);
  p.start_y = (int)((base_y << 4) + (((int64_t)c0 * ys) >> 14) + frac_y);
  return p;
}

// The 8-tap prediction of a w x h region (spec 8.5.2.4) into out.
inline void inter_pred(const Plane16& ref, int last_x, int last_y, const RefPos& p, int w, int h, int filter, int bd,
                       uint16_t* out, int out_stride) {
  const int maxv = (1 << bd) - 1;
  const int ih = (((h - 1) * p.step_y + 15) >> 4) + 8;
  const int y0 = (p.start_y >> 4) - 3;
  uint16_t tmp[136 * 64];
  const int32_t(*f)[8] = vp9t_subpel_filters[filter];
  for (int r = 0; r < ih; ++r) {
    const uint16_t* src = ref.row(std::min(std::max(y0 + r, 0), last_y));
    for (int c = 0; c < w; ++c) {
      int pos = p.start_x + p.step_x * c;
      int base = (pos >> 4) - 3;
      const int32_t* t = f[pos & 15];
      int32_t sum = 0;
      for (int k = 0; k < 8; ++k) sum += t[k] * src[std::min(std::max(base + k, 0), last_x)];
      tmp[r * 64 + c] = (uint16_t)std::min(std::max((sum + 64) >> 7, 0), maxv);
    }
  }
  for (int r = 0; r < h; ++r) {
    int pos = (p.start_y & 15) + p.step_y * r;
    const int32_t* t = f[pos & 15];
    int base = pos >> 4;
    for (int c = 0; c < w; ++c) {
      int32_t sum = 0;
      for (int k = 0; k < 8; ++k) sum += t[k] * tmp[(base + k) * 64 + c];
      out[r * out_stride + c] = (uint16_t)std::min(std::max((sum + 64) >> 7, 0), maxv);
    }
  }
}

// The loop filter of a reconstructed frame (spec 8.8), superblocks in raster
// order, each filtered by the kernels' procedure (vertical edges by rows, then
// horizontal edges by columns, over a tile from 8 samples above and left).
void loop_filter(Picture16& pic, const rv9_frame_desc& d, const rv9_block* blocks, size_t n_blocks);

}  // namespace rv9enc

// Host build of the CUDA kernels' per-sample arithmetic (dsp_math.cuh) for
// the CPU tests: the same 1D transforms, DC-only shortcut, intra closed forms
// and loop-filter line as the kernels, sequenced as the kernels sequence them
// (rows, then columns with the final rounding), without the warp plumbing.
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/rv9_records.h"

#include "../../rivet-vp9_b200/csrc/gpu/dsp_math.cuh"
#include "../../rivet-vp9_b200/csrc/gpu/md5.cuh"

using namespace rv9g;

template <class V, int n>
static void itx2d(const int32_t* coefs, int tx_type, bool lossless, uint16_t* dst, int stride, int maxv) {
  constexpr int n0 = 1 << n;
  typename V::store_t s[n0][n0];
  for (int r = 0; r < n0; ++r)
    for (int c = 0; c < n0; ++c) s[r][c] = coefs[r * n0 + c];
  int row_kind = lossless ? 2 : ((tx_type == 0 || tx_type == 1) ? 0 : 1);
  int col_kind = lossless ? 2 : ((tx_type == 0 || tx_type == 2) ? 0 : 1);
  for (int r = 0; r < n0; ++r) {
    bool nz = false;
    for (int c = 0; c < n0; ++c) nz |= s[r][c] != 0;
    if (!nz) continue;
    V t[n0];
    for (int c = 0; c < n0; ++c) t[c] = V::load(s[r][c]);
    tx1d<n>(t, row_kind, 2);
    for (int c = 0; c < n0; ++c) s[r][c] = t[c].v;
  }
  constexpr int shift = (n + 2) < 6 ? (n + 2) : 6;
  for (int c = 0; c < n0; ++c) {
    V t[n0];
    for (int i = 0; i < n0; ++i) t[i] = V::load(s[i][c]);
    tx1d<n>(t, col_kind, 0);
    for (int i = 0; i < n0; ++i) {
      V r = lossless ? t[i] : t[i].rshift(shift);
      int v = dst[i * stride + c] + r.residual();
      dst[i * stride + c] = (uint16_t)(v < 0 ? 0 : (v > maxv ? maxv : v));
    }
  }
}

template <class V>
static void itx_any(const int32_t* coefs, int n, int tx_type, bool lossless, int eob, int bd, uint16_t* dst,
                    int stride) {
  int maxv = (1 << bd) - 1, n0 = 1 << n;
  if (eob == 1 && tx_type == 0 && !lossless) {
    int shift = (n + 2) < 6 ? (n + 2) : 6;
    V v = V::load(coefs[0]).mul(11585).rshift(14);
    V w2 = v.mul(11585).rshift(14);
    int res = w2.rshift(shift).residual();
    for (int i = 0; i < n0 * n0; ++i) {
      int r = i >> n, c = i & (n0 - 1);
      int x = dst[r * stride + c] + res;
      dst[r * stride + c] = (uint16_t)(x < 0 ? 0 : (x > maxv ? maxv : x));
    }
    return;
  }
  switch (n) {
    case 2: itx2d<V, 2>(coefs, tx_type, lossless, dst, stride, maxv); break;
    case 3: itx2d<V, 3>(coefs, tx_type, lossless, dst, stride, maxv); break;
    case 4: itx2d<V, 4>(coefs, tx_type, lossless, dst, stride, maxv); break;
    default: itx2d<V, 5>(coefs, tx_type, lossless, dst, stride, maxv); break;
  }
}

extern "C" {

void shim_itx(const int32_t* coefs, int n, int tx_type, int lossless, int eob, int bd, uint16_t* dst, int stride) {
  if (bd > 8)
    itx_any<L64>(coefs, n, tx_type, lossless != 0, eob, bd, dst, stride);
  else
    itx_any<L32>(coefs, n, tx_type, lossless != 0, eob, bd, dst, stride);
}

void shim_intra(int mode, int log2, const int32_t* above, const int32_t* left, int have_left, int have_above, int bd,
                uint16_t* dst, int stride) {
  int size = 1 << log2;
  int32_t sa = 0, sl = 0;
  for (int i = 0; i < size; ++i) {
    sa += above[1 + i];
    sl += left[i];
  }
  int32_t dc = intra_dc(log2, sa, sl, have_left != 0, have_above != 0, bd);
  for (int i = 0; i < size; ++i)
    for (int j = 0; j < size; ++j)
      dst[i * stride + j] = (uint16_t)intra_pixel(mode, i, j, size, above, left, dc, (1 << bd) - 1);
}

void shim_lf(uint16_t* buf, int filter_size, int limit, int blimit, int thresh, int bd) {
  int s[16];
  for (int i = 0; i < 16; ++i) s[i] = buf[i];
  lf_line(s, filter_size, limit, blimit, thresh, bd);
  for (int i = 0; i < 16; ++i) buf[i] = (uint16_t)s[i];
}


}  // extern "C"

// The loop-filter kernel's superblock procedure, run over the superblocks in
// raster order: per superblock, the region from 8 samples above and left is
// copied to a tile, the edge entries are decided, vertical edges filter one
// row at a time, horizontal edges one column at a time, and the tile is
// written back. `planes` are SB-aligned with the given strides.
extern "C" void shim_lf_frame(const rv9_frame_desc* d, const rv9_block* blocks, int n_blocks, uint16_t* planes0,
                              uint16_t* planes1, uint16_t* planes2) {
  uint16_t* planes[3] = {planes0, planes1, planes2};
  int aw = d->sb64_cols * 64, ah = d->sb64_rows * 64;
  int stride[3] = {aw, aw >> d->ss_x, aw >> d->ss_x};
  // LvlLookup and limits (8.8.1).
  uint8_t lvl[8][4][2];
  uint8_t lim[64], blim[64], thr[64];
  int n_shift = d->lf_level >> 5;
  for (int seg = 0; seg < 8; ++seg) {
    int lvl_seg = d->lf_level;
    if (d->seg.enabled && d->seg.feature_enabled[seg][1]) {
      int data = d->seg.feature_data[seg][1];
      lvl_seg = d->seg.abs_or_delta_update ? data : data + d->lf_level;
      lvl_seg = lvl_seg < 0 ? 0 : (lvl_seg > 63 ? 63 : lvl_seg);
    }
    for (int rf = 0; rf < 4; ++rf)
      for (int mode = 0; mode < 2; ++mode) {
        int v = lvl_seg;
        if (d->lf_delta_enabled) {
          v = lvl_seg + d->lf_ref_deltas[rf] * (1 << n_shift);
          if (rf > 0) v += d->lf_mode_deltas[mode] * (1 << n_shift);
        }
        lvl[seg][rf][mode] = (uint8_t)(v < 0 ? 0 : (v > 63 ? 63 : v));
      }
  }
  int shift = d->lf_sharpness > 4 ? 2 : (d->lf_sharpness > 0 ? 1 : 0);
  for (int l = 0; l < 64; ++l) {
    int limit = l >> shift;
    if (d->lf_sharpness > 0 && limit > 9 - d->lf_sharpness) limit = 9 - d->lf_sharpness;
    if (limit < 1) limit = 1;
    lim[l] = (uint8_t)limit;
    blim[l] = (uint8_t)(2 * (l + 2) + limit);
    thr[l] = (uint8_t)(l >> 4);
  }
  std::vector<uint32_t> lf_mi((size_t)d->mi_rows * d->mi_cols);
  for (int i = 0; i < n_blocks; ++i) {
    const rv9_block& b = blocks[i];
    uint32_t v = lf_block_record(b.mi_size, b.tx_size, (b.flags & RV9_BLK_SKIP) ? 1 : 0, b.segment_id, b.y_mode,
                                 b.ref_frame[0], lvl, d->legacy_uv, d->ss_x, d->ss_y);
    int w8 = 1 << ((0x3ea5400u >> (2 * b.mi_size)) & 3), h8 = 1 << ((0x3b99100u >> (2 * b.mi_size)) & 3);
    for (int y = b.mi_row; y < (int)std::min<uint32_t>(b.mi_row + h8, d->mi_rows); ++y)
      for (int x = b.mi_col; x < (int)std::min<uint32_t>(b.mi_col + w8, d->mi_cols); ++x)
        lf_mi[(size_t)y * d->mi_cols + x] = v;
  }
  LfParams P{(int)d->mi_cols, (int)d->mi_rows, d->ss_x, d->ss_y, lf_mi.data(), lim, blim, thr};
  static int16_t px[3][72][80];
  static LfEdge edges[3][2][16][16];
  for (int sr = 0; sr < (int)d->sb64_rows; ++sr)
    for (int sc = 0; sc < (int)d->sb64_cols; ++sc) {
      int row = sr * 8, col = sc * 8;
      for (int i = 0; i < 3 * 2 * 256; ++i) {
        int plane = i / 512, pass = (i >> 8) & 1, ed = (i >> 4) & 15, rn = i & 15;
        edges[plane][pass][ed][rn] = lf_edge_entry(P, plane, pass, row, col, ed, rn);
      }
      int rows_p[3], cols_p[3], x0s[3], y0s[3];
      for (int p = 0; p < 3; ++p) {
        int sxp = p ? d->ss_x : 0, syp = p ? d->ss_y : 0;
        rows_p[p] = 64 >> syp;
        cols_p[p] = 64 >> sxp;
        x0s[p] = (col * 8) >> sxp;
        y0s[p] = (row * 8) >> syp;
        for (int r = 0; r < rows_p[p] + 8; ++r)
          for (int c = 0; c < cols_p[p] + 8; ++c) {
            int gy = y0s[p] - 8 + r, gx = x0s[p] - 8 + c;
            if (gy >= 0 && gx >= 0 && (r >= 8 || c >= 8)) px[p][r][c] = (int16_t)planes[p][(size_t)gy * stride[p] + gx];
          }
      }
      for (int p = 0; p < 3; ++p)
        for (int r = 0; r < rows_p[p]; ++r)
          lf_vertical_row(&px[p][8 + r][0], edges[p][0], 16 >> (p ? d->ss_x : 0), r >> 2, d->bit_depth);
      for (int p = 0; p < 3; ++p)
        for (int c = 0; c < cols_p[p]; ++c)
          lf_horizontal_col(&px[p][0][8 + c], 80, 72, edges[p][1], 16 >> (p ? d->ss_y : 0), c >> 2, d->bit_depth);
      for (int p = 0; p < 3; ++p)
        for (int r = 0; r < rows_p[p] + 8; ++r)
          for (int c = 0; c < cols_p[p] + 8; ++c) {
            int gy = y0s[p] - 8 + r, gx = x0s[p] - 8 + c;
            if (gy >= 0 && gx >= 0 && (r >= 8 || c >= 8)) planes[p][(size_t)gy * stride[p] + gx] = (uint16_t)px[p][r][c];
          }
    }
}

// The device MD5's steps on the host: data in 64-byte blocks, then the
// padding, exactly as the frame digest kernel sequences them.
extern "C" void shim_md5(const uint8_t* data, uint64_t len, uint8_t* out) {
  uint32_t t[64];
  md5_sine_table(t);
  Md5State h;
  md5_init(&h);
  const uint64_t total = md5_padded_bytes(len);
  for (uint64_t pos = 0; pos < total; pos += 64) {
    uint32_t w[16];
    for (int q = 0; q < 16; ++q) {
      uint32_t v = 0;
      for (int b = 0; b < 4; ++b) {
        const uint64_t k = pos + 4 * q + b;
        v |= (uint32_t)(k < len ? data[k] : md5_pad_byte(k, len)) << (8 * b);
      }
      w[q] = v;
    }
    md5_block(&h, w, t);
  }
  md5_digest(h, out);
}

// CUDA kernels of VP9 reconstruction for sm_100a.
//
// One frame is reconstructed by a short chain of launches on the decoder's
// stream (reference process: FrameDec::replay, src/decoder/block.rs:1405-1498,
// then loopfilter::filter_frame, src/decoder/loopfilter.rs:51-81):
//
//   k_prep        three independent parts in one launch: zero the samples
//                 beyond the mode-info area (the reference reconstructs into
//                 zeroed planes, src/decoder/pool.rs:1-6), the per-8x8
//                 loop-filter records from the block records, and the
//                 pending marks of intra transform blocks' 4x4 cells
//   k_inter_small / k_inter
//                 inter prediction: a warp per region of at most 16x16, a
//                 CTA per larger one; 8-tap H then V passes through shared
//                 memory, scaled references, compound averaging fused
//                 (src/dsp/inter.rs, pixel.rs)
//   k_inter_res   inverse transform + add of inter blocks' residuals, all
//                 transform sizes in one launch: 8, 4, 2 or 1 blocks per
//                 warp by size (src/dsp/itx.rs)
//   k_intra       intra prediction + residual as a dependency wavefront:
//                 a persistent grid takes rows of transform blocks in
//                 superblock anti-diagonal order and each warp waits only
//                 for the 4x4 cells its edges read
//   k_lf_rows     loop filter: one CTA per superblock row, left to right,
//                 each superblock's vertical then horizontal edges in shared
//                 memory; a row waits only for the row above to be one
//                 superblock ahead
//
// Inter prediction reads only reference frames, so it runs fully parallel
// before the intra wavefront. Every wait is bounded: on timeout a kernel
// records an error code, sets the abort flag and returns.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <mutex>

#include "dsp_math.cuh"
#include "md5.cuh"
#include "engine.h"
#include "engine_types.h"

namespace rv9g {

__constant__ int16_t c_filters[4][16][8];


template <class T>
__device__ __forceinline__ T* plane_ptr(const PlanePtr& p) {
  return reinterpret_cast<T*>(p.data);
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ---------------------------------------------------------------------------
// Zero the samples of the SB-aligned planes outside the mode-info area.

// Zeroing the samples beyond the mode-info area of one plane: part `bx` of
// `gx` (the reference reconstructs into zeroed planes).
template <class T>
__device__ __forceinline__ void zero_pad_part(const KFrame& k, int plane, int bx, int gx) {
  int sx = plane ? k.ss_x : 0, sy = plane ? k.ss_y : 0;
  int mw = (k.mi_cols * 8) >> sx, mh = (k.mi_rows * 8) >> sy;
  int aw = (k.sb64_cols * 64) >> sx, ah = (k.sb64_rows * 64) >> sy;
  T* d = plane_ptr<T>(k.cur[plane]);
  int stride = k.cur[plane].stride;
  // Right strip then bottom strip.
  int right = (aw - mw) * mh;
  int total = right + (ah - mh) * aw;
  for (int i = bx * blockDim.x + threadIdx.x; i < total; i += gx * blockDim.x) {
    int x, y;
    if (i < right) {
      y = i / (aw - mw);
      x = mw + i % (aw - mw);
    } else {
      int j = i - right;
      y = mh + j / aw;
      x = j % aw;
    }
    d[(size_t)y * stride + x] = 0;
  }
}

// Loop-filter record per 8x8 (the MiInfo fields loopfilter.rs reads) of
// block i: bits 0-5 level, 6-7 luma tx size, 8-9 chroma tx size, 10-13
// block size, 14 coded (intra, or not skipped).
__device__ __forceinline__ void lf_mi_block(const KFrame& k, int i) {
  const rv9_block& b = k.blocks[i];
  uint32_t v = lf_block_record(b.mi_size, b.tx_size, (b.flags & RV9_BLK_SKIP) ? 1 : 0, b.segment_id, b.y_mode,
                               b.ref_frame[0], k.lvl, k.legacy_uv, k.ss_x, k.ss_y);
  int w8 = 1 << ((0x3ea5400u >> (2 * b.mi_size)) & 3), h8 = 1 << ((0x3b99100u >> (2 * b.mi_size)) & 3);
  int ye = min((int)b.mi_row + h8, k.mi_rows);
  int xe = min((int)b.mi_col + w8, k.mi_cols);
  for (int y = b.mi_row; y < ye; ++y)
    for (int x = b.mi_col; x < xe; ++x) k.lf_mi[(size_t)y * k.mi_cols + x] = v;
}

// Intra item i's 4x4 cells marked pending.
__device__ __forceinline__ void intra_mark_item(const KFrame& k, int i) {
  const IntraItem it = k.intra[i];
  int n = 1 << it.tx_size;  // cells per side
  uint8_t* cells = k.cells[it.plane];
  int cs = k.cell_stride[it.plane];
  int cx = it.x >> 2, cy = it.y >> 2;
  for (int y = 0; y < n; ++y)
    for (int x = 0; x < n; ++x) cells[(size_t)(cy + y) * cs + cx + x] = 1;
}

// A frame's preparation, three independent parts in one launch by CTA range:
// the zeroed padding (zp_per_plane CTAs per plane), the loop-filter records
// (one thread per block) and the intra cells' marks (one thread per item).
constexpr int kPrepThreads = 256;
struct PrepSplit {
  int zp_per_plane, zp, lf, mark;  // CTAs of each part (zp = 3 zp_per_plane or 0)
  int n_blocks;
};

template <class T>
__device__ __forceinline__ void prep_cta(const KFrame& k, const PrepSplit& ps, int b) {
  if (b < ps.zp) {
    zero_pad_part<T>(k, b / ps.zp_per_plane, b % ps.zp_per_plane, ps.zp_per_plane);
    return;
  }
  b -= ps.zp;
  if (b < ps.lf) {
    const int i = b * kPrepThreads + threadIdx.x;
    if (i < ps.n_blocks) lf_mi_block(k, i);
    return;
  }
  b -= ps.lf;
  const int i = b * kPrepThreads + threadIdx.x;
  if (i < k.n_intra) intra_mark_item(k, i);
}

template <class T>
__global__ void __launch_bounds__(kPrepThreads) k_prep(KFrame k, PrepSplit ps) {
  prep_cta<T>(k, ps, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Inter prediction.

struct RefPos {
  int start_x, start_y, step_x, step_y;
};

__device__ __forceinline__ int32_t q2(int32_t v) { return (v < 0 ? v - 1 : v + 1) / 2; }
__device__ __forceinline__ int32_t q4(int32_t v) { return (v < 0 ? v - 2 : v + 2) / 4; }

// Motion vector selection, clamping and scaling (reference
// src/decoder/recon.rs:115-167, src/decoder/mod.rs:516-541).
__device__ RefPos ref_position(const KFrame& k, const rv9_block& b, int ref_list, int plane, int x, int y,
                               int block_idx) {
  const int32_t(*bm)[2] = b.mv[ref_list];
  int32_t mv0, mv1;
  if (plane == 0 || b.mi_size >= 3) {
    mv0 = bm[block_idx][0];
    mv1 = bm[block_idx][1];
  } else {
    int usx = k.legacy_uv ? 1 : k.ss_x, usy = k.legacy_uv ? 1 : k.ss_y;
    if (usx == 0 && usy == 0) {
      mv0 = bm[block_idx][0];
      mv1 = bm[block_idx][1];
    } else if (usx == 0) {
      mv0 = q2(bm[block_idx][0] + bm[block_idx + 2][0]);
      mv1 = q2(bm[block_idx][1] + bm[block_idx + 2][1]);
    } else if (usy == 0) {
      mv0 = q2(bm[block_idx][0] + bm[block_idx + 1][0]);
      mv1 = q2(bm[block_idx][1] + bm[block_idx + 1][1]);
    } else {
      mv0 = q4(bm[0][0] + bm[1][0] + bm[2][0] + bm[3][0]);
      mv1 = q4(bm[0][1] + bm[1][1] + bm[2][1] + bm[3][1]);
    }
  }
  int sx = plane ? k.ss_x : 0, sy = plane ? k.ss_y : 0;
  // num_8x8 wide / high by block size, as 2-bit log2 fields of a constant.
  int bh = 1 << ((0x3b99100u >> (2 * b.mi_size)) & 3), bw = 1 << ((0x3ea5400u >> (2 * b.mi_size)) & 3);
  int mi_row = b.mi_row, mi_col = b.mi_col;
  int to_top = -((mi_row * 8) * 16) >> sy;
  int to_bottom = (((k.mi_rows - bh - mi_row) * 8) * 16) >> sy;
  int to_left = -((mi_col * 8) * 16) >> sx;
  int to_right = (((k.mi_cols - bw - mi_col) * 8) * 16) >> sx;
  int spel_left = (4 + ((bw * 8) >> sx)) << 4;
  int spel_right = spel_left - 16;
  int spel_top = (4 + ((bh * 8) >> sy)) << 4;
  int spel_bottom = spel_top - 16;
  int32_t c0 = clampi((2 * mv0) >> sy, to_top - spel_top, to_bottom + spel_bottom);
  int32_t c1 = clampi((2 * mv1) >> sx, to_left - spel_left, to_right + spel_right);
  int ri = b.ref_frame[ref_list] - 1;
  int64_t xs = k.ref_xs[ri], ys = k.ref_ys[ri];
  int64_t base_x = ((int64_t)x * xs) >> 14, base_y = ((int64_t)y * ys) >> 14;
  int64_t luma_x = plane ? ((int64_t)x << k.ss_x) : x;
  int64_t luma_y = plane ? ((int64_t)y << k.ss_y) : y;
  int64_t frac_x = ((16 * luma_x * xs) >> 14) & 15;
  int64_t frac_y = ((16 * luma_y * ys) >> 14) & 15;
  int64_t dx = (((int64_t)c1 * xs) >> 14) + frac_x;
  int64_t dy = (((int64_t)c0 * ys) >> 14) + frac_y;
  RefPos p;
  p.step_x = (int)((16 * xs) >> 14);
  p.step_y = (int)((16 * ys) >> 14);
  p.start_x = (int)((base_x << 4) + dx);
  p.start_y = (int)((base_y << 4) + dy);
  return p;
}

constexpr int kInterThreads = 128;
constexpr int kInterTmpRows = 64 * 2 + 8;  // (h-1)*step/16 + 8 rows at steps up to 32

// One prediction region: the horizontal pass over the clamped reference
// rows into shared memory, then the vertical pass; for compound blocks both
// predictions, then their rounded average (spec 8.5.2.3-8.5.2.5). NT
// threads cooperate (a warp, or the whole CTA), `tid` numbering them.
template <class T, int NT>
__device__ __forceinline__ void inter_unit(const KFrame& k, const InterUnit& u, int tid, uint16_t* tmp, int tpitch,
                                           uint16_t* pred, int ppitch) {
  auto sync = [] {
    if (NT == 32)
      __syncwarp();
    else
      __syncthreads();
  };
  const rv9_block& b = k.blocks[u.block];
  const int w = u.w4 * 4, h = u.h4 * 4, plane = u.plane;
  const int lw = 31 - __clz(w);  // widths are powers of two
  const int maxv = (1 << k.bit_depth) - 1;
  const bool compound = b.ref_frame[1] > 0;
  T* dst = plane_ptr<T>(k.cur[plane]) + (size_t)u.y * k.cur[plane].stride + u.x;
  const int dstride = k.cur[plane].stride;
  const int filter = b.interp_filter;
  for (int rl = 0; rl < (compound ? 2 : 1); ++rl) {
    RefPos p = ref_position(k, b, rl, plane, u.x, u.y, u.block_idx);
    const PlanePtr& rp = k.ref[b.ref_frame[rl] - 1][plane];
    const T* ref = plane_ptr<const T>(rp);
    const int last_x = rp.width - 1, last_y = rp.height - 1, rstride = rp.stride;
    const int ih = (((h - 1) * p.step_y + 15) >> 4) + 8;
    const int y0 = (p.start_y >> 4) - 3;
    if (p.step_x == 16) {
      // Unscaled: one filter phase for the whole unit, its taps in registers,
      // and no clamping when the window lies inside the reference.
      const int16_t* fp = c_filters[filter][p.start_x & 15];
      const int f0 = fp[0], f1 = fp[1], f2 = fp[2], f3 = fp[3], f4 = fp[4], f5 = fp[5], f6 = fp[6], f7 = fp[7];
      const int bx = (p.start_x >> 4) - 3;
      const bool inside = bx >= 0 && bx + w + 6 <= last_x;
      for (int i = tid; i < ih * w; i += NT) {
        const int r = i >> lw, c = i & (w - 1);
        const T* src = ref + (size_t)clampi(y0 + r, 0, last_y) * rstride;
        int32_t sum;
        if (inside) {
          const T* q = src + bx + c;
          sum = f0 * (int32_t)q[0] + f1 * (int32_t)q[1] + f2 * (int32_t)q[2] + f3 * (int32_t)q[3] +
                f4 * (int32_t)q[4] + f5 * (int32_t)q[5] + f6 * (int32_t)q[6] + f7 * (int32_t)q[7];
        } else {
          const int x = bx + c;
          sum = f0 * (int32_t)src[clampi(x, 0, last_x)] + f1 * (int32_t)src[clampi(x + 1, 0, last_x)] +
                f2 * (int32_t)src[clampi(x + 2, 0, last_x)] + f3 * (int32_t)src[clampi(x + 3, 0, last_x)] +
                f4 * (int32_t)src[clampi(x + 4, 0, last_x)] + f5 * (int32_t)src[clampi(x + 5, 0, last_x)] +
                f6 * (int32_t)src[clampi(x + 6, 0, last_x)] + f7 * (int32_t)src[clampi(x + 7, 0, last_x)];
        }
        tmp[r * tpitch + c] = (uint16_t)clampi((sum + 64) >> 7, 0, maxv);
      }
    } else {
      for (int i = tid; i < ih * w; i += NT) {
        const int r = i >> lw, c = i & (w - 1);
        int ry = clampi(y0 + r, 0, last_y);
        const T* src = ref + (size_t)ry * rstride;
        int pos = p.start_x + p.step_x * c;
        int base = (pos >> 4) - 3;
        const int16_t* f = c_filters[filter][pos & 15];
        int32_t sum = 0;
#pragma unroll
        for (int t = 0; t < 8; ++t) sum += f[t] * (int32_t)src[clampi(base + t, 0, last_x)];
        tmp[r * tpitch + c] = (uint16_t)clampi((sum + 64) >> 7, 0, maxv);
      }
    }
    sync();
    // The vertical pass: unscaled, one phase and rows r..r+7 of tmp.
    const bool vflat = p.step_y == 16;
    const int16_t* fv = c_filters[filter][p.start_y & 15];
    const int g0 = fv[0], g1 = fv[1], g2 = fv[2], g3 = fv[3], g4 = fv[4], g5 = fv[5], g6 = fv[6], g7 = fv[7];
    for (int i = tid; i < h * w; i += NT) {
      const int r = i >> lw, c = i & (w - 1);
      int32_t sum;
      if (vflat) {
        const uint16_t* q = tmp + r * tpitch + c;
        sum = g0 * (int32_t)q[0] + g1 * (int32_t)q[tpitch] + g2 * (int32_t)q[2 * tpitch] +
              g3 * (int32_t)q[3 * tpitch] + g4 * (int32_t)q[4 * tpitch] + g5 * (int32_t)q[5 * tpitch] +
              g6 * (int32_t)q[6 * tpitch] + g7 * (int32_t)q[7 * tpitch];
      } else {
        int pos = (p.start_y & 15) + p.step_y * r;
        int base = pos >> 4;
        const int16_t* f = c_filters[filter][pos & 15];
        sum = 0;
#pragma unroll
        for (int t = 0; t < 8; ++t) sum += f[t] * (int32_t)tmp[(base + t) * tpitch + c];
      }
      int v = clampi((sum + 64) >> 7, 0, maxv);
      if (!compound)
        dst[(size_t)r * dstride + c] = (T)v;
      else if (rl == 0)
        pred[r * ppitch + c] = (uint16_t)v;
      else
        dst[(size_t)r * dstride + c] = (T)((pred[r * ppitch + c] + v + 1) >> 1);
    }
    sync();
  }
}

// Regions larger than 16x16 (after the small ones in the list): one CTA of
// NT threads each.
template <class T, int NT>
__device__ __forceinline__ void inter_large_cta(const KFrame& k, int b) {
  __shared__ uint16_t tmp[kInterTmpRows * 64];
  __shared__ uint16_t pred[64 * 64];
  const InterUnit u = k.units[k.n_units_small + b];
  inter_unit<T, NT>(k, u, threadIdx.x, tmp, 64, pred, 64);
}

template <class T, int NT>
__global__ void __launch_bounds__(NT) k_inter(KFrame k) {
  inter_large_cta<T, NT>(k, blockIdx.x);
}

// Regions of at most 16x16 (the first n_units_small of the list): one warp
// each, four per CTA. Rows of the horizontal pass: (16-1)*32/16 + 8 at the
// largest reference step (2:1).
constexpr int kInterSmallRows = 38;
template <class T>
__device__ __forceinline__ void inter_small_cta(const KFrame& k, int b) {
  __shared__ uint16_t tmp[kInterThreads / 32][kInterSmallRows * 16];
  __shared__ uint16_t pred[kInterThreads / 32][16 * 16];
  const int warp = threadIdx.x >> 5;
  const int i = b * (kInterThreads / 32) + warp;
  if (i >= k.n_units_small) return;
  const InterUnit u = k.units[i];
  inter_unit<T, 32>(k, u, threadIdx.x & 31, tmp[warp], 16, pred[warp], 16);
}

template <class T>
__global__ void __launch_bounds__(kInterThreads) k_inter_small(KFrame k) {
  inter_small_cta<T>(k, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Inverse transform + add, one warp per transform block.


// Dequantise the recorded coefficients of `t` into the warp's scratch (zeroed
// first) and return the mask of rows holding a nonzero value (reference
// src/decoder/recon.rs:242-264).
template <class V>
__device__ uint32_t load_coefs(const KFrame& k, const rv9_tok& t, int seg, typename V::store_t* s, int lane) {
  const int n = 2 + t.tx_size, n0 = 1 << n, sp = n0 + 1;
  for (int i = lane; i < n0 * sp; i += 32) s[i] = 0;
  __syncwarp();
  const int pt = t.plane ? 1 : 0;
  const int64_t dcq = k.dc_q[seg][pt], acq = k.ac_q[seg][pt];
  uint32_t rows = 0;
  for (int i = lane; i < t.n_coef; i += 32) {
    uint32_t w = k.coefs[t.coef_start + i];
    int pos = RV9_COEF_POS(w);
    int64_t v = RV9_COEF_VAL(w);
    int64_t dq = v * (pos == 0 ? dcq : acq);
    if (t.tx_size == 3) dq /= 2;
    dq = dq < INT32_MIN ? INT32_MIN : (dq > INT32_MAX ? INT32_MAX : dq);
    int r = pos >> n, c = pos & (n0 - 1);
    s[r * sp + c] = (typename V::store_t)(int32_t)dq;
    rows |= 1u << r;
  }
  rows = __reduce_or_sync(0xffffffffu, rows);
  __syncwarp();
  return rows;
}

// The 2D transform of the scratch block added to dst (reference
// inverse_2d_add, src/dsp/itx.rs:519-570): rows by lanes, then columns.
template <class V, int n, class T>
__device__ void itx_add(typename V::store_t* s, uint32_t rows, int tx_type, bool lossless, T* dst, int dstride,
                        int maxv, int lane) {
  constexpr int n0 = 1 << n, sp = n0 + 1;
  const int row_kind = lossless ? 2 : ((tx_type == 0 || tx_type == 1) ? 0 : 1);
  const int col_kind = lossless ? 2 : ((tx_type == 0 || tx_type == 2) ? 0 : 1);
  if (lane < n0 && ((rows >> lane) & 1)) {
    V t[n0];
#pragma unroll
    for (int q = 0; q < n0; ++q) t[q] = V::load(s[lane * sp + q]);
    tx1d<n>(t, row_kind, 2);
#pragma unroll
    for (int q = 0; q < n0; ++q) s[lane * sp + q] = t[q].v;
  }
  __syncwarp();
  if (lane < n0) {
    V t[n0];
#pragma unroll
    for (int i = 0; i < n0; ++i) t[i] = V::load(s[i * sp + lane]);
    tx1d<n>(t, col_kind, 0);
    constexpr int shift = (n + 2) < 6 ? (n + 2) : 6;
#pragma unroll
    for (int i = 0; i < n0; ++i) {
      V r = lossless ? t[i] : t[i].rshift(shift);
      T* px = dst + (size_t)i * dstride + lane;
      *px = (T)clampi((int)*px + r.residual(), 0, maxv);
    }
  }
  __syncwarp();
}

// A transform block's residual added to dst (the prediction), by one warp.
// The residual every sample of a DC-only block gets (the reference's
// dc_only_value, src/dsp/itx.rs:684-694; exact for the 64-bit lane too,
// whose products here fit 32 bits).
template <class V>
__device__ int dc_only_residual(const KFrame& k, const rv9_tok& t, int seg) {
  const int n = 2 + t.tx_size;
  int pt = t.plane ? 1 : 0;
  int32_t dc = 0;
  if (t.n_coef > 0) {
    uint32_t w = k.coefs[t.coef_start];
    int64_t dq = (int64_t)RV9_COEF_VAL(w) * k.dc_q[seg][pt];
    if (t.tx_size == 3) dq /= 2;
    dq = dq < INT32_MIN ? INT32_MIN : (dq > INT32_MAX ? INT32_MAX : dq);
    dc = (int32_t)dq;
  }
  int shift = (n + 2) < 6 ? (n + 2) : 6;
  V v = V::load(dc).mul(11585).rshift(14);
  V w2 = V::load((int32_t)v.v).mul(11585).rshift(14);
  // The 64-bit lane multiplies the low 32 bits: v fits them.
  if (sizeof(typename V::store_t) == 4) w2 = v.mul(11585).rshift(14);
  return w2.rshift(shift).residual();
}

template <class V, class T>
__device__ void itx_add_size(int tx_size, typename V::store_t* s, uint32_t rows, int tx_type, bool lossless, T* dst,
                             int dstride, int maxv, int lane) {
  switch (tx_size) {
    case 0: itx_add<V, 2>(s, rows, tx_type, lossless, dst, dstride, maxv, lane); break;
    case 1: itx_add<V, 3>(s, rows, tx_type, lossless, dst, dstride, maxv, lane); break;
    case 2: itx_add<V, 4>(s, rows, tx_type, lossless, dst, dstride, maxv, lane); break;
    default: itx_add<V, 5>(s, rows, tx_type, lossless, dst, dstride, maxv, lane); break;
  }
}

constexpr int kResWarps = 4;

// A transform block's residual added to dst by a group of n0 lanes of a warp
// (lane l of the group: row l, then column l), `mask` the group's lanes:
// 4x4 blocks go eight to a warp, 8x8 four, 16x16 two, 32x32 one.
template <class V, int n, class T>
__device__ void residual_add_group(const KFrame& k, const rv9_tok& t, int seg, T* dst, int dstride,
                                   typename V::store_t* s, int l, unsigned mask) {
  constexpr int n0 = 1 << n, sp = n0 + 1;
  const int maxv = (1 << k.bit_depth) - 1;
  if (t.eob == 1 && t.tx_type == 0 && !k.lossless) {
    const int res = dc_only_residual<V>(k, t, seg);
    for (int r = 0; r < n0; ++r) {
      T* px = dst + (size_t)r * dstride + l;
      *px = (T)clampi((int)*px + res, 0, maxv);
    }
    return;
  }
  for (int i = l; i < n0 * sp; i += n0) s[i] = 0;
  __syncwarp(mask);
  const int pt = t.plane ? 1 : 0;
  const int64_t dcq = k.dc_q[seg][pt], acq = k.ac_q[seg][pt];
  uint32_t rows = 0;
  for (int i = l; i < t.n_coef; i += n0) {
    uint32_t w = k.coefs[t.coef_start + i];
    int pos = RV9_COEF_POS(w);
    int64_t dq = (int64_t)RV9_COEF_VAL(w) * (pos == 0 ? dcq : acq);
    if (n == 5) dq /= 2;
    dq = dq < INT32_MIN ? INT32_MIN : (dq > INT32_MAX ? INT32_MAX : dq);
    const int r = pos >> n, c = pos & (n0 - 1);
    s[r * sp + c] = (typename V::store_t)(int32_t)dq;
    rows |= 1u << r;
  }
  rows = __reduce_or_sync(mask, rows);
  __syncwarp(mask);
  const int row_kind = k.lossless ? 2 : ((t.tx_type == 0 || t.tx_type == 1) ? 0 : 1);
  const int col_kind = k.lossless ? 2 : ((t.tx_type == 0 || t.tx_type == 2) ? 0 : 1);
  if ((rows >> l) & 1) {
    V v[n0];
#pragma unroll
    for (int q = 0; q < n0; ++q) v[q] = V::load(s[l * sp + q]);
    tx1d<n>(v, row_kind, 2);
#pragma unroll
    for (int q = 0; q < n0; ++q) s[l * sp + q] = v[q].v;
  }
  __syncwarp(mask);
  V v[n0];
#pragma unroll
  for (int i = 0; i < n0; ++i) v[i] = V::load(s[i * sp + l]);
  tx1d<n>(v, col_kind, 0);
  constexpr int shift = (n + 2) < 6 ? (n + 2) : 6;
#pragma unroll
  for (int i = 0; i < n0; ++i) {
    V r = k.lossless ? v[i] : v[i].rshift(shift);
    T* px = dst + (size_t)i * dstride + l;
    *px = (T)clampi((int)*px + r.residual(), 0, maxv);
  }
}

// The inter residuals of all four transform sizes in one launch. The items
// are sorted by size; CTAs take them size by size (the first ctas[0] CTAs the
// 4x4 items, the next ctas[1] the 8x8 ones, and so on), so that the sizes run
// side by side instead of one launch after another.
struct ResSplit {
  int count[4];  // items per size
  int ctas[4];   // CTAs per size
};

// One CTA's share of the items of size n: CTA b of that size, items from
// `first` (the size's first item) on.
template <class T, class V, int n>
__device__ __forceinline__ void res_cta(const KFrame& k, int b, int first, int count, typename V::store_t* smem) {
  constexpr int n0 = 1 << n, G = 32 / n0, sp = n0 + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, grp = lane / n0, l = lane & (n0 - 1);
  const int i = (b * kResWarps + warp) * G + grp;
  if (i >= count) return;  // the whole group
  const unsigned mask = n0 == 32 ? 0xffffffffu : (((1u << n0) - 1u) << (grp * n0));
  const ResItem it = k.res[first + i];
  const rv9_tok& t = k.toks[it.tok];
  const rv9_block& bk = k.blocks[it.block];
  const PlanePtr& pp = k.cur[t.plane];
  T* dst = plane_ptr<T>(pp) + (size_t)t.y * pp.stride + t.x;
  residual_add_group<V, n, T>(k, t, bk.segment_id, dst, pp.stride, smem + (warp * G + grp) * (n0 * sp), l, mask);
}

template <class T, class V>
__device__ __forceinline__ void inter_res_cta(const KFrame& k, const ResSplit& sp, int b) {
  // Per warp 32 (n0 + 1) words at most (one 32x32 block, or G smaller ones).
  __shared__ typename V::store_t sc[kResWarps * 32 * 33];
  int first = 0;
  if (b < sp.ctas[0]) return res_cta<T, V, 2>(k, b, first, sp.count[0], sc);
  b -= sp.ctas[0];
  first += sp.count[0];
  if (b < sp.ctas[1]) return res_cta<T, V, 3>(k, b, first, sp.count[1], sc);
  b -= sp.ctas[1];
  first += sp.count[1];
  if (b < sp.ctas[2]) return res_cta<T, V, 4>(k, b, first, sp.count[2], sc);
  b -= sp.ctas[2];
  first += sp.count[2];
  res_cta<T, V, 5>(k, b, first, sp.count[3], sc);
}

template <class T, class V>
__global__ void __launch_bounds__(32 * kResWarps) k_inter_res(KFrame k, ResSplit sp) {
  inter_res_cta<T, V>(k, sp, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Intra wavefront.

constexpr int kIntraWarps = 4;

template <class V>
struct IntraSmem {
  typename V::store_t s[32 * 33];
  int32_t pred[32 * 32];
  int32_t above[66];
  int32_t left[32];
};

// One intra job of frame `k` by one warp: a row of a block's transform
// blocks of one plane, done in order, so that the links along the row cost
// no ticket and no wait on another warp. False when a wait gave up (this
// warp's or, through the frame's error word, another's).
template <class T, class V>
__device__ __forceinline__ bool intra_job(const KFrame& k, int job, IntraSmem<V>* sm, int lane) {
  const int maxv = (1 << k.bit_depth) - 1;
  volatile int32_t* err = k.error;
  {
    const int idx_end = (int)k.intra_jobs[job + 1];
    for (int idx = (int)k.intra_jobs[job]; idx < idx_end; ++idx) {
    const IntraItem it = k.intra[idx];
    const int plane = it.plane, log2 = it.tx_size + 2, size = 1 << log2;
    const int sx = plane ? k.ss_x : 0, sy = plane ? k.ss_y : 0;
    const int max_x = ((k.mi_cols * 8) >> sx) - 1, max_y = ((k.mi_rows * 8) >> sy) - 1;
    const bool have_left = it.flags & 1, have_above = it.flags & 2;
    const bool not_on_right = it.flags & 4;
    const int x = it.x, y = it.y;
    // The residual does not depend on the neighbours: its coefficients are
    // dequantised into shared memory (or its DC-only value taken) before
    // the wait, off the wavefront's critical path.
    bool dc_only = false;
    int dc_res = 0;
    uint32_t rows = 0;
    int tx_type = 0, res_tx = 0;
    if (it.tok != NO_TOK) {
      const rv9_tok t = k.toks[it.tok];
      const int seg = k.blocks[it.block].segment_id;
      tx_type = t.tx_type;
      res_tx = t.tx_size;
      if (t.eob == 1 && t.tx_type == 0 && !k.lossless) {
        dc_only = true;
        dc_res = dc_only_residual<V>(k, t, seg);
      } else {
        rows = load_coefs<V>(k, t, seg, sm->s, lane);
      }
    }
    // Wait for the cells the edges read: row y-1 and column x-1.
    {
      const uint8_t* cells = k.cells[plane];
      const int cs = k.cell_stride[plane];
      int ax1 = min(x + ((not_on_right && it.tx_size == 0) ? 2 * size : size) - 1, max_x);
      int ax0 = have_left ? x - 1 : x;
      int na = have_above ? ((ax1 >> 2) - (ax0 >> 2) + 1) : 0;
      int ly1 = min(y + size - 1, max_y);
      int nl = have_left ? ((ly1 >> 2) - (y >> 2) + 1) : 0;
      const volatile uint8_t* cell = nullptr;
      if (lane < na)
        cell = cells + (size_t)((y - 1) >> 2) * cs + (ax0 >> 2) + lane;
      else if (lane < na + nl)
        cell = cells + (size_t)((y >> 2) + lane - na) * cs + ((x - 1) >> 2);
      int polls = 0;
      for (;;) {
        bool pending = cell != nullptr && *cell != 0;
        if (!__any_sync(0xffffffffu, pending)) break;
        if (__any_sync(0xffffffffu, *err != 0)) return false;
        if (++polls > k.wait_limit) {
          if (lane == 0) atomicCAS(k.error, 0, 1);
          return false;
        }
        __nanosleep(64);
      }
      __threadfence();
    }
    // Edges (reference src/decoder/recon.rs:42-89).
    const T* buf = plane_ptr<const T>(k.cur[plane]);
    const int stride = k.cur[plane].stride;
    const int base = 1 << (k.bit_depth - 1);
    if (have_above) {
      const T* row = buf + (size_t)(y - 1) * stride;
      for (int i = lane; i < 2 * size; i += 32) {
        int v;
        if (i < size || (not_on_right && it.tx_size == 0))
          v = __ldcg(row + min(max_x, x + i));
        else
          v = __ldcg(row + min(max_x, x + size - 1));
        sm->above[1 + i] = v;
      }
      if (lane == 0) sm->above[0] = have_left ? (int)__ldcg(row + min(max_x, x - 1)) : base + 1;
    } else {
      for (int i = lane; i <= 2 * size; i += 32) sm->above[i] = base - 1;
    }
    for (int i = lane; i < size; i += 32)
      sm->left[i] = have_left ? (int)__ldcg(buf + (size_t)min(max_y, y + i) * stride + x - 1) : base + 1;
    __syncwarp();
    int32_t dc = 0;
    if (it.mode == 0) {
      int32_t sa = 0, sl = 0;
      for (int i = lane; i < size; i += 32) {
        sa += sm->above[1 + i];
        sl += sm->left[i];
      }
      sa = __reduce_add_sync(0xffffffffu, sa);
      sl = __reduce_add_sync(0xffffffffu, sl);
      dc = intra_dc(log2, sa, sl, have_left, have_above, k.bit_depth);
    }
    for (int i = lane; i < size * size; i += 32) {
      int r = i >> log2, c = i & (size - 1);
      sm->pred[i] = intra_pixel(it.mode, r, c, size, sm->above, sm->left, dc, maxv);
    }
    __syncwarp();
    if (it.tok != NO_TOK) {
      if (dc_only) {
        for (int i = lane; i < size * size; i += 32) sm->pred[i] = clampi(sm->pred[i] + dc_res, 0, maxv);
        __syncwarp();
      } else {
        itx_add_size<V, int32_t>(res_tx, sm->s, rows, tx_type, k.lossless, sm->pred, size, maxv, lane);
      }
    }
    T* dst = plane_ptr<T>(k.cur[plane]) + (size_t)y * stride + x;
    for (int i = lane; i < size * size; i += 32) {
      int r = i >> log2, c = i & (size - 1);
      dst[(size_t)r * stride + c] = (T)sm->pred[i];
    }
    __threadfence();
    __syncwarp();
    {
      uint8_t* cells = k.cells[plane];
      const int cs = k.cell_stride[plane];
      int nc = size >> 2;
      for (int i = lane; i < nc * nc; i += 32) {
        int cy = i / nc, cx = i - cy * nc;
        ((volatile uint8_t*)cells)[(size_t)((y >> 2) + cy) * cs + (x >> 2) + cx] = 0;
      }
    }
    __syncwarp();
    }
  }
  return true;
}

template <class T, class V>
__global__ void __launch_bounds__(32 * kIntraWarps) k_intra(KFrame k) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  IntraSmem<V>* sm = reinterpret_cast<IntraSmem<V>*>(smem_raw) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  for (;;) {
    // One job per ticket.
    int job = 0;
    if (lane == 0) job = atomicAdd(&k.counters[0], 1);
    job = __shfl_sync(0xffffffffu, job, 0) + (k.test_skip & 1);
    if (job >= k.n_intra_jobs) return;
    if (!intra_job<T, V>(k, job, sm, lane)) return;
  }
}

// ---------------------------------------------------------------------------
// Loop filter wavefront.

constexpr int kLfW = 80;   // tile row pitch (int16): 8 left + 64 + 8 of slack
constexpr int kLfH = 72;   // 8 above + 64

// Eight samples at a time between a plane (8-sample aligned) and the tile.
template <class T>
struct Chunk;
template <>
struct Chunk<uint8_t> {
  // The raw 8 samples, loaded ahead of the tile store.
  using Raw = uint2;
  static __device__ __forceinline__ Raw ldg(const uint8_t* g) { return __ldcg(reinterpret_cast<const uint2*>(g)); }
  static __device__ __forceinline__ void put(Raw v, int16_t* t) {
    int4 o;
    o.x = (int)(v.x & 0xff) | (int)((v.x >> 8) & 0xff) << 16;
    o.y = (int)((v.x >> 16) & 0xff) | (int)(v.x >> 24) << 16;
    o.z = (int)(v.y & 0xff) | (int)((v.y >> 8) & 0xff) << 16;
    o.w = (int)((v.y >> 16) & 0xff) | (int)(v.y >> 24) << 16;
    *reinterpret_cast<int4*>(t) = o;
  }
  static __device__ __forceinline__ void load(const uint8_t* g, int16_t* t) {
    uint2 v = __ldcg(reinterpret_cast<const uint2*>(g));
    int4 o;
    o.x = (int)(v.x & 0xff) | (int)((v.x >> 8) & 0xff) << 16;
    o.y = (int)((v.x >> 16) & 0xff) | (int)(v.x >> 24) << 16;
    o.z = (int)(v.y & 0xff) | (int)((v.y >> 8) & 0xff) << 16;
    o.w = (int)((v.y >> 16) & 0xff) | (int)(v.y >> 24) << 16;
    *reinterpret_cast<int4*>(t) = o;
  }
  // 8 samples held as ints (a line in registers) to global memory.
  static __device__ __forceinline__ void store_vals(uint8_t* g, const int* v) {
    uint2 o;
    o.x = (uint32_t)(v[0] & 0xff) | (uint32_t)(v[1] & 0xff) << 8 | (uint32_t)(v[2] & 0xff) << 16 |
          (uint32_t)(v[3] & 0xff) << 24;
    o.y = (uint32_t)(v[4] & 0xff) | (uint32_t)(v[5] & 0xff) << 8 | (uint32_t)(v[6] & 0xff) << 16 |
          (uint32_t)(v[7] & 0xff) << 24;
    __stcg(reinterpret_cast<uint2*>(g), o);
  }
  static __device__ __forceinline__ void store(uint8_t* g, const int16_t* t) {
    int4 o = *reinterpret_cast<const int4*>(t);
    uint2 v;
    v.x = (uint32_t)(o.x & 0xff) | (uint32_t)((o.x >> 16) & 0xff) << 8 | (uint32_t)(o.y & 0xff) << 16 |
          (uint32_t)((o.y >> 16) & 0xff) << 24;
    v.y = (uint32_t)(o.z & 0xff) | (uint32_t)((o.z >> 16) & 0xff) << 8 | (uint32_t)(o.w & 0xff) << 16 |
          (uint32_t)((o.w >> 16) & 0xff) << 24;
    __stcg(reinterpret_cast<uint2*>(g), v);
  }
};
template <>
struct Chunk<uint16_t> {
  using Raw = int4;
  static __device__ __forceinline__ Raw ldg(const uint16_t* g) { return __ldcg(reinterpret_cast<const int4*>(g)); }
  static __device__ __forceinline__ void put(Raw v, int16_t* t) { *reinterpret_cast<int4*>(t) = v; }
  static __device__ __forceinline__ void load(const uint16_t* g, int16_t* t) {
    *reinterpret_cast<int4*>(t) = __ldcg(reinterpret_cast<const int4*>(g));
  }
  static __device__ __forceinline__ void store_vals(uint16_t* g, const int* v) {
    int4 o;
    o.x = (v[0] & 0xffff) | (v[1] << 16);
    o.y = (v[2] & 0xffff) | (v[3] << 16);
    o.z = (v[4] & 0xffff) | (v[5] << 16);
    o.w = (v[6] & 0xffff) | (v[7] << 16);
    __stcg(reinterpret_cast<int4*>(g), o);
  }
  static __device__ __forceinline__ void store(uint16_t* g, const int16_t* t) {
    __stcg(reinterpret_cast<int4*>(g), *reinterpret_cast<const int4*>(t));
  }
};

// Vertical edges of one sample row (the row from 8 samples left of the
// superblock), left to right, with one 16-sample window in registers that
// rolls along the line: after edge e the window's first 4 samples are final
// (edge e + 1 starts 4 samples on), so they go back to shared memory and the
// next 4 come in. The loop body, and so lf_line, appears once in the kernel
// instead of once per edge, which keeps the loop filter's code within the
// instruction cache (unrolled per edge it measured 2 % slower). Samples past
// the 72 of the tile read as zero; only the last edges' p3..q3 reach them.
// The first edge is the last to touch the 8 samples left of the superblock
// (the next edge is a 4-wide one at offset 4, or none): right after it they
// go to `strip` (the previous superblock's last 8 columns, final for this
// row), when given, and with `publish` the warp then adds one step to its
// row's progress.
template <class T>
__device__ __forceinline__ void lf_row_rolled(int16_t* line, const LfEdge (*e)[16], int n_edges, int run, int bd,
                                              T* strip, uint32_t* publish) {
  int w[16];
#pragma unroll
  for (int q = 0; q < 16; q += 8) {
    int4 x = *reinterpret_cast<const int4*>(line + q);
    w[q] = (int16_t)(x.x & 0xffff); w[q + 1] = x.x >> 16;
    w[q + 2] = (int16_t)(x.y & 0xffff); w[q + 3] = x.y >> 16;
    w[q + 4] = (int16_t)(x.z & 0xffff); w[q + 5] = x.z >> 16;
    w[q + 6] = (int16_t)(x.w & 0xffff); w[q + 7] = x.w >> 16;
  }
#pragma unroll 1
  for (int ed = 0; ed < n_edges; ++ed) {
    const LfEdge f = e[ed][run];
    if (f.fs >= 0) lf_line(w, f.fs, f.limit, f.blimit, f.thresh, bd);
    if (ed == 0 && strip) {
      Chunk<T>::store_vals(strip, w);
      if (publish) {
        // Each lane's store before its fence; the warp's step after all.
        __threadfence();
        __syncwarp();
        if ((threadIdx.x & 31) == 0) atomicAdd(publish, 1u);
      }
    }
    int2 o;
    o.x = (w[0] & 0xffff) | (w[1] << 16);
    o.y = (w[2] & 0xffff) | (w[3] << 16);
    *reinterpret_cast<int2*>(line + 4 * ed) = o;
#pragma unroll
    for (int q = 0; q < 12; ++q) w[q] = w[q + 4];
    const int nxt = 4 * ed + 16;
    if (nxt + 4 <= 72) {
      const int2 x = *reinterpret_cast<const int2*>(line + nxt);
      w[12] = (int16_t)(x.x & 0xffff); w[13] = x.x >> 16;
      w[14] = (int16_t)(x.y & 0xffff); w[15] = x.y >> 16;
    } else {
      w[12] = w[13] = w[14] = w[15] = 0;
    }
  }
  // The window now holds the line's last 8 samples first.
  int4 o;
  o.x = (w[0] & 0xffff) | (w[1] << 16);
  o.y = (w[2] & 0xffff) | (w[3] << 16);
  o.z = (w[4] & 0xffff) | (w[5] << 16);
  o.w = (w[6] & 0xffff) | (w[7] << 16);
  *reinterpret_cast<int4*>(line + 4 * n_edges) = o;
}

// Horizontal edges of one sample column (from 8 rows above the superblock),
// top to bottom, with the same rolling window.
__device__ __forceinline__ void lf_col_rolled(int16_t* col, const LfEdge (*e)[16], int n_edges, int run, int bd) {
  int w[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) w[q] = col[q * kLfW];
#pragma unroll 1
  for (int ed = 0; ed < n_edges; ++ed) {
    const LfEdge f = e[ed][run];
    if (f.fs >= 0) lf_line(w, f.fs, f.limit, f.blimit, f.thresh, bd);
#pragma unroll
    for (int q = 0; q < 4; ++q) col[(4 * ed + q) * kLfW] = (int16_t)w[q];
#pragma unroll
    for (int q = 0; q < 12; ++q) w[q] = w[q + 4];
    const int nxt = 4 * ed + 16;
#pragma unroll
    for (int q = 0; q < 4; ++q) w[12 + q] = nxt + q < 72 ? col[(nxt + q) * kLfW] : 0;
  }
#pragma unroll
  for (int q = 0; q < 8; ++q) col[(4 * n_edges + q) * kLfW] = (int16_t)w[q];
}

// ---------------------------------------------------------------------------
// Loop filter, one CTA per superblock row.
//
// A CTA owns a superblock row and filters its superblocks left to right, as
// the reference does (vertical then horizontal edges per superblock,
// src/decoder/loopfilter.rs:466-620). The strip that superblock c's filters
// share with c+1 stays in shared memory, so the only wait is on the row
// above: superblock (r, c)'s horizontal pass reads the row above's bottom
// strip, final once that row has written superblock c back and filtered the
// first vertical edge of c+1 (the only one that reaches back into c, up to 7
// samples). Each row publishes its progress as (epoch << 16 | steps): per
// superblock one step when it is written back and one from each filter warp
// when the next superblock's first vertical edge has made its last 8 columns
// final, so superblock c of the row above is ready at kLfSteps (c + 1) steps.
//
// Warps 0-3 filter: vertical pass, top strip, horizontal pass. Warps 4-7
// do the rest off that chain: they stage the next superblock (its 8x8
// loop-filter records, edge decisions and 64x64 interior) into the other of
// two buffers, and write filtered samples back. The groups meet at named
// barriers: HDONE (filters -> stagers) and READY (stagers -> filters), each
// alternating between two barriers by superblock parity, since either group
// may run up to a superblock ahead of the other.


constexpr int kLfRowThreads = 256;
constexpr int kLfFilterThreads = 128;
constexpr int kLfStageThreads = kLfRowThreads - kLfFilterThreads;
constexpr int kBarFilter = 1, kBarStage = 2, kBarReady0 = 4, kBarHDone0 = 6;  // READY, HDONE: id + parity
// Progress steps per superblock: one from the stagers' write-back, one from
// each filter warp when the next superblock's first vertical edge has made
// its last 8 columns final.
constexpr int kLfSteps = 1 + kLfFilterThreads / 32;

struct LfRowSmem {
  int16_t px[2][3][kLfH][kLfW];
  LfEdge edges[2][2][2][16][16];  // [buffer][luma, chroma][pass][edge][run]
  uint32_t mi[2][64];
  uint8_t limit[64], blimit[64], thresh[64];
  int row;
  int frame;  // batched launches: the frame of `row`, -1 when none is left
  int abort_flag;
};

__device__ __forceinline__ void named_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}
__device__ __forceinline__ void named_arrive(int id, int count) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Stages superblock (sr, sc) into buffer `b`: records, edge decisions (the
// two chroma planes share theirs), interior. Run by `n` threads numbered
// `t`, synchronised by barrier `bar` (0: the whole CTA).
template <class T>
__device__ void lf_row_prepare(const KFrame& k, LfRowSmem& S, const LfParams& P, int sr, int sc, int b, int t, int n,
                               int bar) {
  for (int i = t; i < 64; i += n) {
    int mr = sr * 8 + (i >> 3), mc = sc * 8 + (i & 7);
    S.mi[b][i] = (mr < k.mi_rows && mc < k.mi_cols) ? k.lf_mi[(size_t)mr * k.mi_cols + mc] : 0u;
  }
  if (bar == 0)
    __syncthreads();
  else
    named_sync(bar, n);
  const LfMiTile at{S.mi[b], sr * 8, sc * 8};
  // Luma: 2 passes x 16 edges x 16 runs; chroma: its edges and runs only.
  const int ce0 = 16 >> k.ss_x, ce1 = 16 >> k.ss_y;  // chroma edges of pass 0 / 1 (runs: the other)
  const int n_luma = 512, n_c0 = ce0 * ce1, n_total = n_luma + 2 * n_c0;
  for (int i = t; i < n_total; i += n) {
    int plane, pass, ed, rn;
    if (i < n_luma) {
      plane = 0;
      pass = i >> 8;
      ed = (i >> 4) & 15;
      rn = i & 15;
    } else {
      int j = i - n_luma;
      plane = 1;
      pass = j >= n_c0;
      j -= pass * n_c0;
      const int ne = pass ? ce1 : ce0, nrun = pass ? ce0 : ce1;
      ed = j / nrun;
      rn = j - ed * nrun;
      (void)ne;
    }
    S.edges[b][plane][pass][ed][rn] = lf_edge_entry_at(P, at, plane, pass, sr * 8, sc * 8, ed, rn);
  }
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    const int sxp = p ? k.ss_x : 0, syp = p ? k.ss_y : 0;
    const int nc = (64 >> sxp) / 8, nr = 64 >> syp;
    const int x0 = (sc * 64) >> sxp, y0 = (sr * 64) >> syp;
    const T* src = plane_ptr<const T>(k.cur[p]);
    const int stride = k.cur[p].stride;
#pragma unroll 4
    for (int i = t; i < nr * nc; i += n) {
      int r = i / nc, c = i - r * nc;
      Chunk<T>::load(src + (size_t)(y0 + r) * stride + x0 + 8 * c, &S.px[b][p][8 + r][8 + 8 * c]);
    }
  }
}

// Filters superblock row `sr` of frame `k` (the whole CTA), the row's
// progress word already set to the epoch with no steps and S.abort_flag
// clear. False when a wait gave up (this row's, or another's through the
// frame's error word).
template <class T>
__device__ __forceinline__ bool lf_row(const KFrame& k, LfRowSmem& S, const int sr) {
  const int tid = threadIdx.x;
  const int bd = sizeof(T) == 1 ? 8 : k.bit_depth;  // a constant for 8-bit content
  const int cols = k.sb64_cols;
  const uint32_t ep = (uint32_t)(k.epoch & 0xffff) << 16;
  // (The previous row's last barrier orders these stores after its reads.)
  for (int i = tid; i < 64; i += kLfRowThreads) {
    S.limit[i] = k.lf_limit[i];
    S.blimit[i] = k.lf_blimit[i];
    S.thresh[i] = k.lf_thresh[i];
  }
  const LfParams P{k.mi_cols, k.mi_rows, k.ss_x, k.ss_y, nullptr, S.limit, S.blimit, S.thresh};
  int W[3], Hh[3];
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    W[p] = 64 >> (p ? k.ss_x : 0);
    Hh[p] = 64 >> (p ? k.ss_y : 0);
  }
  {
    uint32_t* const prog = k.sb_done + sr;
    lf_row_prepare<T>(k, S, P, sr, 0, 0, tid, kLfRowThreads, 0);
    __syncthreads();
    if (tid < kLfFilterThreads) {
      // ---- filters ----
      const int tf = tid;
      for (int sc = 0, cur = 0; sc < cols; ++sc, cur ^= 1) {
        if (sc > 0) named_sync(kBarReady0 + (sc & 1), kLfRowThreads);
        const bool live = !S.abort_flag;
        // The top strip (the row above's bottom 8 rows), loaded into
        // registers before the vertical pass when the row above is already
        // far enough; after the wait below otherwise.
        const int need = kLfSteps * (sc + 1);
        typename Chunk<T>::Raw top[2];
        bool top_early = false;
        const int top_total = 8 * (W[0] + W[1] + W[2]) / 8;
        auto top_addr = [&](int i) -> const T* {
          int p = i < W[0] ? 0 : (i < W[0] + W[1] ? 1 : 2);
          int j = i - (p == 0 ? 0 : (p == 1 ? W[0] : W[0] + W[1]));  // chunk within the plane's 8 rows
          const int nc = W[p] / 8, r = j / nc, c = j - r * nc;
          const int x0 = (sc * 64) >> (p ? k.ss_x : 0), y0 = (sr * 64) >> (p ? k.ss_y : 0);
          return plane_ptr<const T>(k.cur[p]) + (size_t)(y0 - 8 + r) * k.cur[p].stride + x0 + 8 * c;
        };
        auto top_tile = [&](int i) -> int16_t* {
          int p = i < W[0] ? 0 : (i < W[0] + W[1] ? 1 : 2);
          int j = i - (p == 0 ? 0 : (p == 1 ? W[0] : W[0] + W[1]));
          const int nc = W[p] / 8, r = j / nc, c = j - r * nc;
          return &S.px[cur][p][r][8 + 8 * c];
        };
        if (live && sr > 0) {
          uint32_t v;
          asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(k.sb_done + (sr - 1)) : "memory");
          if ((v & 0xffff0000u) == ep && (int)(v & 0xffffu) >= need) {
            top_early = true;
#pragma unroll
            for (int q = 0; q < 2; ++q)
              if (tf + q * kLfFilterThreads < top_total) top[q] = Chunk<T>::ldg(top_addr(tf + q * kLfFilterThreads));
          }
        }
        if (live) {
          // Vertical edges, one thread per sample row. Superblock c-1's last
          // 8 columns are final for a row once its first edge is filtered:
          // they go out then, and each warp publishes a progress step after
          // its last row's (the row below waits for their bottom 8 rows).
          const int total = Hh[0] + Hh[1] + Hh[2];
          for (int task = tf; task < total; task += kLfFilterThreads) {
            int p = task < Hh[0] ? 0 : (task < Hh[0] + Hh[1] ? 1 : 2);
            int r = task - (p == 0 ? 0 : (p == 1 ? Hh[0] : Hh[0] + Hh[1]));
            T* strip = nullptr;
            uint32_t* pub = nullptr;
            if (sc > 0) {
              const int x0 = (sc * 64) >> (p ? k.ss_x : 0), y0 = (sr * 64) >> (p ? k.ss_y : 0);
              strip = plane_ptr<T>(k.cur[p]) + (size_t)(y0 + r) * k.cur[p].stride + x0 - 8;
              if (task + kLfFilterThreads >= total) pub = prog;
            }
            lf_row_rolled<T>(&S.px[cur][p][8 + r][0], S.edges[cur][p ? 1 : 0][0], 16 >> (p ? k.ss_x : 0), r >> 2, bd,
                           strip, pub);
          }
        }
        named_sync(kBarFilter, kLfFilterThreads);
        // Wait for the row above: superblock c's bottom strip final there
        // (already seen, by an acquiring load, when the strip came early).
        if (live && sr > 0 && tf == 0 && !top_early) {
          const volatile uint32_t* above = k.sb_done + (sr - 1);
          int polls = 0;
          for (;;) {
            uint32_t v = *above;
            if ((v & 0xffff0000u) == ep && (int)(v & 0xffffu) >= need) break;
            if (*(volatile int32_t*)k.error || ++polls > k.wait_limit) {
              atomicCAS(k.error, 0, 2);
              S.abort_flag = 1;
              break;
            }
            if (polls > 32) __nanosleep(32);
          }
          __threadfence();
        }
        named_sync(kBarFilter, kLfFilterThreads);
        if (!S.abort_flag) {
          if (sr > 0) {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
              const int i = tf + q * kLfFilterThreads;
              if (i < top_total) Chunk<T>::put(top_early ? top[q] : Chunk<T>::ldg(top_addr(i)), top_tile(i));
            }
            named_sync(kBarFilter, kLfFilterThreads);
          }
          // Horizontal edges, one thread per sample column.
          const int total = W[0] + W[1] + W[2];
          for (int task = tf; task < total; task += kLfFilterThreads) {
            int p = task < W[0] ? 0 : (task < W[0] + W[1] ? 1 : 2);
            int c = task - (p == 0 ? 0 : (p == 1 ? W[0] : W[0] + W[1]));
            lf_col_rolled(&S.px[cur][p][0][8 + c], S.edges[cur][p ? 1 : 0][1], 16 >> (p ? k.ss_y : 0), c >> 2, bd);
          }
          named_sync(kBarFilter, kLfFilterThreads);
          // This superblock's right strip becomes the next one's left strip.
          if (sc + 1 < cols) {
            const int nxt = cur ^ 1;
            const int total_r = Hh[0] + Hh[1] + Hh[2];
            for (int task = tf; task < total_r; task += kLfFilterThreads) {
              int p = task < Hh[0] ? 0 : (task < Hh[0] + Hh[1] ? 1 : 2);
              int r = task - (p == 0 ? 0 : (p == 1 ? Hh[0] : Hh[0] + Hh[1]));
              *reinterpret_cast<int4*>(&S.px[nxt][p][8 + r][0]) =
                  *reinterpret_cast<const int4*>(&S.px[cur][p][8 + r][W[p]]);
            }
          }
        }
        named_arrive(kBarHDone0 + (sc & 1), kLfRowThreads);
      }
    } else {
      // ---- stagers ----
      const int ts = tid - kLfFilterThreads;
      if (cols > 1) {
        lf_row_prepare<T>(k, S, P, sr, 1, 1, ts, kLfStageThreads, kBarStage);
        named_arrive(kBarReady0 + 1, kLfRowThreads);
      }
      for (int sc = 0, cur = 0; sc < cols; ++sc, cur ^= 1) {
        named_sync(kBarHDone0 + (sc & 1), kLfRowThreads);
        const bool last = sc + 1 == cols;
        // Write-back of the top strip and the superblock but its last 8
        // columns (the next superblock's first vertical edge still reaches
        // them), or with them at the row's end; tile rows [lo, hi) of each
        // plane (tile row 8 is the superblock's first).
        auto write_back = [&](bool bottom) {
#pragma unroll
          for (int p = 0; p < 3; ++p) {
            T* dst = plane_ptr<T>(k.cur[p]);
            const int stride = k.cur[p].stride;
            const int x0 = (sc * 64) >> (p ? k.ss_x : 0), y0 = (sr * 64) >> (p ? k.ss_y : 0);
            const int lnc = (p && k.ss_x) ? 2 : 3, nc = 1 << lnc;
            const int lo = bottom ? Hh[p] : (sr > 0 ? 0 : 8), hi = bottom ? Hh[p] + 8 : Hh[p];
            for (int i = ts; i < (hi - lo) * nc; i += kLfStageThreads) {
              int r = lo + (i >> lnc), c = i & (nc - 1);
              if (r >= 8 && c == nc - 1 && !last) continue;
              Chunk<T>::store(dst + (size_t)(y0 - 8 + r) * stride + x0 + 8 * c, &S.px[cur][p][r][8 + 8 * c]);
            }
          }
        };
        // The bottom 8 rows first, the only ones the row below reads: one
        // step of the row's progress as soon as they are out (all kLfSteps
        // at the row's end, whose last strip goes out here). The filter
        // warps add the others when they write the superblock's last 8
        // columns, final after the next superblock's first vertical edge.
        if (!S.abort_flag) write_back(true);
        named_sync(kBarStage, kLfStageThreads);
        if (ts == 0) {
          __threadfence();
          atomicAdd(prog, last ? (uint32_t)kLfSteps : 1u);
        }
        // Then the rest, none of which the row below touches. (The filters
        // own columns 0-7 of a buffer: they overwrite them with the next
        // left strip while this group may still be writing the buffer back.)
        if (!S.abort_flag) write_back(false);
        named_sync(kBarStage, kLfStageThreads);
        // Stage superblock c+2 into this superblock's buffer, now written back.
        if (sc + 2 < cols) {
          lf_row_prepare<T>(k, S, P, sr, sc + 2, cur, ts, kLfStageThreads, kBarStage);
          named_arrive(kBarReady0 + ((sc + 2) & 1), kLfRowThreads);
        }
      }
    }
    __syncthreads();
  }
  return !S.abort_flag;
}

// This row's progress: kLfSteps per superblock, from 0 (thread 0, when it
// takes row r of frame k).
__device__ __forceinline__ void lf_row_start(const KFrame& k, LfRowSmem& S, int r) {
  S.row = r;
  S.abort_flag = 0;
  if (r < k.sb64_rows) *(volatile uint32_t*)&k.sb_done[r] = (uint32_t)(k.epoch & 0xffff) << 16;
}

template <class T>
__global__ void __launch_bounds__(kLfRowThreads) k_lf_rows(KFrame k) {
  extern __shared__ __align__(16) unsigned char lf_raw[];
  LfRowSmem& S = *reinterpret_cast<LfRowSmem*>(lf_raw);
  for (;;) {
    if (threadIdx.x == 0) lf_row_start(k, S, atomicAdd(&k.counters[1], 1) + ((k.test_skip >> 1) & 1));
    __syncthreads();
    const int sr = S.row;
    if (sr >= k.sb64_rows) return;
    if (!lf_row<T>(k, S, sr)) return;
  }
}

// ---------------------------------------------------------------------------
// Batched stages: one launch per stage for the next frames of many streams,
// frames that do not depend on one another. The CTAs of a data-parallel stage
// are split among the frames by a prefix of their per-frame grids. The two
// wavefront stages hand out each frame's jobs (intra rows of transform
// blocks, loop-filter superblock rows) from that frame's own tickets, in the
// frame's order: a warp (a CTA for the loop filter) takes them from its home
// frame and moves on to the next frame with tickets left when those are
// gone. A job waits only for jobs of its own frame with earlier tickets,
// all held by warps already running, so every wait ends. A job of a frame
// whose wait gave up is abandoned quickly (the frame's error word is set)
// and the warp goes on with the other frames.

struct BatchArgs {
  const KFrame* frames;
  const PrepSplit* prep;
  const ResSplit* res;
  // [6][n + 1] prefixes over the frames: the CTAs of the preparation, small
  // inter, large inter and residual launches, then the intra jobs and the
  // loop-filter rows (which place the wavefront stages' home frames).
  const uint32_t* base;
  int n;
};
enum { kBasePrep = 0, kBaseSmall, kBaseLarge, kBaseRes, kBaseIntraJobs, kBaseLfRows, kBases };


// The frame whose CTA range holds CTA b: the last f with base[f] <= b.
__device__ __forceinline__ int batch_frame(const uint32_t* base, int n, uint32_t b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (base[mid] <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// The home frame of worker w of `workers`: workers are spread over the
// frames in proportion to their share of the work prefix `base`.
__device__ __forceinline__ int batch_home(const uint32_t* base, int n, uint32_t w, uint32_t workers) {
  return batch_frame(base, n, (uint32_t)(((uint64_t)w * base[n]) / workers));
}

// Warp-collective: a ticket of counter `which` (0 intra jobs, 1 loop-filter
// rows) from the first frame at or after `home` (cyclically) that has any
// left; returns that frame, or -1 when no frame has any.
__device__ __forceinline__ int batch_take(const BatchArgs& a, int home, int which, int* ticket) {
  const int lane = threadIdx.x & 31;
  for (int s = 0; s < a.n; s += 32) {
    int f = home + s + lane;
    if (f >= a.n) f -= a.n;
    const bool mine = s + lane < a.n;
    int limit = 0;
    if (mine) {
      const KFrame& k = a.frames[f];
      limit = which ? (k.lf_on ? k.sb64_rows : 0) : k.n_intra_jobs;
    }
    for (;;) {
      const bool left = mine && *(volatile int32_t*)&a.frames[f].counters[which] < limit;
      const unsigned m = __ballot_sync(0xffffffffu, left);
      if (!m) break;  // none among these 32 frames
      const int src = __ffs(m) - 1;
      int t = 0;
      if (lane == src) t = atomicAdd(&a.frames[f].counters[which], 1);
      t = __shfl_sync(0xffffffffu, t, src);
      const int lim = __shfl_sync(0xffffffffu, limit, src);
      const int fr = __shfl_sync(0xffffffffu, f, src);
      if (t < lim) {
        *ticket = t;
        return fr;
      }
      // Another warp took that frame's last ticket first: look again.
    }
  }
  return -1;
}

template <class T>
__global__ void __launch_bounds__(kPrepThreads) k_prep_batch(BatchArgs a) {
  // The frames' wavefront tickets start at zero; the later stages take them.
  if (blockIdx.x == 0)
    for (int f = threadIdx.x; f < a.n; f += kPrepThreads) {
      a.frames[f].counters[0] = 0;
      a.frames[f].counters[1] = 0;
    }
  const uint32_t* base = a.base + kBasePrep * (a.n + 1);
  if (blockIdx.x >= base[a.n]) return;
  const int f = batch_frame(base, a.n, blockIdx.x);
  prep_cta<T>(a.frames[f], a.prep[f], blockIdx.x - base[f]);
}

template <class T>
__global__ void __launch_bounds__(kInterThreads) k_inter_small_batch(BatchArgs a) {
  const uint32_t* base = a.base + kBaseSmall * (a.n + 1);
  const int f = batch_frame(base, a.n, blockIdx.x);
  inter_small_cta<T>(a.frames[f], blockIdx.x - base[f]);
}

template <class T>
__global__ void __launch_bounds__(kInterThreads) k_inter_batch(BatchArgs a) {
  const uint32_t* base = a.base + kBaseLarge * (a.n + 1);
  const int f = batch_frame(base, a.n, blockIdx.x);
  inter_large_cta<T, kInterThreads>(a.frames[f], blockIdx.x - base[f]);
}

template <class T, class V>
__global__ void __launch_bounds__(32 * kResWarps) k_inter_res_batch(BatchArgs a) {
  const uint32_t* base = a.base + kBaseRes * (a.n + 1);
  const int f = batch_frame(base, a.n, blockIdx.x);
  inter_res_cta<T, V>(a.frames[f], a.res[f], blockIdx.x - base[f]);
}

template <class T, class V>
__global__ void __launch_bounds__(32 * kIntraWarps) k_intra_batch(BatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  IntraSmem<V>* sm = reinterpret_cast<IntraSmem<V>*>(smem_raw) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const int home = batch_home(a.base + kBaseIntraJobs * (a.n + 1), a.n, blockIdx.x * kIntraWarps + (threadIdx.x >> 5),
                              gridDim.x * kIntraWarps);
  for (;;) {
    int job = 0;
    const int f = batch_take(a, home, 0, &job);
    if (f < 0) return;
    job += a.frames[f].test_skip & 1;
    if (job < a.frames[f].n_intra_jobs) intra_job<T, V>(a.frames[f], job, sm, lane);
  }
}

template <class T>
__global__ void __launch_bounds__(kLfRowThreads) k_lf_rows_batch(BatchArgs a) {
  extern __shared__ __align__(16) unsigned char lf_raw[];
  LfRowSmem& S = *reinterpret_cast<LfRowSmem*>(lf_raw);
  const int home = batch_home(a.base + kBaseLfRows * (a.n + 1), a.n, blockIdx.x, gridDim.x);
  for (;;) {
    if (threadIdx.x < 32) {
      int r = 0;
      const int f = batch_take(a, home, 1, &r);
      if (threadIdx.x == 0) {
        S.frame = f;
        if (f >= 0) lf_row_start(a.frames[f], S, r + ((a.frames[f].test_skip >> 1) & 1));
      }
    }
    __syncthreads();
    const int f = S.frame, sr = S.row;
    if (f < 0) return;
    if (sr < a.frames[f].sb64_rows)
      lf_row<T>(a.frames[f], S, sr);
    else
      __syncthreads();  // (a skipped row: S is rewritten only after every thread has read it)
  }
}

// ---------------------------------------------------------------------------
// Host-side launch of one frame's chain.

cudaError_t upload_filters(const int16_t* f) { return cudaMemcpyToSymbol(c_filters, f, sizeof(int16_t) * 4 * 16 * 8); }

// Kernel attributes are per device: the shared-memory opt-ins of the intra
// and loop-filter kernels (above the 48 KB default) are set on each device
// an engine starts on, and the batched launches' grids come from that
// device's occupancy.
constexpr int kMaxDevices = 64;
static DeviceKernels g_devices[kMaxDevices];
static std::mutex g_devices_mu;

const DeviceKernels& device_kernels(int device) {
  static const DeviceKernels none;
  return device >= 0 && device < kMaxDevices ? g_devices[device] : none;
}

template <class T, class V>
static cudaError_t init_device_t(DeviceKernels* d) {
  const int i = sizeof(T) - 1;
  const int intra_smem = (int)(sizeof(IntraSmem<V>) * kIntraWarps), lf_smem = (int)sizeof(LfRowSmem);
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_intra<T, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, intra_smem)) ||
      (e = cudaFuncSetAttribute(k_intra_batch<T, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, intra_smem)) ||
      (e = cudaFuncSetAttribute(k_lf_rows<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, lf_smem)) ||
      (e = cudaFuncSetAttribute(k_lf_rows_batch<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, lf_smem)))
    return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d->intra_batch_per_sm[i], k_intra_batch<T, V>,
                                                         32 * kIntraWarps, intra_smem)) ||
      (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d->lf_batch_per_sm[i], k_lf_rows_batch<T>, kLfRowThreads,
                                                         lf_smem)))
    return e;
  d->intra_batch_per_sm[i] = std::max(d->intra_batch_per_sm[i], 1);
  d->lf_batch_per_sm[i] = std::max(d->lf_batch_per_sm[i], 1);
  return cudaSuccess;
}

cudaError_t kernels_init_device(int device) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_devices_mu);
  DeviceKernels& d = g_devices[device];
  if (d.ready.load(std::memory_order_acquire)) return cudaSuccess;
  int cur = -1;
  cudaError_t e = cudaGetDevice(&cur);
  if (e != cudaSuccess) return e;
  if (cur != device) return cudaErrorInvalidDevice;  // the caller makes `device` current
  if ((e = init_device_t<uint8_t, L32>(&d)) != cudaSuccess || (e = init_device_t<uint16_t, L64>(&d)) != cudaSuccess)
    return e;
  d.ready.store(true, std::memory_order_release);
  return cudaSuccess;
}

// The preparation launch's parts for a frame of n_blocks blocks.
static PrepSplit prep_split(const KFrame& k, int n_blocks) {
  const int aw = k.sb64_cols * 64, ah = k.sb64_rows * 64;
  PrepSplit ps;
  ps.zp_per_plane = 64;
  ps.zp = (k.mi_cols * 8 < aw || k.mi_rows * 8 < ah) ? 3 * ps.zp_per_plane : 0;
  ps.n_blocks = (k.lf_on && n_blocks > 0) ? n_blocks : 0;
  ps.lf = (ps.n_blocks + kPrepThreads - 1) / kPrepThreads;
  ps.mark = (k.n_intra + kPrepThreads - 1) / kPrepThreads;
  return ps;
}

// The residual launch's CTAs per transform size; *grid receives their sum.
static ResSplit res_split(const KFrame& k, int* grid) {
  ResSplit rs;
  *grid = 0;
  for (int z = 0; z < 4; ++z) {
    const int per_cta = kResWarps * (32 >> (z + 2));
    rs.count[z] = (int)k.n_res_by_size[z];
    rs.ctas[z] = (rs.count[z] + per_cta - 1) / per_cta;
    *grid += rs.ctas[z];
  }
  return rs;
}

// The batch tables in one buffer: the frames' KFrames, their launch splits
// and the four CTA prefixes, each at a 16-byte boundary.
struct BatchLayout {
  size_t o_frames, o_prep, o_res, o_base, bytes;
};
static BatchLayout batch_layout(int n) {
  auto up = [](size_t v) { return (v + 15) & ~(size_t)15; };
  BatchLayout l;
  l.o_frames = 0;
  l.o_prep = up(l.o_frames + sizeof(KFrame) * n);
  l.o_res = up(l.o_prep + sizeof(PrepSplit) * n);
  l.o_base = up(l.o_res + sizeof(ResSplit) * n);
  l.bytes = up(l.o_base + sizeof(uint32_t) * kBases * (n + 1));
  return l;
}

size_t batch_table_bytes(int n) { return batch_layout(n).bytes; }

void batch_fill(const KFrame* ks, const int* n_blocks, int n, uint8_t* host, BatchTotals* tot, int n_sm,
                const TuneParams& tune) {
  const uint32_t intra_cap = (uint32_t)((n_sm * tune.intra_ctas_per_sm_x4 + 3) / 4);
  const BatchLayout l = batch_layout(n);
  KFrame* fr = reinterpret_cast<KFrame*>(host + l.o_frames);
  PrepSplit* pp = reinterpret_cast<PrepSplit*>(host + l.o_prep);
  ResSplit* rr = reinterpret_cast<ResSplit*>(host + l.o_res);
  uint32_t* base = reinterpret_cast<uint32_t*>(host + l.o_base);
  memset(tot, 0, sizeof *tot);
  for (int f = 0; f < n; ++f) {
    const KFrame& k = ks[f];
    fr[f] = k;
    pp[f] = prep_split(k, n_blocks[f]);
    int res_grid = 0;
    rr[f] = res_split(k, &res_grid);
    const uint32_t grids[4] = {(uint32_t)(pp[f].zp + pp[f].lf + pp[f].mark),
                               (uint32_t)((k.n_units_small + kInterThreads / 32 - 1) / (kInterThreads / 32)),
                               (uint32_t)(k.n_units - k.n_units_small), (uint32_t)res_grid};
    for (int st = 0; st < 4; ++st) {
      base[st * (n + 1) + f] = tot->ctas[st];
      tot->ctas[st] += grids[st];
    }
    base[kBaseIntraJobs * (n + 1) + f] = tot->intra_jobs;
    base[kBaseLfRows * (n + 1) + f] = tot->lf_rows;
    tot->intra_jobs += (uint32_t)k.n_intra_jobs;
    tot->intra_ctas += std::min<uint32_t>(((uint32_t)k.n_intra_jobs + kIntraWarps - 1) / kIntraWarps, intra_cap);
    tot->lf_rows += k.lf_on ? (uint32_t)k.sb64_rows : 0;
  }
  for (int st = 0; st < 4; ++st) base[st * (n + 1) + n] = tot->ctas[st];
  base[kBaseIntraJobs * (n + 1) + n] = tot->intra_jobs;
  base[kBaseLfRows * (n + 1) + n] = tot->lf_rows;
}

template <class T, class V>
static cudaError_t launch_batch_t(const uint8_t* tables, int n, const BatchTotals& tot, cudaStream_t s, int n_sm,
                                  const TuneParams& tune, int* launches) {
  const BatchLayout l = batch_layout(n);
  BatchArgs a;
  a.frames = reinterpret_cast<const KFrame*>(tables + l.o_frames);
  a.prep = reinterpret_cast<const PrepSplit*>(tables + l.o_prep);
  a.res = reinterpret_cast<const ResSplit*>(tables + l.o_res);
  a.base = reinterpret_cast<const uint32_t*>(tables + l.o_base);
  a.n = n;
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return e;
  const DeviceKernels& dev = device_kernels(device);
  if (!dev.ready.load(std::memory_order_acquire)) return cudaErrorInitializationError;
  int L = 0;
  // The preparation launch always runs: its first CTA clears the tickets.
  k_prep_batch<T><<<tot.ctas[kBasePrep] ? tot.ctas[kBasePrep] : 1, kPrepThreads, 0, s>>>(a);
  ++L;
  if (tot.ctas[kBaseSmall]) {
    k_inter_small_batch<T><<<tot.ctas[kBaseSmall], kInterThreads, 0, s>>>(a);
    ++L;
  }
  if (tot.ctas[kBaseLarge]) {
    k_inter_batch<T><<<tot.ctas[kBaseLarge], kInterThreads, 0, s>>>(a);
    ++L;
  }
  if (tot.ctas[kBaseRes]) {
    k_inter_res_batch<T, V><<<tot.ctas[kBaseRes], 32 * kResWarps, 0, s>>>(a);
    ++L;
  }
  if (tot.intra_jobs) {
    // As many CTAs as the frames would take on their own streams (a wide
    // keyframe wavefront needs its warps whatever else is in the batch), up
    // to what fits on the device at once.
    const size_t smem = sizeof(IntraSmem<V>) * kIntraWarps;
    const int per_sm = dev.intra_batch_per_sm[sizeof(T) - 1];
    const int grid = (int)std::min<uint32_t>(tot.intra_ctas, (uint32_t)(n_sm * per_sm));
    k_intra_batch<T, V><<<grid > 0 ? grid : 1, 32 * kIntraWarps, smem, s>>>(a);
    ++L;
  }
  if (tot.lf_rows) {
    // As many row CTAs as fit on the device at once (more would only wait).
    const int cap = n_sm * dev.lf_batch_per_sm[sizeof(T) - 1];
    k_lf_rows_batch<T><<<(int)tot.lf_rows < cap ? (int)tot.lf_rows : cap, kLfRowThreads, sizeof(LfRowSmem), s>>>(a);
    ++L;
  }
  *launches += L;
  return cudaGetLastError();
}

cudaError_t launch_batch(const uint8_t* dev, int n, const BatchTotals& tot, bool high, cudaStream_t s, int n_sm,
                         const TuneParams& tune, int* launches) {
  if (high) return launch_batch_t<uint16_t, L64>(dev, n, tot, s, n_sm, tune, launches);
  return launch_batch_t<uint8_t, L32>(dev, n, tot, s, n_sm, tune, launches);
}

template <class T, class V>
static cudaError_t launch_frame_t(const KFrame& k, int n_blocks, cudaStream_t s, int n_sm, int* launches,
                                  LaunchHook hook, void* hctx, const TuneParams& tune, const LaunchAux* aux) {
  int L = 0;
  auto mark = [&](int id, int phase) {
    if (hook) hook(hctx, id, phase);
  };
  {
    const PrepSplit ps = prep_split(k, n_blocks);
    const int grid = ps.zp + ps.lf + ps.mark;
    if (grid > 0) {
      mark(K_PREP, 0);
      k_prep<T><<<grid, kPrepThreads, 0, s>>>(k, ps);
      mark(K_PREP, 1);
      ++L;
    }
  }
  if (k.n_units > 0) {
    mark(K_INTER, 0);
    // The two inter kernels write disjoint regions: with a side stream, the
    // small regions run there beside the large ones (fork and join events on
    // the frame's stream keep the chain's order around them).
    const bool small = k.n_units_small > 0, large = k.n_units > k.n_units_small;
    const bool fork = small && large && aux && aux->side && tune.inter_fork;
    cudaError_t e;
    if (fork) {
      if ((e = cudaEventRecord(aux->fork, s)) != cudaSuccess) return e;
      if ((e = cudaStreamWaitEvent(aux->side, aux->fork, 0)) != cudaSuccess) return e;
    }
    if (small) {
      cudaStream_t ss = fork ? aux->side : s;
      k_inter_small<T><<<(k.n_units_small + kInterThreads / 32 - 1) / (kInterThreads / 32), kInterThreads, 0, ss>>>(k);
      ++L;
    }
    if (fork && (e = cudaEventRecord(aux->join, aux->side)) != cudaSuccess) return e;
    if (large) {
      const int nl = k.n_units - k.n_units_small;
      if (tune.inter_threads == 64)
        k_inter<T, 64><<<nl, 64, 0, s>>>(k);
      else if (tune.inter_threads == 256)
        k_inter<T, 256><<<nl, 256, 0, s>>>(k);
      else
        k_inter<T, 128><<<nl, 128, 0, s>>>(k);
      ++L;
    }
    if (fork && (e = cudaStreamWaitEvent(s, aux->join, 0)) != cudaSuccess) return e;
    mark(K_INTER, 1);
  }
  if (k.n_res > 0) {
    mark(K_INTER_RES, 0);
    int grid = 0;
    const ResSplit rs = res_split(k, &grid);
    k_inter_res<T, V><<<grid, 32 * kResWarps, 0, s>>>(k, rs);
    ++L;
    mark(K_INTER_RES, 1);
  }
  if (k.n_intra > 0) {
    size_t smem = sizeof(IntraSmem<V>) * kIntraWarps;
    // One CTA per SM at most: a warp per job of the wavefront's width (a
    // diagonal of superblocks, a few rows of transform blocks each) with
    // room to spare; more warps would only poll further ahead, taking issue
    // slots and L2 bandwidth from the warps on the chain and from other
    // streams' kernels.
    int want = (k.n_intra_jobs + kIntraWarps - 1) / kIntraWarps;
    int cap = (n_sm * tune.intra_ctas_per_sm_x4 + 3) / 4;
    int grid = want < cap ? want : cap;
    mark(K_INTRA, 0);
    k_intra<T, V><<<grid, 32 * kIntraWarps, smem, s>>>(k);
    mark(K_INTRA, 1);
    ++L;
  }
  if (k.lf_on) {
    // One CTA per superblock row (rows are taken in order from a ticket).
    int grid = k.sb64_rows < n_sm ? k.sb64_rows : n_sm;
    mark(K_LF, 0);
    k_lf_rows<T><<<grid, kLfRowThreads, sizeof(LfRowSmem), s>>>(k);
    mark(K_LF, 1);
    ++L;
  }
  *launches += L;
  return cudaGetLastError();
}

cudaError_t launch_frame(const KFrame& k, int n_blocks, cudaStream_t s, int n_sm, int* launches, LaunchHook hook,
                         void* hook_ctx, const TuneParams& tune, const LaunchAux* aux) {
  if (k.bit_depth > 8)
    return launch_frame_t<uint16_t, L64>(k, n_blocks, s, n_sm, launches, hook, hook_ctx, tune, aux);
  return launch_frame_t<uint8_t, L32>(k, n_blocks, s, n_sm, launches, hook, hook_ctx, tune, aux);
}

// ---------------------------------------------------------------------------
// On-device MD5 of shown frames: the digest of the packed planes (the bytes
// of the reference's Frame::packed()) computed from the frame's strided
// device planes, one warp per frame. MD5 is a chain of 64-byte blocks, so a
// frame's lanes gather the next 32 blocks of the byte stream (data, then the
// RFC 1321 padding) into shared memory together, and lane 0 runs the
// compression over them.

__constant__ uint32_t c_md5_t[64];

cudaError_t upload_md5_table() {
  uint32_t t[64];
  md5_sine_table(t);
  return cudaMemcpyToSymbol(c_md5_t, t, sizeof t);
}

constexpr int kMd5Lanes = 32;

__global__ void __launch_bounds__(kMd5Lanes) k_md5_frames(Md5Jobs jobs) {
  __shared__ uint32_t words[kMd5Lanes * 16];
  const Md5Job& j = jobs.job[blockIdx.x];
  const int lane = threadIdx.x;
  uint64_t plane_len[3], len = 0;
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    plane_len[p] = (uint64_t)j.row_bytes[p] * j.rows[p];
    len += plane_len[p];
  }
  const uint64_t total = md5_padded_bytes(len);
  Md5State h;
  md5_init(&h);
  for (uint64_t pos = 0; pos < total; pos += 64 * kMd5Lanes) {
    const uint64_t k0 = pos + 64 * (uint64_t)lane;
    if (k0 < total) {
      // The byte stream's cursor at k0: plane, row, column.
      int p = 0;
      uint64_t r = k0;
      while (p < 2 && r >= plane_len[p]) r -= plane_len[p++];
      uint32_t row = 0, col = 0;
      if (k0 < len) {
        row = (uint32_t)(r / j.row_bytes[p]);
        col = (uint32_t)(r - (uint64_t)row * j.row_bytes[p]);
      }
      for (int q = 0; q < 16; ++q) {
        uint32_t w = 0;
        for (int b = 0; b < 4; ++b) {
          const uint64_t k = k0 + 4 * q + b;
          uint32_t v;
          if (k < len) {
            v = __ldg(j.plane[p] + (uint64_t)row * j.stride[p] + col);
            if (++col == j.row_bytes[p]) {
              col = 0;
              if (++row == j.rows[p] && p < 2) {
                row = 0;
                ++p;
              }
            }
          } else {
            v = md5_pad_byte(k, len);
          }
          w |= v << (8 * b);
        }
        words[lane * 16 + q] = w;
      }
    }
    __syncwarp();
    if (lane == 0) {
      const uint64_t left = (total - pos) / 64;
      const int nb = left < (uint64_t)kMd5Lanes ? (int)left : kMd5Lanes;
      for (int b = 0; b < nb; ++b) md5_block(&h, &words[b * 16], c_md5_t);
    }
    __syncwarp();
  }
  if (lane == 0) md5_digest(h, j.out);
}

cudaError_t launch_md5(const Md5Jobs& jobs, int n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_md5_frames<<<n, kMd5Lanes, 0, s>>>(jobs);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Fixed wavefront scratch, for callers that must not allocate device memory.
//
// The loop-filter and intra wavefront kernels take their scratch (tickets,
// error word, superblock done flags, per-8x8 loop-filter records) through
// KFrame pointers; Engine::sequence_run_fixed points them into this array
// instead of the engine's allocations. The array is zero at module load.
// Every caller on a device shares it, so calls that overlap on one device
// (two decoders, two host threads) race on it.
static __device__ __align__(256) uint8_t g_fixed_scratch[kFixedScratchBytes];

cudaError_t fixed_scratch_address(int device, void** ptr) {
  // Resolved once per device, with that device current, and kept for the
  // life of the process: the address belongs to the device's primary
  // context, so a host application that destroys that context
  // (cudaDeviceReset) must not call the no-allocation entry point again in
  // this process.
  static std::mutex mu;
  static void* addr[kMaxDevices] = {nullptr};
  *ptr = nullptr;
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[device]) {
    void* p = nullptr;
    cudaError_t rc = cudaGetSymbolAddress(&p, g_fixed_scratch);
    if (rc != cudaSuccess) return rc;
    addr[device] = p;
  }
  *ptr = addr[device];
  return cudaSuccess;
}

}  // namespace rv9g

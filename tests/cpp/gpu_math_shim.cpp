// Host build of the CUDA kernels' per-sample arithmetic (dsp_math.cuh) for
// the CPU tests: the same 1D transforms, DC-only shortcut, intra closed forms
// and loop-filter line as the kernels, sequenced as the kernels sequence them
// (rows, then columns with the final rounding), without the warp plumbing.
#include <stdint.h>
#include <string.h>

#include "../../rivet-vp9_b200/csrc/gpu/dsp_math.cuh"

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

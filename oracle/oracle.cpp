// ORACLE — test infrastructure only. A CPU restatement of the reference
// decoder's reconstruction (safewords/rivet-vp9), used to check the CUDA
// engine and as the timed CPU baseline. Only tests/, __graft_entry__.smoke()
// and bench.py's cpu_baseline / reference legs load it; the product never
// does.
//
// It replays the records of the host parser (rv9_records.h) the way the
// reference's FrameDec::replay does (src/decoder/block.rs:1405-1498), with the
// reference's scalar kernels restated in C++:
//   - inverse transforms: src/dsp/itx.rs:117-570 (butterflies), :574-666
//     (the 32-bit wrapping lane at 8 bits, the 64-bit lane above), :689-749
//     (DC-only shortcut and dispatch);
//   - inter prediction: src/dsp/inter.rs:52-395 (8-tap, edge clamp, scaled);
//   - compound average: src/dsp/pixel.rs:22-50; DC add: :9-16;
//   - intra prediction: src/dsp/intra.rs:19-175, edges recon.rs:17-103;
//   - dequantisation: src/decoder/recon.rs:219-281;
//   - motion vector selection/clamping/scaling: recon.rs:106-217,
//     src/decoder/mod.rs:495-541;
//   - loop filter: src/decoder/loopfilter.rs:15-181,466-620 and
//     src/dsp/lf.rs:24-259;
//   - output packing: src/decoder/mod.rs:79-106.
// Parity of this oracle with the reference is pinned by the per-frame MD5s of
// the reference's committed conformance vectors (tests/data/*.md5).
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../include/rv9.h"
#include "../rivet-vp9_b200/csrc/common/vp9_consts.h"
#include "../rivet-vp9_b200/csrc/common/vp9_tables.h"
#include "../rivet-vp9_b200/csrc/host/parser.h"

using namespace vp9;

namespace oracle {

template <class T>
static inline T clampv(T v, T lo, T hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}

// ---------------------------------------------------------------------------
// Inverse transforms (reference src/dsp/itx.rs).

static const int32_t COS64[33] = {16384, 16364, 16305, 16207, 16069, 15893, 15679, 15426, 15137,
                                  14811, 14449, 14053, 13623, 13160, 12665, 12140, 11585, 11003,
                                  10394, 9760,  9102,  8423,  7723,  7005,  6270,  5520,  4756,
                                  3981,  3196,  2404,  1606,  804,   0};
static const int32_t SINPI_1_9 = 5283, SINPI_2_9 = 9929, SINPI_3_9 = 13377, SINPI_4_9 = 15212;

static inline int32_t cos64(int32_t angle) {
  int32_t a2 = angle & 127;
  if (a2 <= 32) return COS64[a2];
  if (a2 <= 64) return -COS64[64 - a2];
  if (a2 <= 96) return -COS64[a2 - 64];
  return COS64[128 - a2];
}
static inline int32_t sin64(int32_t angle) { return cos64(angle - 32); }

static inline int brev(int num_bits, int x) {
  int t = 0;
  for (int i = 0; i < num_bits; ++i) t |= ((x >> i) & 1) << (num_bits - 1 - i);
  return t;
}

// The 8-bit lane: 32-bit integers with wrapping arithmetic.
struct S32 {
  int32_t v;
  static S32 zero() { return S32{0}; }
  S32 add(S32 o) const { return S32{(int32_t)((uint32_t)v + (uint32_t)o.v)}; }
  S32 sub(S32 o) const { return S32{(int32_t)((uint32_t)v - (uint32_t)o.v)}; }
  S32 mul(int32_t c) const { return S32{(int32_t)((uint32_t)v * (uint32_t)c)}; }
  S32 round_shift(int n) const { return S32{(int32_t)((uint32_t)v + (1u << (n - 1))) >> n}; }
  S32 sar(int n) const { return S32{v >> n}; }
  static S32 load(int32_t x) { return S32{x}; }
  void add_to(uint16_t* d, int32_t max) const {
    int32_t r = clampv<int32_t>(v, -(1 << 16), 1 << 16);
    *d = (uint16_t)clampv<int32_t>((int32_t)*d + r, 0, max);
  }
};

// The lane above 8 bits: 64-bit values; a multiplication takes the low 32
// bits of its operand, sign-extended (reference src/dsp/itx.rs:616-666).
struct S64 {
  int64_t v;
  static S64 zero() { return S64{0}; }
  S64 add(S64 o) const { return S64{(int64_t)((uint64_t)v + (uint64_t)o.v)}; }
  S64 sub(S64 o) const { return S64{(int64_t)((uint64_t)v - (uint64_t)o.v)}; }
  S64 mul(int32_t c) const { return S64{(int64_t)(int32_t)(uint32_t)(uint64_t)v * (int64_t)c}; }
  S64 round_shift(int n) const { return S64{(int64_t)((uint64_t)v + (1ull << (n - 1))) >> n}; }
  S64 sar(int n) const { return S64{v >> n}; }
  static S64 load(int32_t x) { return S64{x}; }
  void add_to(uint16_t* d, int32_t max) const {
    int32_t r = (int32_t)clampv<int64_t>(v, -(1 << 16), 1 << 16);
    *d = (uint16_t)clampv<int32_t>((int32_t)*d + r, 0, max);
  }
};

template <class V>
static inline V round14(V x) {
  return x.round_shift(14);
}

// B( a, b, angle, flip ).
template <class V>
static inline void bfly(V* t, int a, int b, int angle, bool flip) {
  int32_t c = cos64(angle), s = sin64(angle);
  V x = round14(t[a].mul(c).sub(t[b].mul(s)));
  V y = round14(t[a].mul(s).add(t[b].mul(c)));
  if (flip) {
    t[a] = y;
    t[b] = x;
  } else {
    t[a] = x;
    t[b] = y;
  }
}
// H( a, b, flip ).
template <class V>
static inline void hada(V* t, int a, int b, bool flip) {
  if (flip) std::swap(a, b);
  V x = t[a], y = t[b];
  t[a] = x.add(y);
  t[b] = x.sub(y);
}
// SB( a, b, angle, flip ).
template <class V>
static inline void sbfly(const V* t, V* s, int a, int b, int angle, bool flip) {
  int32_t c = cos64(angle), sn = sin64(angle);
  V x = t[a].mul(c).sub(t[b].mul(sn));
  V y = t[a].mul(sn).add(t[b].mul(c));
  if (flip) {
    s[a] = y;
    s[b] = x;
  } else {
    s[a] = x;
    s[b] = y;
  }
}
// SH( a, b ).
template <class V>
static inline void shada(V* t, const V* s, int a, int b) {
  t[a] = round14(s[a].add(s[b]));
  t[b] = round14(s[a].sub(s[b]));
}

// The inverse DCT steps after the recursive call (spec 8.7.1.3).
template <class V>
static void idct_stage(V* t, int n) {
  int n0 = 1 << n, n1 = n0 >> 1, n2 = n0 >> 2, n3 = n0 >> 3;
  for (int i = 0; i < n2; ++i) bfly(t, n1 + i, n0 - 1 - i, 32 - brev(5, n1 + i), false);
  if (n >= 3)
    for (int i = 0; i < n3; ++i)
      for (int j = 0; j < 2; ++j) hada(t, n1 + 4 * i + 2 * j, n1 + 1 + 4 * i + 2 * j, j == 1);
  if (n == 5) {
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j)
        bfly(t, n0 - n + 3 - n2 * j - 4 * i, n1 + n - 4 + n2 * j + 4 * i, 28 - 16 * i + 56 * j, true);
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 4; ++j) hada(t, n1 + n3 * j + i, n1 + n2 - 5 + n3 * j - i, (j & 1) == 1);
  }
  if (n >= 4) {
    int imax = n == 5 ? 1 : 0;
    for (int i = 0; i <= imax; ++i)
      for (int j = 0; j < 2; ++j) bfly(t, n0 - n + 2 - i - n2 * j, n1 + n - 3 + i + n2 * j, 24 + 48 * j, true);
    for (int i = 0; i < 2 * n - 6; ++i)
      for (int j = 0; j < 2; ++j) hada(t, n1 + n2 * j + i, n1 + n2 - 1 + n2 * j - i, (j & 1) == 1);
  }
  if (n >= 3)
    for (int i = 0; i < n3; ++i) bfly(t, n0 - n3 - 1 - i, n1 + n3 + i, 16, true);
  for (int i = 0; i < n1; ++i) hada(t, i, n0 - 1 - i, false);
}

template <class V>
static void idct(V* t, int n) {
  int n0 = 1 << n;
  V copy[32];
  for (int i = 0; i < n0; ++i) copy[i] = t[i];
  for (int i = 0; i < n0; ++i) t[i] = copy[brev(n, i)];
  bfly(t, 0, 1, 16, true);
  idct_stage(t, 2);
  for (int k = 3; k <= n; ++k) idct_stage(t, k);
}

template <class V>
static void adst_in_perm(V* t, int n) {
  int n0 = 1 << n, n1 = n0 >> 1;
  V copy[16];
  for (int i = 0; i < n0; ++i) copy[i] = t[i];
  for (int i = 0; i < n1; ++i) {
    t[2 * i] = copy[n0 - 1 - 2 * i];
    t[2 * i + 1] = copy[2 * i];
  }
}

template <class V>
static void adst_out_perm(V* t, int n) {
  V copy[16];
  for (int i = 0; i < (1 << n); ++i) copy[i] = t[i];
  if (n == 4) {
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int c = 0; c < 2; ++c)
          for (int d = 0; d < 2; ++d) t[8 * a + 4 * b + 2 * c + d] = copy[8 * (d ^ c) + 4 * (c ^ b) + 2 * (b ^ a) + a];
  } else {
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int c = 0; c < 2; ++c) t[4 * a + 2 * b + c] = copy[4 * (c ^ b) + 2 * (b ^ a) + a];
  }
}

template <class V>
static void iadst4(V* t) {
  V s0 = t[0].mul(SINPI_1_9), s1 = t[0].mul(SINPI_2_9), s2 = t[1].mul(SINPI_3_9);
  V s3 = t[2].mul(SINPI_4_9), s4 = t[2].mul(SINPI_1_9), s5 = t[3].mul(SINPI_2_9);
  V s6 = t[3].mul(SINPI_4_9);
  V v = t[0].sub(t[2]).add(t[3]);
  V s7 = v.mul(SINPI_3_9);
  V x0 = s0.add(s3).add(s5), x1 = s1.sub(s4).sub(s6), x2 = s7, x3 = s2;
  t[0] = round14(x0.add(x3));
  t[1] = round14(x1.add(x3));
  t[2] = round14(x2);
  t[3] = round14(x0.add(x1).sub(x3));
}

template <class V>
static void iadst8(V* t) {
  V s[8];
  for (auto& x : s) x = V::zero();
  adst_in_perm(t, 3);
  for (int i = 0; i < 4; ++i) sbfly(t, s, 2 * i, 1 + 2 * i, 30 - 8 * i, true);
  for (int i = 0; i < 4; ++i) shada(t, s, i, 4 + i);
  for (int i = 0; i < 2; ++i) sbfly(t, s, 4 + 3 * i, 5 + i, 24 - 16 * i, true);
  for (int i = 0; i < 2; ++i) shada(t, s, 4 + i, 6 + i);
  for (int i = 0; i < 2; ++i) hada(t, i, 2 + i, false);
  for (int i = 0; i < 2; ++i) bfly(t, 2 + 4 * i, 3 + 4 * i, 16, true);
  adst_out_perm(t, 3);
  for (int i = 0; i < 4; ++i) t[1 + 2 * i] = V::zero().sub(t[1 + 2 * i]);
}

template <class V>
static void iadst16(V* t) {
  V s[16];
  for (auto& x : s) x = V::zero();
  adst_in_perm(t, 4);
  for (int i = 0; i < 8; ++i) sbfly(t, s, 2 * i, 1 + 2 * i, 31 - 4 * i, true);
  for (int i = 0; i < 8; ++i) shada(t, s, i, 8 + i);
  for (int i = 0; i < 4; ++i) sbfly(t, s, 8 + 2 * i, 9 + 2 * i, 28 - 16 * i, true);
  for (int i = 0; i < 4; ++i) shada(t, s, 8 + i, 12 + i);
  for (int i = 0; i < 4; ++i) hada(t, i, 4 + i, false);
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) sbfly(t, s, 4 + 8 * i + 3 * j, 5 + 8 * i + j, 24 - 16 * j, true);
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) shada(t, s, 4 + 8 * j + i, 6 + 8 * j + i);
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) hada(t, 8 * j + i, 2 + 8 * j + i, false);
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) bfly(t, 2 + 4 * j + 8 * i, 3 + 4 * j + 8 * i, 48 + 64 * (i ^ j), false);
  adst_out_perm(t, 4);
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) t[1 + 12 * j + 2 * i] = V::zero().sub(t[1 + 12 * j + 2 * i]);
}

// The inverse Walsh-Hadamard transform (spec 8.7.1.10).
template <class V>
static void iwht(V* t, int shift) {
  V a = t[0].sar(shift), c = t[1].sar(shift), d = t[2].sar(shift), b = t[3].sar(shift);
  a = a.add(c);
  d = d.sub(b);
  V e = a.sub(d).sar(1);
  b = e.sub(b);
  c = e.sub(c);
  a = a.sub(b);
  d = d.add(c);
  t[0] = a;
  t[1] = b;
  t[2] = c;
  t[3] = d;
}

template <class V>
static void tx1d(V* t, int n, bool dct, bool lossless, int wht_shift) {
  if (lossless)
    iwht(t, wht_shift);
  else if (dct)
    idct(t, n);
  else if (n == 2)
    iadst4(t);
  else if (n == 3)
    iadst8(t);
  else
    iadst16(t);
}

// The 2D inverse transform added to dst (reference inverse_2d_add,
// src/dsp/itx.rs:519-570), one row or column per 1D transform.
template <class V>
static void inverse_2d_add(const int32_t* coefs, int n, int tx_type, bool lossless, uint16_t* dst, int stride,
                           int32_t max) {
  int n0 = 1 << n;
  V cols[32][32];  // [row][col] of the row transforms' output
  bool row_dct = tx_type == DCT_DCT || tx_type == ADST_DCT;
  bool col_dct = tx_type == DCT_DCT || tx_type == DCT_ADST;
  V t[32];
  for (int r = 0; r < n0; ++r) {
    const int32_t* src = coefs + r * n0;
    bool zero = true;
    for (int k = 0; k < n0; ++k) zero &= src[k] == 0;
    if (!lossless && zero) {
      for (int k = 0; k < n0; ++k) cols[r][k] = V::zero();
      continue;
    }
    for (int k = 0; k < n0; ++k) t[k] = V::load(src[k]);
    tx1d(t, n, row_dct, lossless, 2);
    for (int k = 0; k < n0; ++k) cols[r][k] = t[k];
  }
  int shift = std::min(n + 2, 6);
  for (int c = 0; c < n0; ++c) {
    for (int i = 0; i < n0; ++i) t[i] = cols[i][c];
    tx1d(t, n, col_dct, lossless, 0);
    for (int i = 0; i < n0; ++i) {
      V r = lossless ? t[i] : t[i].round_shift(shift);
      r.add_to(&dst[i * stride + c], max);
    }
  }
}

static int32_t dc_only_value(int32_t dc, int n) {
  int32_t c = cos64(16);
  S32 v = S32{dc}.mul(c).round_shift(14);
  S32 w = v.mul(c).round_shift(14);
  return w.round_shift(std::min(n + 2, 6)).v;
}

static void add_const(uint16_t* dst, int stride, int n, int32_t v) {
  v = clampv<int32_t>(v, -(1 << 16), 1 << 16);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) dst[i * stride + j] = (uint16_t)clampv<int32_t>(dst[i * stride + j] + v, 0, 255);
}

// inverse_transform_add (reference src/dsp/itx.rs:701-749).
static void inverse_transform_add(const int32_t* coefs, int n, int tx_type, bool lossless, int eob, int bit_depth,
                                  uint16_t* dst, int stride) {
  if (bit_depth > 8) {
    inverse_2d_add<S64>(coefs, n, tx_type, lossless, dst, stride, (1 << bit_depth) - 1);
    return;
  }
  if (eob == 1 && tx_type == DCT_DCT && !lossless) {
    add_const(dst, stride, 1 << n, dc_only_value(coefs[0], n));
    return;
  }
  inverse_2d_add<S32>(coefs, n, tx_type, lossless, dst, stride, 255);
}

// ---------------------------------------------------------------------------
// Inter prediction (reference src/dsp/inter.rs:289-395): the specification's
// formula with clamped reference coordinates; a horizontal pass rounded and
// clamped, then a vertical pass.

struct RefPlane {
  const uint16_t* data;
  int stride;
  int last_x, last_y;
};

static void inter_predict(const RefPlane& r, int x, int y, int x_step, int y_step, int w, int h, int filter,
                          int bit_depth, uint16_t* out, int out_stride) {
  int max = (1 << bit_depth) - 1;
  int ih = (((h - 1) * y_step + 15) >> 4) + 8;
  int y0 = (y >> 4) - 3;
  std::vector<uint16_t> tmp((size_t)ih * w);
  const int32_t(*f)[8] = vp9t_subpel_filters[filter];
  for (int row = 0; row < ih; ++row) {
    int ry = clampv(y0 + row, 0, r.last_y);
    const uint16_t* src = r.data + (size_t)ry * r.stride;
    for (int c = 0; c < w; ++c) {
      int p = x + x_step * c;
      int base = (p >> 4) - 3;
      const int32_t* t = f[p & 15];
      int32_t sum = 0;
      for (int k = 0; k < 8; ++k) sum += t[k] * src[clampv(base + k, 0, r.last_x)];
      tmp[(size_t)row * w + c] = (uint16_t)clampv((sum + 64) >> 7, 0, max);
    }
  }
  for (int rr = 0; rr < h; ++rr) {
    int p = (y & 15) + y_step * rr;
    int base = p >> 4;
    const int32_t* t = f[p & 15];
    for (int c = 0; c < w; ++c) {
      int32_t sum = 0;
      for (int k = 0; k < 8; ++k) sum += t[k] * tmp[(size_t)(base + k) * w + c];
      out[rr * out_stride + c] = (uint16_t)clampv((sum + 64) >> 7, 0, max);
    }
  }
}

// ---------------------------------------------------------------------------
// Intra prediction (reference src/dsp/intra.rs:19-175).

static inline int32_t r2(int32_t x, int n) { return (x + (1 << (n - 1))) >> n; }

static void intra_predict(int mode, int log2, const int32_t* above, const int32_t* left, bool have_left,
                          bool have_above, int bit_depth, uint16_t* dst, int stride) {
  int size = 1 << log2;
  auto a = [&](int i) { return above[i + 1]; };
  auto l = [&](int i) { return left[i]; };
  auto at = [&](int i, int j) -> uint16_t& { return dst[i * stride + j]; };
  switch (mode) {
    case V_PRED:
      for (int i = 0; i < size; ++i)
        for (int j = 0; j < size; ++j) at(i, j) = (uint16_t)a(j);
      break;
    case H_PRED:
      for (int i = 0; i < size; ++i)
        for (int j = 0; j < size; ++j) at(i, j) = (uint16_t)l(i);
      break;
    case D207_PRED:
      for (int j = 0; j < size; ++j) at(size - 1, j) = (uint16_t)l(size - 1);
      for (int i = 0; i < size - 1; ++i) at(i, 0) = (uint16_t)r2(l(i) + l(i + 1), 1);
      for (int i = 0; i < size - 2; ++i) at(i, 1) = (uint16_t)r2(l(i) + 2 * l(i + 1) + l(i + 2), 2);
      at(size - 2, 1) = (uint16_t)r2(l(size - 2) + 3 * l(size - 1), 2);
      for (int j = 2; j < size; ++j)
        for (int i = size - 2; i >= 0; --i) at(i, j) = at(i + 1, j - 2);
      break;
    case D45_PRED:
      for (int i = 0; i < size; ++i)
        for (int j = 0; j < size; ++j) {
          int k = i + j;
          at(i, j) = (uint16_t)(i + j + 2 < size * 2 ? r2(a(k) + a(k + 1) * 2 + a(k + 2), 2) : a(2 * size - 1));
        }
      break;
    case D63_PRED:
      for (int i = 0; i < size; ++i)
        for (int j = 0; j < size; ++j) {
          int k = i / 2 + j;
          at(i, j) = (uint16_t)((i & 1) ? r2(a(k) + a(k + 1) * 2 + a(k + 2), 2) : r2(a(k) + a(k + 1), 1));
        }
      break;
    case D117_PRED:
      for (int j = 0; j < size; ++j) at(0, j) = (uint16_t)r2(a(j - 1) + a(j), 1);
      at(1, 0) = (uint16_t)r2(l(0) + 2 * a(-1) + a(0), 2);
      for (int j = 1; j < size; ++j) at(1, j) = (uint16_t)r2(a(j - 2) + 2 * a(j - 1) + a(j), 2);
      at(2, 0) = (uint16_t)r2(a(-1) + 2 * l(0) + l(1), 2);
      for (int i = 3; i < size; ++i) at(i, 0) = (uint16_t)r2(l(i - 3) + 2 * l(i - 2) + l(i - 1), 2);
      for (int i = 2; i < size; ++i)
        for (int j = 1; j < size; ++j) at(i, j) = at(i - 2, j - 1);
      break;
    case D135_PRED:
      at(0, 0) = (uint16_t)r2(l(0) + 2 * a(-1) + a(0), 2);
      for (int j = 1; j < size; ++j) at(0, j) = (uint16_t)r2(a(j - 2) + 2 * a(j - 1) + a(j), 2);
      at(1, 0) = (uint16_t)r2(a(-1) + 2 * l(0) + l(1), 2);
      for (int i = 2; i < size; ++i) at(i, 0) = (uint16_t)r2(l(i - 2) + 2 * l(i - 1) + l(i), 2);
      for (int i = 1; i < size; ++i)
        for (int j = 1; j < size; ++j) at(i, j) = at(i - 1, j - 1);
      break;
    case D153_PRED:
      at(0, 0) = (uint16_t)r2(l(0) + a(-1), 1);
      for (int i = 1; i < size; ++i) at(i, 0) = (uint16_t)r2(l(i - 1) + l(i), 1);
      at(0, 1) = (uint16_t)r2(l(0) + 2 * a(-1) + a(0), 2);
      at(1, 1) = (uint16_t)r2(a(-1) + 2 * l(0) + l(1), 2);
      for (int i = 2; i < size; ++i) at(i, 1) = (uint16_t)r2(l(i - 2) + 2 * l(i - 1) + l(i), 2);
      for (int j = 2; j < size; ++j) at(0, j) = (uint16_t)r2(a(j - 3) + 2 * a(j - 2) + a(j - 1), 2);
      for (int i = 1; i < size; ++i)
        for (int j = 2; j < size; ++j) at(i, j) = at(i - 1, j - 2);
      break;
    case TM_PRED: {
      int max = (1 << bit_depth) - 1;
      for (int i = 0; i < size; ++i)
        for (int j = 0; j < size; ++j) at(i, j) = (uint16_t)clampv(a(j) + l(i) - a(-1), 0, max);
      break;
    }
    default: {  // DC_PRED
      int32_t v;
      if (have_left && have_above) {
        int32_t sum = 0;
        for (int k = 0; k < size; ++k) sum += l(k) + a(k);
        v = (sum + size) >> (log2 + 1);
      } else if (have_left) {
        int32_t sum = 0;
        for (int k = 0; k < size; ++k) sum += l(k);
        v = (sum + (1 << (log2 - 1))) >> log2;
      } else if (have_above) {
        int32_t sum = 0;
        for (int k = 0; k < size; ++k) sum += a(k);
        v = (sum + (1 << (log2 - 1))) >> log2;
      } else {
        v = 1 << (bit_depth - 1);
      }
      for (int i = 0; i < size; ++i)
        for (int j = 0; j < size; ++j) at(i, j) = (uint16_t)v;
    }
  }
}

// ---------------------------------------------------------------------------
// Loop filter samples (reference src/dsp/lf.rs:24-143).

static void lf_narrow(uint16_t* buf, ptrdiff_t pos, ptrdiff_t step, bool hev, int bd, int p1, int p0, int q0,
                      int q1) {
  int lo = -(1 << (bd - 1)), hi = (1 << (bd - 1)) - 1;
  auto c = [&](int v) { return clampv(v, lo, hi); };
  int off = 0x80 << (bd - 8);
  int ps1 = p1 - off, ps0 = p0 - off, qs0 = q0 - off, qs1 = q1 - off;
  int f = hev ? c(ps1 - qs1) : 0;
  f = c(f + 3 * (qs0 - ps0));
  int f1 = c(f + 4) >> 3, f2 = c(f + 3) >> 3;
  buf[pos] = (uint16_t)(c(qs0 - f1) + off);
  buf[pos - step] = (uint16_t)(c(ps0 + f2) + off);
  if (!hev) {
    int g = (f1 + 1) >> 1;
    buf[pos + step] = (uint16_t)(c(qs1 - g) + off);
    buf[pos - 2 * step] = (uint16_t)(c(ps1 + g) + off);
  }
}

static void lf_wide(uint16_t* buf, ptrdiff_t pos, ptrdiff_t step, int log2_size) {
  int n = (1 << (log2_size - 1)) - 1;
  int s[16], f[16];
  for (int k = -(n + 1); k <= n; ++k) s[k + 8] = buf[pos + k * step];
  for (int i = -n; i < n; ++i) {
    int t = s[i + 8];
    for (int j = -n; j <= n; ++j) t += s[clampv(i + j, -(n + 1), n) + 8];
    f[i + 8] = (t + (1 << (log2_size - 1))) >> log2_size;
  }
  for (int i = -n; i < n; ++i) buf[pos + i * step] = (uint16_t)f[i + 8];
}

static void lf_filter(uint16_t* buf, ptrdiff_t pos, ptrdiff_t step, int filter_size, int limit, int blimit,
                      int thresh, int bd) {
  auto at = [&](int k) { return (int)buf[pos + k * step]; };
  int q0 = at(0), q1 = at(1), q2 = at(2), q3 = at(3);
  int p0 = at(-1), p1 = at(-2), p2 = at(-3), p3 = at(-4);
  int sh = bd - 8;
  int limit_bd = limit << sh, blimit_bd = blimit << sh;
  if (std::abs(p3 - p2) > limit_bd || std::abs(p2 - p1) > limit_bd || std::abs(p1 - p0) > limit_bd ||
      std::abs(q1 - q0) > limit_bd || std::abs(q2 - q1) > limit_bd || std::abs(q3 - q2) > limit_bd ||
      std::abs(p0 - q0) * 2 + std::abs(p1 - q1) / 2 > blimit_bd)
    return;
  int thresh_bd = thresh << sh;
  bool hev = std::abs(p1 - p0) > thresh_bd || std::abs(q1 - q0) > thresh_bd;
  int one = 1 << sh;
  bool flat = filter_size >= 1 && std::abs(p1 - p0) <= one && std::abs(q1 - q0) <= one &&
              std::abs(p2 - p0) <= one && std::abs(q2 - q0) <= one && std::abs(p3 - p0) <= one &&
              std::abs(q3 - q0) <= one;
  if (filter_size == 0 || !flat) {
    lf_narrow(buf, pos, step, hev, bd, p1, p0, q0, q1);
    return;
  }
  bool flat2 = false;
  if (filter_size >= 2) {
    flat2 = true;
    for (int k = 4; k < 8; ++k)
      if (std::abs(at(-k - 1) - p0) > one || std::abs(at(k) - q0) > one) {
        flat2 = false;
        break;
      }
  }
  lf_wide(buf, pos, step, (filter_size == 1 || !flat2) ? 3 : 4);
}

// ---------------------------------------------------------------------------
// Frames and reconstruction.

struct Plane {
  std::vector<uint16_t> data;
  int stride = 0, height = 0;
};

struct Picture {
  uint32_t width = 0, height = 0, ss_x = 1, ss_y = 1, bit_depth = 8;
  uint8_t color_space = 1, color_range = 0;
  uint32_t render_w = 0, render_h = 0;
  Plane planes[3];
};

struct MiLf {
  uint8_t mi_size, skip, tx_size, y_mode, segment_id;
  int8_t ref_frame0;
};

struct FrameRecon {
  const rv9_frame_desc& d;
  Picture& cur;
  const Picture* refs[3];
  std::vector<int32_t> coefs = std::vector<int32_t>(1024, 0);
  std::vector<uint16_t> pred_buf = std::vector<uint16_t>(2 * 64 * 64, 0);

  FrameRecon(const rv9_frame_desc& desc, Picture& c) : d(desc), cur(c) {}

  bool seg_active(int seg, int f) const { return d.seg.enabled && d.seg.feature_enabled[seg][f]; }

  int uv_tx_size(const rv9_block& b) const {
    if (b.mi_size < BLOCK_8X8) return TX_4X4;
    int sx = d.legacy_uv ? 1 : d.ss_x, sy = d.legacy_uv ? 1 : d.ss_y;
    int uv = SS_SIZE_LOOKUP[b.mi_size][sx][sy];
    return std::min<int>(b.tx_size, MAX_TXSIZE_LOOKUP[uv]);
  }

  // predict_intra (reference src/decoder/recon.rs:17-103).
  void predict_intra(const rv9_block& b, int plane, int x, int y, bool have_left, bool have_above,
                     bool not_on_right, int tx_sz, int block_idx) {
    int mode = plane > 0 ? b.uv_mode : (b.mi_size >= BLOCK_8X8 ? b.y_mode : b.sub_modes[block_idx]);
    int log2 = tx_sz + 2, size = 1 << log2;
    int sx = plane > 0 ? d.ss_x : 0, sy = plane > 0 ? d.ss_y : 0;
    int max_x = (int)((d.mi_cols * 8) >> sx) - 1;
    int max_y = (int)((d.mi_rows * 8) >> sy) - 1;
    int base = 1 << (d.bit_depth - 1);
    Plane& buf = cur.planes[plane];
    int stride = buf.stride;
    int32_t above[65], left[32];
    if (have_above) {
      const uint16_t* row = buf.data.data() + (size_t)(y - 1) * stride;
      for (int i = 0; i < size; ++i) above[1 + i] = row[std::min(max_x, x + i)];
      if (not_on_right && tx_sz == TX_4X4) {
        for (int i = size; i < 2 * size; ++i) above[1 + i] = row[std::min(max_x, x + i)];
      } else {
        for (int i = size; i < 2 * size; ++i) above[1 + i] = above[size];
      }
      above[0] = have_left ? row[std::min(max_x, x - 1)] : base + 1;
    } else {
      for (int i = 0; i < 2 * size; ++i) above[1 + i] = base - 1;
      above[0] = base - 1;
    }
    if (have_left) {
      for (int i = 0; i < size; ++i) left[i] = buf.data[(size_t)std::min(max_y, y + i) * stride + x - 1];
    } else {
      for (int i = 0; i < size; ++i) left[i] = base + 1;
    }
    intra_predict(mode, log2, above, left, have_left, have_above, d.bit_depth,
                  buf.data.data() + (size_t)y * stride + x, stride);
  }

  static int32_t q2(int32_t v) { return (v < 0 ? v - 1 : v + 1) / 2; }
  static int32_t q4(int32_t v) { return (v < 0 ? v - 2 : v + 2) / 4; }

  // predict_inter (reference src/decoder/recon.rs:106-217).
  void predict_inter(const rv9_block& b, int plane, int x, int y, int w, int h, int block_idx) {
    bool is_compound = b.ref_frame[1] > INTRA_FRAME;
    for (int ref_list = 0; ref_list < 1 + (is_compound ? 1 : 0); ++ref_list) {
      const int32_t(*bm)[2] = b.mv[ref_list];
      int32_t mv[2];
      if (plane == 0 || b.mi_size >= BLOCK_8X8) {
        mv[0] = bm[block_idx][0];
        mv[1] = bm[block_idx][1];
      } else {
        int usx = d.legacy_uv ? 1 : d.ss_x, usy = d.legacy_uv ? 1 : d.ss_y;
        if (usx == 0 && usy == 0) {
          mv[0] = bm[block_idx][0];
          mv[1] = bm[block_idx][1];
        } else if (usx == 0) {
          mv[0] = q2(bm[block_idx][0] + bm[block_idx + 2][0]);
          mv[1] = q2(bm[block_idx][1] + bm[block_idx + 2][1]);
        } else if (usy == 0) {
          mv[0] = q2(bm[block_idx][0] + bm[block_idx + 1][0]);
          mv[1] = q2(bm[block_idx][1] + bm[block_idx + 1][1]);
        } else {
          mv[0] = q4(bm[0][0] + bm[1][0] + bm[2][0] + bm[3][0]);
          mv[1] = q4(bm[0][1] + bm[1][1] + bm[2][1] + bm[3][1]);
        }
      }
      int sx = plane > 0 ? d.ss_x : 0, sy = plane > 0 ? d.ss_y : 0;
      int bh = vp9t_num_8x8_high[b.mi_size], bw = vp9t_num_8x8_wide[b.mi_size];
      int mi_row = b.mi_row, mi_col = b.mi_col;
      int to_top = -((mi_row * 8) * 16) >> sy;
      int to_bottom = ((((int)d.mi_rows - bh - mi_row) * 8) * 16) >> sy;
      int to_left = -((mi_col * 8) * 16) >> sx;
      int to_right = ((((int)d.mi_cols - bw - mi_col) * 8) * 16) >> sx;
      int spel_left = (INTERP_EXTEND + ((bw * 8) >> sx)) << 4;
      int spel_right = spel_left - 16;
      int spel_top = (INTERP_EXTEND + ((bh * 8) >> sy)) << 4;
      int spel_bottom = spel_top - 16;
      int32_t cmv[2] = {clampv((2 * mv[0]) >> sy, to_top - spel_top, to_bottom + spel_bottom),
                        clampv((2 * mv[1]) >> sx, to_left - spel_left, to_right + spel_right)};
      // Scaling (reference src/decoder/mod.rs:503-541).
      int ri = b.ref_frame[ref_list] - LAST_FRAME;
      const Picture* r = refs[ri];
      int64_t xs = ((int64_t)r->width << 14) / d.width;
      int64_t ys = ((int64_t)r->height << 14) / d.height;
      int64_t base_x = ((int64_t)x * xs) >> 14, base_y = ((int64_t)y * ys) >> 14;
      int64_t luma_x = plane > 0 ? ((int64_t)x << d.ss_x) : x;
      int64_t luma_y = plane > 0 ? ((int64_t)y << d.ss_y) : y;
      int64_t frac_x = ((16 * luma_x * xs) >> 14) & 15;
      int64_t frac_y = ((16 * luma_y * ys) >> 14) & 15;
      int64_t dx = (((int64_t)cmv[1] * xs) >> 14) + frac_x;
      int64_t dy = (((int64_t)cmv[0] * ys) >> 14) + frac_y;
      int step_x = (int)((16 * xs) >> 14), step_y = (int)((16 * ys) >> 14);
      int start_x = (int)((base_x << 4) + dx), start_y = (int)((base_y << 4) + dy);
      const Plane& rp = r->planes[plane];
      RefPlane refp{rp.data.data(), rp.stride, (int)((r->width + sx) >> sx) - 1, (int)((r->height + sy) >> sy) - 1};
      uint16_t* out;
      int out_stride;
      if (is_compound) {
        out = pred_buf.data() + ref_list * 64 * 64;
        out_stride = w;
      } else {
        Plane& buf = cur.planes[plane];
        out = buf.data.data() + (size_t)y * buf.stride + x;
        out_stride = buf.stride;
      }
      inter_predict(refp, start_x, start_y, step_x, step_y, w, h, b.interp_filter, d.bit_depth, out, out_stride);
    }
    if (is_compound) {
      Plane& buf = cur.planes[plane];
      uint16_t* dst = buf.data.data() + (size_t)y * buf.stride + x;
      for (int i = 0; i < h; ++i)
        for (int j = 0; j < w; ++j)
          dst[i * buf.stride + j] = (uint16_t)((pred_buf[i * w + j] + pred_buf[64 * 64 + i * w + j] + 1) >> 1);
    }
  }

  int qindex(int seg) const {
    if (seg_active(seg, SEG_LVL_ALT_Q)) {
      int data = d.seg.feature_data[seg][SEG_LVL_ALT_Q];
      if (!d.seg.abs_or_delta_update) data += d.base_q_idx;
      return clampv(data, 0, 255);
    }
    return d.base_q_idx;
  }

  // reconstruct (reference src/decoder/recon.rs:233-281) for one recorded
  // transform block.
  void reconstruct(const rv9_block& b, const rv9_tok& t, const uint32_t* words) {
    int plane = t.plane, tx_sz = t.tx_size;
    int bd_idx = (d.bit_depth - 8) >> 1;
    int q = qindex(b.segment_id);
    int dc_delta = plane == 0 ? d.delta_q_y_dc : d.delta_q_uv_dc;
    int ac_delta = plane == 0 ? 0 : d.delta_q_uv_ac;
    int64_t dc_q = vp9t_dc_qlookup[bd_idx][clampv(q + dc_delta, 0, 255)];
    int64_t ac_q = vp9t_ac_qlookup[bd_idx][clampv(q + ac_delta, 0, 255)];
    int n = 2 + tx_sz, n0 = 1 << n;
    std::fill(coefs.begin(), coefs.begin() + n0 * n0, 0);
    for (uint32_t i = 0; i < t.n_coef; ++i) {
      uint32_t w = words[t.coef_start + i];
      int pos = RV9_COEF_POS(w);
      int64_t v = RV9_COEF_VAL(w);
      int64_t dq = v * (pos == 0 ? dc_q : ac_q);
      if (tx_sz == TX_32X32) dq /= 2;
      coefs[pos] = (int32_t)clampv<int64_t>(dq, INT32_MIN, INT32_MAX);
    }
    Plane& buf = cur.planes[plane];
    inverse_transform_add(coefs.data(), n, t.tx_type, d.lossless, t.eob, d.bit_depth,
                          buf.data.data() + (size_t)t.y * buf.stride + t.x, buf.stride);
  }

  // replay (reference src/decoder/block.rs:1405-1498).
  bool replay(const rv9_block* blocks, size_t nb, const rv9_tok* toks, size_t ntoks, const uint32_t* words,
              std::string* err) {
    size_t tok = 0;
    for (size_t bi = 0; bi < nb; ++bi) {
      const rv9_block& b = blocks[bi];
      bool is_inter = b.flags & RV9_BLK_INTER;
      bool avail_l = b.flags & RV9_BLK_AVAIL_L, avail_u = b.flags & RV9_BLK_AVAIL_U;
      int bsize = std::max<int>(b.mi_size, BLOCK_8X8);
      tok = b.tok_start;
      for (int plane = 0; plane < 3; ++plane) {
        int tx_sz = plane > 0 ? uv_tx_size(b) : b.tx_size;
        int step = 1 << tx_sz;
        int sx = plane > 0 ? d.ss_x : 0, sy = plane > 0 ? d.ss_y : 0;
        int plane_sz = SS_SIZE_LOOKUP[bsize][sx][sy];
        int n4w = vp9t_num_4x4_wide[plane_sz], n4h = vp9t_num_4x4_high[plane_sz];
        int base_x = (b.mi_col * 8) >> sx, base_y = (b.mi_row * 8) >> sy;
        if (is_inter) {
          if (b.mi_size < BLOCK_8X8) {
            for (int y = 0; y < n4h; ++y)
              for (int x = 0; x < n4w; ++x) predict_inter(b, plane, base_x + 4 * x, base_y + 4 * y, 4, 4, y * n4w + x);
          } else {
            predict_inter(b, plane, base_x, base_y, n4w * 4, n4h * 4, 0);
          }
        }
        int max_x = (int)((d.mi_cols * 8) >> sx), max_y = (int)((d.mi_rows * 8) >> sy);
        int block_idx = 0;
        for (int y = 0; y < n4h; y += step)
          for (int x = 0; x < n4w; x += step) {
            int start_x = base_x + 4 * x, start_y = base_y + 4 * y;
            if (start_x < max_x && start_y < max_y) {
              if (!is_inter)
                predict_intra(b, plane, start_x, start_y, avail_l || x > 0, avail_u || y > 0, x + step < n4w, tx_sz,
                              block_idx);
              if (!b.coded_skip) {
                if (tok >= ntoks) {
                  *err = "records: missing transform block";
                  return false;
                }
                const rv9_tok& t = toks[tok++];
                if (t.x != start_x || t.y != start_y || t.plane != plane) {
                  *err = "records: transform block out of order";
                  return false;
                }
                if (t.eob > 0) reconstruct(b, t, words);
              }
            }
            ++block_idx;
          }
      }
    }
    return true;
  }

  // ---- Loop filter (reference src/decoder/loopfilter.rs) ----

  uint8_t lvl[8][4][2];
  int params[64][3];

  void lf_setup() {
    int n_shift = d.lf_level >> 5;
    for (int segment_id = 0; segment_id < 8; ++segment_id) {
      int lvl_seg = d.lf_level;
      if (seg_active(segment_id, SEG_LVL_ALT_L)) {
        int data = d.seg.feature_data[segment_id][SEG_LVL_ALT_L];
        lvl_seg = d.seg.abs_or_delta_update ? data : data + d.lf_level;
        lvl_seg = clampv(lvl_seg, 0, MAX_LOOP_FILTER);
      }
      if (!d.lf_delta_enabled) {
        for (int r = 0; r < 4; ++r) lvl[segment_id][r][0] = lvl[segment_id][r][1] = (uint8_t)lvl_seg;
      } else {
        int intra = lvl_seg + (d.lf_ref_deltas[INTRA_FRAME] * (1 << n_shift));
        lvl[segment_id][0][0] = lvl[segment_id][0][1] = (uint8_t)clampv(intra, 0, MAX_LOOP_FILTER);
        for (int rf = 1; rf < 4; ++rf)
          for (int mode = 0; mode < 2; ++mode) {
            int inter = lvl_seg + d.lf_ref_deltas[rf] * (1 << n_shift) + d.lf_mode_deltas[mode] * (1 << n_shift);
            lvl[segment_id][rf][mode] = (uint8_t)clampv(inter, 0, MAX_LOOP_FILTER);
          }
      }
    }
    int shift = d.lf_sharpness > 4 ? 2 : (d.lf_sharpness > 0 ? 1 : 0);
    for (int l = 0; l < 64; ++l) {
      int limit = d.lf_sharpness > 0 ? clampv(l >> shift, 1, 9 - (int)d.lf_sharpness) : std::max(l >> shift, 1);
      params[l][0] = limit;
      params[l][1] = 2 * (l + 2) + limit;
      params[l][2] = l >> 4;
    }
  }

  struct Edges {
    int8_t fs[16][16];
    uint8_t limit[16][16], blimit[16][16], thresh[16][16];
  };

  // superblock (reference src/decoder/loopfilter.rs:466-620).
  void superblock(const std::vector<MiLf>& mi, int plane, int pass, uint32_t row, uint32_t col, Edges& e, int* gx0,
                  int* gy0, int* n_edges_out, int* n_runs_out) {
    uint32_t sub_x = plane > 0 ? d.ss_x : 0, sub_y = plane > 0 ? d.ss_y : 0;
    uint32_t sub = pass == 0 ? sub_x : sub_y;
    uint32_t edge_len = pass == 0 ? (64 >> sub_y) : (64 >> sub_x);
    uint32_t mi_rows = d.mi_rows, mi_cols = d.mi_cols;
    int n_edges = 16 >> sub, n_runs = edge_len / 4;
    for (int i = 0; i < n_edges; ++i)
      for (int j = 0; j < n_runs; ++j) e.fs[i][j] = -1;
    auto at = [&](uint32_t ed, uint32_t rn, uint32_t* x, uint32_t* y) {
      if (pass == 0) {
        *x = col * 8 + ed * (4 << sub_x);
        *y = row * 8 + ((4 * rn) << sub_y);
      } else {
        *x = col * 8 + ((4 * rn) << sub_x);
        *y = row * 8 + ed * (4 << sub_y);
      }
    };
    int ux = d.legacy_uv ? 1 : d.ss_x, uy = d.legacy_uv ? 1 : d.ss_y;
    for (uint32_t ca = 0; ca < (uint32_t)n_edges / 2; ++ca)
      for (uint32_t cb = 0; cb < (uint32_t)n_runs / 2; ++cb) {
        uint32_t x, y;
        at(2 * ca, 2 * cb, &x, &y);
        if (x >= 8 * mi_cols || y >= 8 * mi_rows) continue;
        uint32_t loop_col = ((x >> 3) >> sub_x) << sub_x;
        uint32_t loop_row = ((y >> 3) >> sub_y) << sub_y;
        const MiLf& m = mi[(size_t)loop_row * mi_cols + loop_col];
        int mode = m.y_mode;
        int mode_type = (mode == NEARESTMV || mode == NEARMV || mode == NEWMV) ? 1 : 0;
        int rf = std::max<int>(m.ref_frame0, 0);
        int l = lvl[m.segment_id][rf][mode_type];
        if (l == 0) continue;
        int limit = params[l][0], blimit = params[l][1], thresh = params[l][2];
        int mi_size = m.mi_size;
        int tx_sz;
        if (plane > 0) {
          if (mi_size < BLOCK_8X8) {
            tx_sz = TX_4X4;
          } else {
            int uv = SS_SIZE_LOOKUP[mi_size][ux][uy];
            tx_sz = std::min<int>(m.tx_size, MAX_TXSIZE_LOOKUP[uv]);
          }
        } else {
          tx_sz = m.tx_size;
        }
        int sb_size = sub == 0 ? mi_size : std::max<int>(mi_size, BLOCK_16X16);
        uint32_t block_mask = pass == 0 ? 8 * vp9t_num_8x8_wide[sb_size] - 1 : 8 * vp9t_num_8x8_high[sb_size] - 1;
        bool coded = m.ref_frame0 <= INTRA_FRAME || !m.skip;
        for (uint32_t eo = 0; eo < 2; ++eo) {
          uint32_t ed = 2 * ca + eo;
          at(ed, 2 * cb, &x, &y);
          if ((pass == 0 && x == 0) || (pass == 1 && y == 0)) continue;
          uint32_t across = pass == 0 ? x : y;
          bool is_block_edge = (across & block_mask) == 0;
          bool tx_edge = (ed & ((1u << tx_sz) - 1)) == 0;
          if (!is_block_edge && !(tx_edge && coded)) continue;
          bool is_32_edge = ed % 8 == 0;
          int base_size = (tx_sz == TX_4X4 && is_32_edge) ? TX_8X8 : std::min<int>(tx_sz, TX_16X16);
          int filter_size = base_size;
          if ((pass == 0 && sub_x == 1 && base_size == TX_16X16 && (x >> 3) == mi_cols - 1) ||
              (pass == 1 && sub_y == 1 && base_size == TX_16X16 && (y >> 3) == mi_rows - 1))
            filter_size = TX_8X8;
          for (uint32_t k = 0; k < 2; ++k) {
            uint32_t rn = 2 * cb + k;
            at(ed, rn, &x, &y);
            if (k == 1 && (x >= 8 * mi_cols || y >= 8 * mi_rows)) break;
            bool is_tx_edge = tx_edge;
            if (pass == 1 && sub_x == 1 && (mi_cols & 1) == 1 && (ed & 1) == 1 && (x + 8) >= mi_cols * 8)
              is_tx_edge = false;
            if (!(is_block_edge || (is_tx_edge && coded))) continue;
            e.fs[ed][rn] = (int8_t)filter_size;
            e.limit[ed][rn] = (uint8_t)limit;
            e.blimit[ed][rn] = (uint8_t)blimit;
            e.thresh[ed][rn] = (uint8_t)thresh;
          }
        }
      }
    *gx0 = (int)((col * 8) >> sub_x);
    *gy0 = (int)((row * 8) >> sub_y);
    *n_edges_out = n_edges;
    *n_runs_out = n_runs;
  }

  // The planes are filtered independently (each in the reference's order),
  // on their own threads when `threads` > 1.
  void filter_frame(const std::vector<MiLf>& mi, int threads = 1) {
    lf_setup();
    if (threads > 1) {
      std::thread t[3];
      for (int plane = 0; plane < 3; ++plane) t[plane] = std::thread([&, plane] { filter_plane(mi, plane); });
      for (auto& x : t) x.join();
    } else {
      for (int plane = 0; plane < 3; ++plane) filter_plane(mi, plane);
    }
  }

  void filter_plane(const std::vector<MiLf>& mi, int plane) {
    Edges e;
    {
      Plane& buf = cur.planes[plane];
      int stride = buf.stride;
      for (uint32_t row = 0; row < d.mi_rows; row += 8)
        for (uint32_t col = 0; col < d.mi_cols; col += 8)
          for (int pass = 0; pass < 2; ++pass) {
            int x0, y0, ne, nr;
            superblock(mi, plane, pass, row, col, e, &x0, &y0, &ne, &nr);
            bool vertical = pass == 0;
            ptrdiff_t step = vertical ? 1 : stride, along = vertical ? stride : 1;
            for (int ed = 0; ed < ne; ++ed)
              for (int r = 0; r < nr; ++r) {
                int fs = e.fs[ed][r];
                if (fs < 0) continue;
                ptrdiff_t pos = vertical ? (ptrdiff_t)(y0 + 4 * r) * stride + x0 + 4 * ed
                                         : (ptrdiff_t)(y0 + 4 * ed) * stride + x0 + 4 * r;
                for (int k = 0; k < 4; ++k)
                  lf_filter(buf.data.data(), pos + k * along, step, fs, e.limit[ed][r], e.blimit[ed][r],
                            e.thresh[ed][r], d.bit_depth);
              }
          }
    }
  }
};

// A decoder: the host parser and this CPU reconstruction.
struct Decoder {
  rv9::Parser parser;
  std::shared_ptr<Picture> slots[8];
  std::string err;
  double recon_seconds = 0;
  int threads = 1;  // tile columns reconstructed, and planes filtered, at once

  // Replays the frame's blocks, each tile column on its own thread when
  // threads > 1, as the reference decodes tile columns in parallel
  // (src/decoder/block.rs:1768-1863): a column reads nothing of another.
  bool replay_columns(const rv9::ParsedFrame& pf, Picture& pic) {
    const rv9_frame_desc& d = pf.desc;
    const uint32_t cols = 1u << d.tile_cols_log2;
    auto make = [&](FrameRecon* fr) {
      if (!d.frame_is_intra)
        for (int i = 0; i < 3; ++i) fr->refs[i] = slots[pf.ref_slot[i]].get();
    };
    if (threads <= 1 || cols <= 1) {
      FrameRecon fr(d, pic);
      make(&fr);
      return fr.replay(pf.blocks.data(), pf.blocks.size(), pf.toks.data(), pf.toks.size(), pf.coefs.data(), &err);
    }
    // Blocks of each column, in bitstream order. A column starts at
    // get_tile_offset (spec 6.4.1): ((c * sb64_cols) >> log2) superblocks.
    auto col_start = [&](uint32_t c) { return std::min<uint32_t>(((c * d.sb64_cols) >> d.tile_cols_log2) * 8, d.mi_cols); };
    std::vector<std::vector<rv9_block>> by_col(cols);
    for (const rv9_block& b : pf.blocks) {
      uint32_t c = 0;
      while (c + 1 < cols && b.mi_col >= col_start(c + 1)) ++c;
      by_col[c].push_back(b);
    }
    std::vector<std::string> errs(cols);
    std::vector<char> ok(cols, 1);
    std::vector<std::thread> pool;
    const uint32_t workers = std::min<uint32_t>(cols, (uint32_t)threads);
    for (uint32_t w = 0; w < workers; ++w)
      pool.emplace_back([&, w] {
        for (uint32_t c = w; c < cols; c += workers) {
          FrameRecon fr(d, pic);
          make(&fr);
          ok[c] = fr.replay(by_col[c].data(), by_col[c].size(), pf.toks.data(), pf.toks.size(), pf.coefs.data(),
                            &errs[c]);
        }
      });
    for (auto& t : pool) t.join();
    for (uint32_t c = 0; c < cols; ++c)
      if (!ok[c]) {
        err = errs[c];
        return false;
      }
    return true;
  }

  rv9_status decode_frame(const uint8_t* data, size_t len, std::vector<std::shared_ptr<Picture>>* shown) {
    rv9::ParsedFrame pf;
    rv9::Status st = parser.parse_frame(data, len, &pf, &err);
    if (st != rv9::ST_OK) return (rv9_status)st;
    if (pf.show_existing) {
      shown->push_back(slots[pf.show_slot]);
      return RV9_OK;
    }
    auto t0 = std::chrono::steady_clock::now();
    const rv9_frame_desc& d = pf.desc;
    auto pic = std::make_shared<Picture>();
    pic->width = d.width;
    pic->height = d.height;
    pic->ss_x = d.ss_x;
    pic->ss_y = d.ss_y;
    pic->bit_depth = d.bit_depth;
    pic->color_space = d.color_space;
    pic->color_range = d.color_range;
    pic->render_w = d.render_width;
    pic->render_h = d.render_height;
    int w = d.sb64_cols * 64, h = d.sb64_rows * 64;
    for (int p = 0; p < 3; ++p) {
      int pw = p ? w >> d.ss_x : w, ph = p ? h >> d.ss_y : h;
      pic->planes[p].data.assign((size_t)pw * ph, 0);
      pic->planes[p].stride = pw;
      pic->planes[p].height = ph;
    }
    if (!replay_columns(pf, *pic)) return RV9_BITSTREAM;
    FrameRecon fr(d, *pic);
    if (d.lf_level != 0) {
      std::vector<MiLf> mi((size_t)d.mi_rows * d.mi_cols);
      for (const rv9_block& b : pf.blocks) {
        MiLf m{b.mi_size, (uint8_t)((b.flags & RV9_BLK_SKIP) ? 1 : 0), b.tx_size, b.y_mode, b.segment_id,
               b.ref_frame[0]};
        uint32_t bh = vp9t_num_8x8_high[b.mi_size], bw = vp9t_num_8x8_wide[b.mi_size];
        for (uint32_t y = b.mi_row; y < std::min(b.mi_row + bh, d.mi_rows); ++y)
          for (uint32_t x = b.mi_col; x < std::min(b.mi_col + bw, d.mi_cols); ++x) mi[(size_t)y * d.mi_cols + x] = m;
      }
      fr.filter_frame(mi, threads);
    }
    recon_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int i = 0; i < 8; ++i)
      if ((pf.refresh_mask >> i) & 1) slots[i] = pic;
    if (pf.show_frame) shown->push_back(pic);
    return RV9_OK;
  }
};

static size_t frame_bytes(const Picture& p) {
  size_t bps = p.bit_depth > 8 ? 2 : 1;
  size_t cw = (p.width + p.ss_x) >> p.ss_x, ch = (p.height + p.ss_y) >> p.ss_y;
  return ((size_t)p.width * p.height + 2 * cw * ch) * bps;
}

// to_frame (reference src/decoder/mod.rs:79-106): the visible planes packed.
static void pack(const Picture& p, uint8_t* out, rv9_frame* f) {
  bool high = p.bit_depth > 8;
  size_t off = 0;
  for (int i = 0; i < 3; ++i) {
    uint32_t w = i ? (p.width + p.ss_x) >> p.ss_x : p.width;
    uint32_t h = i ? (p.height + p.ss_y) >> p.ss_y : p.height;
    const Plane& src = p.planes[i];
    if (f) {
      f->planes[i].offset = off;
      f->planes[i].width = w;
      f->planes[i].height = h;
    }
    for (uint32_t y = 0; y < h; ++y) {
      const uint16_t* row = src.data.data() + (size_t)y * src.stride;
      if (high) {
        for (uint32_t x = 0; x < w; ++x) {
          out[off + 2 * ((size_t)y * w + x)] = (uint8_t)(row[x] & 0xff);
          out[off + 2 * ((size_t)y * w + x) + 1] = (uint8_t)(row[x] >> 8);
        }
      } else {
        for (uint32_t x = 0; x < w; ++x) out[off + (size_t)y * w + x] = (uint8_t)row[x];
      }
    }
    off += (size_t)w * h * (high ? 2 : 1);
  }
  if (f) {
    f->width = p.width;
    f->height = p.height;
    f->bit_depth = p.bit_depth;
    f->chroma = p.ss_x ? (p.ss_y ? RV9_YUV420 : RV9_YUV422) : (p.ss_y ? RV9_YUV440 : RV9_YUV444);
    f->color_space = p.color_space;
    f->full_range = p.color_range;
    f->render_width = p.render_w;
    f->render_height = p.render_h;
    f->size = off;
  }
}

}  // namespace oracle

// ---------------------------------------------------------------------------
// C ABI of the oracle: the decoder API of rv9.h with an rv9o_ prefix.

extern "C" {

struct rv9o_decoder {
  oracle::Decoder dec;
};

rv9o_decoder* rv9o_decoder_new(void) { return new rv9o_decoder; }
void rv9o_decoder_free(rv9o_decoder* d) { delete d; }
void rv9o_decoder_set_threads(rv9o_decoder* d, uint32_t t) {
  d->dec.parser.set_threads((int)t);
  d->dec.threads = t ? (int)t : (int)std::max(1u, std::thread::hardware_concurrency());
}
void rv9o_decoder_set_max_pixels(rv9o_decoder* d, uint64_t p) { d->dec.parser.set_max_pixels(p); }
uint64_t rv9o_decoder_frames_decoded(const rv9o_decoder* d) { return d->dec.parser.frames_decoded(); }
const char* rv9o_last_error(const rv9o_decoder* d) { return d->dec.err.c_str(); }
double rv9o_recon_seconds(const rv9o_decoder* d) { return d->dec.recon_seconds; }

rv9_status rv9o_decode_all(rv9o_decoder* d, const uint8_t* pkt, size_t len, rv9_frame* out, size_t cap,
                           size_t* n_out) {
  std::vector<std::pair<size_t, size_t>> frames;
  rv9::superframe_split(pkt, len, &frames);
  std::vector<std::shared_ptr<oracle::Picture>> shown;
  *n_out = 0;
  for (auto& f : frames) {
    rv9_status st = d->dec.decode_frame(pkt + f.first, f.second, &shown);
    if (st != RV9_OK) return st;
  }
  for (auto& p : shown) {
    if (*n_out < cap) {
      rv9_frame* fr = &out[*n_out];
      size_t nbytes = oracle::frame_bytes(*p);
      fr->data = (uint8_t*)malloc(nbytes ? nbytes : 1);
      oracle::pack(*p, fr->data, fr);
    }
    ++*n_out;
  }
  return RV9_OK;
}

void rv9o_frame_release(rv9_frame* f) {
  free(f->data);
  f->data = nullptr;
  f->size = 0;
}

// Decodes `n` packets, writing every shown frame packed into `out`.
rv9_status rv9o_decode_packets(rv9o_decoder* d, const uint8_t* const* pkts, const size_t* lens, size_t n,
                               uint8_t* out, size_t cap, size_t* n_frames, size_t* bytes) {
  *n_frames = 0;
  *bytes = 0;
  std::vector<std::pair<size_t, size_t>> frames;
  std::vector<std::shared_ptr<oracle::Picture>> shown;
  for (size_t i = 0; i < n; ++i) {
    rv9::superframe_split(pkts[i], lens[i], &frames);
    for (auto& f : frames) {
      rv9_status st = d->dec.decode_frame(pkts[i] + f.first, f.second, &shown);
      if (st != RV9_OK) return st;
    }
    for (auto& p : shown) {
      size_t nb = oracle::frame_bytes(*p);
      if (*bytes + nb > cap) {
        d->dec.err = "output buffer too small";
        return RV9_INVALID_INPUT;
      }
      oracle::pack(*p, out + *bytes, nullptr);
      *bytes += nb;
      ++*n_frames;
    }
    shown.clear();
  }
  return RV9_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Entry points for the kernel-arithmetic tests: the oracle's sample
// operations on caller buffers.
extern "C" {

void rv9o_test_itx(const int32_t* coefs, int n, int tx_type, int lossless, int eob, int bit_depth, uint16_t* dst,
                   int stride) {
  oracle::inverse_transform_add(coefs, n, tx_type, lossless != 0, eob, bit_depth, dst, stride);
}

void rv9o_test_intra(int mode, int log2, const int32_t* above, const int32_t* left, int have_left, int have_above,
                     int bit_depth, uint16_t* dst, int stride) {
  oracle::intra_predict(mode, log2, above, left, have_left != 0, have_above != 0, bit_depth, dst, stride);
}

// Filters the line of 16 samples whose q0 is buf[8].
void rv9o_test_lf(uint16_t* buf, int filter_size, int limit, int blimit, int thresh, int bit_depth) {
  oracle::lf_filter(buf, 8, 1, filter_size, limit, blimit, thresh, bit_depth);
}

}  // extern "C"

// The oracle's loop filter over SB-aligned u16 planes, with the mode info of
// the given blocks.
extern "C" void rv9o_test_lf_frame(const rv9_frame_desc* d, const rv9_block* blocks, int n_blocks, uint16_t* y,
                                   uint16_t* u, uint16_t* v) {
  oracle::Picture pic;
  int w = d->sb64_cols * 64, h = d->sb64_rows * 64;
  uint16_t* src[3] = {y, u, v};
  for (int p = 0; p < 3; ++p) {
    int pw = p ? w >> d->ss_x : w, ph = p ? h >> d->ss_y : h;
    pic.planes[p].data.assign(src[p], src[p] + (size_t)pw * ph);
    pic.planes[p].stride = pw;
    pic.planes[p].height = ph;
  }
  oracle::FrameRecon fr(*d, pic);
  std::vector<oracle::MiLf> mi((size_t)d->mi_rows * d->mi_cols);
  for (int i = 0; i < n_blocks; ++i) {
    const rv9_block& b = blocks[i];
    oracle::MiLf m{b.mi_size, (uint8_t)((b.flags & RV9_BLK_SKIP) ? 1 : 0), b.tx_size, b.y_mode, b.segment_id,
                   b.ref_frame[0]};
    uint32_t bh = vp9t_num_8x8_high[b.mi_size], bw = vp9t_num_8x8_wide[b.mi_size];
    for (uint32_t yy = b.mi_row; yy < std::min(b.mi_row + bh, d->mi_rows); ++yy)
      for (uint32_t xx = b.mi_col; xx < std::min(b.mi_col + bw, d->mi_cols); ++xx) mi[(size_t)yy * d->mi_cols + xx] = m;
  }
  fr.filter_frame(mi);
  for (int p = 0; p < 3; ++p) std::copy(pic.planes[p].data.begin(), pic.planes[p].data.end(), src[p]);
}

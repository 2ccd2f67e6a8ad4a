// Per-sample arithmetic of VP9 reconstruction, written once for the CUDA
// kernels. Every function here is __host__ __device__ so that the same code
// can be compiled for the CPU and checked against the oracle without a GPU.
//
// - Inverse DCT / ADST / WHT (spec 8.7.1): the butterfly network with its
//   intermediate rounding, compile-time sized so that the index arithmetic and
//   the cosine constants fold away. Lanes: L32 (8 bits; 32-bit wrapping
//   arithmetic) and L64 (10/12 bits; 64-bit values whose multiplications take
//   the low 32 bits of the operand), matching the reference's S32 / S64
//   (rivet-vp9 src/dsp/itx.rs:574-666).
// - Intra predictors (spec 8.5.1.1) as closed forms: each sample computed
//   directly from the edge arrays, so a warp predicts a block in parallel; the
//   directional modes' copy recurrences (reference src/dsp/intra.rs:49-144)
//   are unrolled into an index into their first row or column.
// - Loop filter sample operations (spec 8.8.5; reference src/dsp/lf.rs:24-143)
//   on one line of 16 samples across an edge.
#pragma once
#include <stdint.h>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

#define RV9_HD __host__ __device__ __forceinline__

namespace rv9g {

// ---------------------------------------------------------------------------
// Transforms.

RV9_HD constexpr int32_t cos64(int angle) {
  // cos64_lookup (spec 8.7.1.1), folded by quadrant.
  constexpr int32_t C[33] = {16384, 16364, 16305, 16207, 16069, 15893, 15679, 15426, 15137, 14811, 14449,
                             14053, 13623, 13160, 12665, 12140, 11585, 11003, 10394, 9760,  9102,  8423,
                             7723,  7005,  6270,  5520,  4756,  3981,  3196,  2404,  1606,  804,   0};
  return (angle & 127) <= 32   ? C[angle & 127]
         : (angle & 127) <= 64 ? -C[64 - (angle & 127)]
         : (angle & 127) <= 96 ? -C[(angle & 127) - 64]
                               : C[128 - (angle & 127)];
}
RV9_HD constexpr int32_t sin64(int angle) { return cos64(angle - 32); }

RV9_HD constexpr int brev(int num_bits, int x) {
  int t = 0;
  for (int i = 0; i < num_bits; ++i) t |= ((x >> i) & 1) << (num_bits - 1 - i);
  return t;
}

struct L32 {
  typedef int32_t store_t;
  int32_t v;
  static RV9_HD L32 zero() { return L32{0}; }
  static RV9_HD L32 load(int32_t x) { return L32{x}; }
  RV9_HD L32 add(L32 o) const { return L32{(int32_t)((uint32_t)v + (uint32_t)o.v)}; }
  RV9_HD L32 sub(L32 o) const { return L32{(int32_t)((uint32_t)v - (uint32_t)o.v)}; }
  RV9_HD L32 mul(int32_t c) const { return L32{(int32_t)((uint32_t)v * (uint32_t)c)}; }
  RV9_HD L32 rshift(int n) const { return L32{(int32_t)((uint32_t)v + (1u << (n - 1))) >> n}; }
  RV9_HD L32 sar(int n) const { return L32{v >> n}; }
  // Residual clamped to +-2^16, as the reference's lanes clamp it.
  RV9_HD int32_t residual() const { return v < -(1 << 16) ? -(1 << 16) : (v > (1 << 16) ? (1 << 16) : v); }
};

struct L64 {
  typedef int64_t store_t;
  int64_t v;
  static RV9_HD L64 zero() { return L64{0}; }
  static RV9_HD L64 load(int64_t x) { return L64{x}; }
  RV9_HD L64 add(L64 o) const { return L64{(int64_t)((uint64_t)v + (uint64_t)o.v)}; }
  RV9_HD L64 sub(L64 o) const { return L64{(int64_t)((uint64_t)v - (uint64_t)o.v)}; }
  RV9_HD L64 mul(int32_t c) const { return L64{(int64_t)(int32_t)(uint32_t)(uint64_t)v * (int64_t)c}; }
  RV9_HD L64 rshift(int n) const { return L64{(int64_t)((uint64_t)v + (1ull << (n - 1))) >> n}; }
  RV9_HD L64 sar(int n) const { return L64{v >> n}; }
  RV9_HD int32_t residual() const {
    return (int32_t)(v < -(1 << 16) ? -(1 << 16) : (v > (1 << 16) ? (1 << 16) : v));
  }
};

template <class V>
RV9_HD V round14(V x) {
  return x.rshift(14);
}

template <class V>
RV9_HD void bfly(V* t, int a, int b, int angle, bool flip) {
  const int32_t c = cos64(angle), s = sin64(angle);
  V x = round14(t[a].mul(c).sub(t[b].mul(s)));
  V y = round14(t[a].mul(s).add(t[b].mul(c)));
  t[a] = flip ? y : x;
  t[b] = flip ? x : y;
}

template <class V>
RV9_HD void hada(V* t, int a, int b, bool flip) {
  int p = flip ? b : a, q = flip ? a : b;
  V x = t[p], y = t[q];
  t[p] = x.add(y);
  t[q] = x.sub(y);
}

template <class V>
RV9_HD void sbfly(const V* t, V* s, int a, int b, int angle, bool flip) {
  const int32_t c = cos64(angle), sn = sin64(angle);
  V x = t[a].mul(c).sub(t[b].mul(sn));
  V y = t[a].mul(sn).add(t[b].mul(c));
  s[a] = flip ? y : x;
  s[b] = flip ? x : y;
}

template <class V>
RV9_HD void shada(V* t, const V* s, int a, int b) {
  t[a] = round14(s[a].add(s[b]));
  t[b] = round14(s[a].sub(s[b]));
}

// The inverse DCT steps of size 2^n after the recursive call (spec 8.7.1.3).
template <int n, class V>
RV9_HD void idct_stage(V* t) {
  constexpr int n0 = 1 << n, n1 = n0 >> 1, n2 = n0 >> 2, n3 = n0 >> 3;
#pragma unroll
  for (int i = 0; i < n2; ++i) bfly(t, n1 + i, n0 - 1 - i, 32 - brev(5, n1 + i), false);
  if (n >= 3) {
#pragma unroll
    for (int i = 0; i < n3; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) hada(t, n1 + 4 * i + 2 * j, n1 + 1 + 4 * i + 2 * j, j == 1);
  }
  if (n == 5) {
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j)
        bfly(t, n0 - n + 3 - n2 * j - 4 * i, n1 + n - 4 + n2 * j + 4 * i, 28 - 16 * i + 56 * j, true);
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) hada(t, n1 + n3 * j + i, n1 + n2 - 5 + n3 * j - i, (j & 1) == 1);
  }
  if (n >= 4) {
    constexpr int imax = n == 5 ? 1 : 0;
#pragma unroll
    for (int i = 0; i <= imax; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) bfly(t, n0 - n + 2 - i - n2 * j, n1 + n - 3 + i + n2 * j, 24 + 48 * j, true);
#pragma unroll
    for (int i = 0; i < 2 * n - 6; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) hada(t, n1 + n2 * j + i, n1 + n2 - 1 + n2 * j - i, (j & 1) == 1);
  }
  if (n >= 3) {
#pragma unroll
    for (int i = 0; i < n3; ++i) bfly(t, n0 - n3 - 1 - i, n1 + n3 + i, 16, true);
  }
#pragma unroll
  for (int i = 0; i < n1; ++i) hada(t, i, n0 - 1 - i, false);
}

template <int n, class V>
RV9_HD void idct(V* t) {
  constexpr int n0 = 1 << n;
  V c[n0];
#pragma unroll
  for (int i = 0; i < n0; ++i) c[i] = t[i];
#pragma unroll
  for (int i = 0; i < n0; ++i) t[i] = c[brev(n, i)];
  bfly(t, 0, 1, 16, true);
  idct_stage<2>(t);
  if (n >= 3) idct_stage<(n >= 3 ? 3 : 2)>(t);
  if (n >= 4) idct_stage<(n >= 4 ? 4 : 2)>(t);
  if (n >= 5) idct_stage<(n >= 5 ? 5 : 2)>(t);
}

template <int n, class V>
RV9_HD void adst_in_perm(V* t) {
  constexpr int n0 = 1 << n, n1 = n0 >> 1;
  V c[n0];
#pragma unroll
  for (int i = 0; i < n0; ++i) c[i] = t[i];
#pragma unroll
  for (int i = 0; i < n1; ++i) {
    t[2 * i] = c[n0 - 1 - 2 * i];
    t[2 * i + 1] = c[2 * i];
  }
}

template <int n, class V>
RV9_HD void adst_out_perm(V* t) {
  constexpr int n0 = 1 << n;
  V c[n0];
#pragma unroll
  for (int i = 0; i < n0; ++i) c[i] = t[i];
  if (n == 4) {
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      int a = (q >> 3) & 1, b = (q >> 2) & 1, cc = (q >> 1) & 1, d = q & 1;
      t[q] = c[8 * (d ^ cc) + 4 * (cc ^ b) + 2 * (b ^ a) + a];
    }
  } else {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      int a = (q >> 2) & 1, b = (q >> 1) & 1, cc = q & 1;
      t[q] = c[4 * (cc ^ b) + 2 * (b ^ a) + a];
    }
  }
}

template <class V>
RV9_HD void iadst4(V* t) {
  V s0 = t[0].mul(5283), s1 = t[0].mul(9929), s2 = t[1].mul(13377);
  V s3 = t[2].mul(15212), s4 = t[2].mul(5283), s5 = t[3].mul(9929);
  V s6 = t[3].mul(15212);
  V v = t[0].sub(t[2]).add(t[3]);
  V s7 = v.mul(13377);
  V x0 = s0.add(s3).add(s5), x1 = s1.sub(s4).sub(s6), x2 = s7, x3 = s2;
  t[0] = round14(x0.add(x3));
  t[1] = round14(x1.add(x3));
  t[2] = round14(x2);
  t[3] = round14(x0.add(x1).sub(x3));
}

template <class V>
RV9_HD void iadst8(V* t) {
  V s[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) s[i] = V::zero();
  adst_in_perm<3>(t);
#pragma unroll
  for (int i = 0; i < 4; ++i) sbfly(t, s, 2 * i, 1 + 2 * i, 30 - 8 * i, true);
#pragma unroll
  for (int i = 0; i < 4; ++i) shada(t, s, i, 4 + i);
#pragma unroll
  for (int i = 0; i < 2; ++i) sbfly(t, s, 4 + 3 * i, 5 + i, 24 - 16 * i, true);
#pragma unroll
  for (int i = 0; i < 2; ++i) shada(t, s, 4 + i, 6 + i);
#pragma unroll
  for (int i = 0; i < 2; ++i) hada(t, i, 2 + i, false);
#pragma unroll
  for (int i = 0; i < 2; ++i) bfly(t, 2 + 4 * i, 3 + 4 * i, 16, true);
  adst_out_perm<3>(t);
#pragma unroll
  for (int i = 0; i < 4; ++i) t[1 + 2 * i] = V::zero().sub(t[1 + 2 * i]);
}

template <class V>
RV9_HD void iadst16(V* t) {
  V s[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) s[i] = V::zero();
  adst_in_perm<4>(t);
#pragma unroll
  for (int i = 0; i < 8; ++i) sbfly(t, s, 2 * i, 1 + 2 * i, 31 - 4 * i, true);
#pragma unroll
  for (int i = 0; i < 8; ++i) shada(t, s, i, 8 + i);
#pragma unroll
  for (int i = 0; i < 4; ++i) sbfly(t, s, 8 + 2 * i, 9 + 2 * i, 28 - 16 * i, true);
#pragma unroll
  for (int i = 0; i < 4; ++i) shada(t, s, 8 + i, 12 + i);
#pragma unroll
  for (int i = 0; i < 4; ++i) hada(t, i, 4 + i, false);
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) sbfly(t, s, 4 + 8 * i + 3 * j, 5 + 8 * i + j, 24 - 16 * j, true);
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) shada(t, s, 4 + 8 * j + i, 6 + 8 * j + i);
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) hada(t, 8 * j + i, 2 + 8 * j + i, false);
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) bfly(t, 2 + 4 * j + 8 * i, 3 + 4 * j + 8 * i, 48 + 64 * (i ^ j), false);
  adst_out_perm<4>(t);
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) t[1 + 12 * j + 2 * i] = V::zero().sub(t[1 + 12 * j + 2 * i]);
}

template <class V>
RV9_HD void iwht(V* t, int shift) {
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

// One 1D inverse transform of size 2^n: `kind` 0 DCT, 1 ADST, 2 WHT.
template <int n, class V>
RV9_HD void tx1d(V* t, int kind, int wht_shift) {
  if (kind == 2) {
    if (n == 2) iwht(t, wht_shift);
  } else if (kind == 0) {
    idct<n>(t);
  } else {
    if (n == 2) iadst4(t);
    if (n == 3) iadst8(t);
    if (n == 4) iadst16(t);
  }
}

// ---------------------------------------------------------------------------
// Intra prediction: sample (i, j) of a 2^log2 square block.
// `above[k + 1]` is aboveRow[k] for k in -1 .. 2*size-1; `left[k]` leftCol[k].
// `dc` is the DC_PRED value (computed once per block). Modes use the
// specification's numbering (DC 0, V 1, H 2, D45 3, D135 4, D117 5, D153 6,
// D207 7, D63 8, TM 9).

RV9_HD int32_t r2(int32_t x, int n) { return (x + (1 << (n - 1))) >> n; }

RV9_HD int32_t intra_pixel(int mode, int i, int j, int size, const int32_t* above, const int32_t* left,
                           int32_t dc, int32_t maxv) {
#define A(k) above[(k) + 1]
#define L(k) left[(k)]
  switch (mode) {
    case 1:  // V
      return A(j);
    case 2:  // H
      return L(i);
    case 3: {  // D45
      int k = i + j;
      return (i + j + 2 < size * 2) ? r2(A(k) + A(k + 1) * 2 + A(k + 2), 2) : A(2 * size - 1);
    }
    case 4: {  // D135: dst[i][j] = dst[i-1][j-1]
      int k = i < j ? i : j;
      int ii = i - k, jj = j - k;
      if (ii == 0) return jj == 0 ? r2(L(0) + 2 * A(-1) + A(0), 2) : r2(A(jj - 2) + 2 * A(jj - 1) + A(jj), 2);
      return ii == 1 ? r2(A(-1) + 2 * L(0) + L(1), 2) : r2(L(ii - 2) + 2 * L(ii - 1) + L(ii), 2);
    }
    case 5: {  // D117: dst[i][j] = dst[i-2][j-1]
      int k = (i >> 1) < j ? (i >> 1) : j;
      int ii = i - 2 * k, jj = j - k;
      if (ii == 0) return r2(A(jj - 1) + A(jj), 1);
      if (ii == 1) return jj == 0 ? r2(L(0) + 2 * A(-1) + A(0), 2) : r2(A(jj - 2) + 2 * A(jj - 1) + A(jj), 2);
      return ii == 2 ? r2(A(-1) + 2 * L(0) + L(1), 2) : r2(L(ii - 3) + 2 * L(ii - 2) + L(ii - 1), 2);
    }
    case 6: {  // D153: dst[i][j] = dst[i-1][j-2]
      int k = i < (j >> 1) ? i : (j >> 1);
      int ii = i - k, jj = j - 2 * k;
      if (jj == 0) return ii == 0 ? r2(L(0) + A(-1), 1) : r2(L(ii - 1) + L(ii), 1);
      if (jj == 1) {
        if (ii == 0) return r2(L(0) + 2 * A(-1) + A(0), 2);
        if (ii == 1) return r2(A(-1) + 2 * L(0) + L(1), 2);
        return r2(L(ii - 2) + 2 * L(ii - 1) + L(ii), 2);
      }
      return r2(A(jj - 3) + 2 * A(jj - 2) + A(jj - 1), 2);
    }
    case 7: {  // D207: dst[i][j] = dst[i+1][j-2]; the last row is leftCol[size-1]
      int ii = i + (j >> 1);
      if (ii >= size - 1) return L(size - 1);
      if ((j & 1) == 0) return r2(L(ii) + L(ii + 1), 1);
      if (ii < size - 2) return r2(L(ii) + 2 * L(ii + 1) + L(ii + 2), 2);
      return r2(L(size - 2) + 3 * L(size - 1), 2);
    }
    case 8: {  // D63
      int k = (i >> 1) + j;
      return (i & 1) ? r2(A(k) + A(k + 1) * 2 + A(k + 2), 2) : r2(A(k) + A(k + 1), 1);
    }
    case 9: {  // TM
      int32_t v = A(j) + L(i) - A(-1);
      return v < 0 ? 0 : (v > maxv ? maxv : v);
    }
    default:
      return dc;
  }
#undef A
#undef L
}

// DC_PRED's value (reference src/dsp/intra.rs:153-174) from the edge sums.
RV9_HD int32_t intra_dc(int log2, int32_t sum_above, int32_t sum_left, bool have_left, bool have_above,
                        int bit_depth) {
  int size = 1 << log2;
  if (have_left && have_above) return (sum_above + sum_left + size) >> (log2 + 1);
  if (have_left) return (sum_left + (1 << (log2 - 1))) >> log2;
  if (have_above) return (sum_above + (1 << (log2 - 1))) >> log2;
  return 1 << (bit_depth - 1);
}

// ---------------------------------------------------------------------------
// Loop filter on one line across an edge: s[0..15] are the samples at
// offsets -8..7 from the edge (s[8] is q0). Returns nothing; modifies s.

RV9_HD int iabs(int v) { return v < 0 ? -v : v; }
RV9_HD int iclamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// The wide filter (spec 8.8.5.3): a rounded sliding mean over 2^log2 taps of
// the samples at -(n+1) .. n (n = 2^(log2-1) - 1), replacing -n .. n-1. All
// indices are compile-time constants so the line stays in registers.
// Index t of the wide filter's window, clamped to its ends p(n)..q(n)
// (relative to the edge at 8).
RV9_HD constexpr int lfw_at(int t, int n) { return (t < -(n + 1) ? -(n + 1) : (t > n ? n : t)) + 8; }

// The 8- and 16-wide filters (spec 8.8.5.3): each output is the rounded mean
// of the sample itself and the 2n+1 samples centred on it, the window's ends
// repeated. The window sum is carried from one output to the next.
template <int LOG2>
RV9_HD void lf_wide(int* s) {
  constexpr int n = (1 << (LOG2 - 1)) - 1;
  int w = 0;
#pragma unroll
  for (int j = -n; j <= n; ++j) w += s[lfw_at(-n + j, n)];
  int f[16];
#pragma unroll
  for (int i = -n; i < n; ++i) {
    f[i + 8] = (s[i + 8] + w + (1 << (LOG2 - 1))) >> LOG2;
    w += s[lfw_at(i + n + 1, n)] - s[lfw_at(i - n, n)];
  }
#pragma unroll
  for (int i = -n; i < n; ++i) s[i + 8] = f[i + 8];
}

RV9_HD int imax(int a, int b) { return a > b ? a : b; }

RV9_HD void lf_line(int* s, int filter_size, int limit, int blimit, int thresh, int bd) {
  const int q0 = s[8], q1 = s[9], q2 = s[10], q3 = s[11];
  const int p0 = s[7], p1 = s[6], p2 = s[5], p3 = s[4];
  const int sh = bd - 8;
  const int ap1 = iabs(p1 - p0), aq1 = iabs(q1 - q0);
  // filterMask: every step within limit, the edge within blimit.
  const int m = imax(imax(imax(iabs(p3 - p2), iabs(p2 - p1)), imax(ap1, aq1)), imax(iabs(q2 - q1), iabs(q3 - q2)));
  if (m > (limit << sh) || iabs(p0 - q0) * 2 + (iabs(p1 - q1) >> 1) > (blimit << sh)) return;
  const int thresh_bd = thresh << sh;
  const bool hev = ap1 > thresh_bd || aq1 > thresh_bd;
  const int one = 1 << sh;
  const bool flat = filter_size >= 1 && imax(imax(ap1, aq1), imax(imax(iabs(p2 - p0), iabs(q2 - q0)),
                                                                  imax(iabs(p3 - p0), iabs(q3 - q0)))) <= one;
  if (!flat) {
    // Narrow filter (spec 8.8.5.2).
    const int lo = -(1 << (bd - 1)), hi = (1 << (bd - 1)) - 1;
    const int off = 0x80 << sh;
    const int ps1 = p1 - off, ps0 = p0 - off, qs0 = q0 - off, qs1 = q1 - off;
    int f = hev ? iclamp(ps1 - qs1, lo, hi) : 0;
    f = iclamp(f + 3 * (qs0 - ps0), lo, hi);
    const int f1 = iclamp(f + 4, lo, hi) >> 3, f2 = iclamp(f + 3, lo, hi) >> 3;
    s[8] = iclamp(qs0 - f1, lo, hi) + off;
    s[7] = iclamp(ps0 + f2, lo, hi) + off;
    if (!hev) {
      const int g = (f1 + 1) >> 1;
      s[9] = iclamp(qs1 - g, lo, hi) + off;
      s[6] = iclamp(ps1 + g, lo, hi) + off;
    }
    return;
  }
  bool flat2 = filter_size >= 2;
  if (flat2) {
    int m2 = 0;
#pragma unroll
    for (int k = 4; k < 8; ++k) m2 = imax(m2, imax(iabs(s[8 - k - 1] - p0), iabs(s[8 + k] - q0)));
    flat2 = m2 <= one;
  }
  if (!flat2)
    lf_wide<3>(s);
  else
    lf_wide<4>(s);
}

// ---------------------------------------------------------------------------
// Loop filter edge decisions (reference superblock(),
// src/decoder/loopfilter.rs:466-620), one (edge, run) entry at a time.

// Per 8x8 loop-filter record: bits 0-5 level, 6-7 luma tx size, 8-9 chroma tx
// size, 10-13 block size, 14 coded (intra, or not skipped).
RV9_HD uint32_t lf_pack(int level, int tx_y, int tx_uv, int mi_size, bool coded) {
  return (uint32_t)level | ((uint32_t)tx_y << 6) | ((uint32_t)tx_uv << 8) | ((uint32_t)mi_size << 10) |
         ((coded ? 1u : 0u) << 14);
}

struct LfParams {
  int mi_cols, mi_rows, ss_x, ss_y;
  const uint32_t* lf_mi;
  const uint8_t* limit;   // [64] by level
  const uint8_t* blimit;
  const uint8_t* thresh;
};

struct LfEdge {
  int8_t fs;
  uint8_t limit, blimit, thresh;
};

RV9_HD void lf_at(int pass, int sub_x, int sub_y, int row, int col, int e, int r, int* x, int* y) {
  if (pass == 0) {
    *x = col * 8 + e * (4 << sub_x);
    *y = row * 8 + ((4 * r) << sub_y);
  } else {
    *x = col * 8 + ((4 * r) << sub_x);
    *y = row * 8 + e * (4 << sub_y);
  }
}

// Where the per-8x8 loop-filter records come from: the frame's array, or a
// superblock's 8x8 of them staged in shared memory.
struct LfMiFrame {
  const uint32_t* p;
  int stride;
  RV9_HD uint32_t operator()(int r, int c) const { return p[(size_t)r * stride + c]; }
};
struct LfMiTile {
  const uint32_t* t;  // 8 x 8, row-major
  int row0, col0;
  RV9_HD uint32_t operator()(int r, int c) const { return t[(r - row0) * 8 + (c - col0)]; }
};

// The filter of edge `ed`, run `rn` of pass `pass` (0 vertical, 1 horizontal)
// of plane `plane` in the superblock at mode-info (row, col).
template <class MiAt>
RV9_HD LfEdge lf_edge_entry_at(const LfParams& k, const MiAt& mi_at, int plane, int pass, int row, int col, int ed,
                               int rn) {
  LfEdge e{-1, 0, 0, 0};
  const int sub_x = plane ? k.ss_x : 0, sub_y = plane ? k.ss_y : 0;
  const int sub = pass == 0 ? sub_x : sub_y;
  int ca = ed >> 1, cb = rn >> 1;
  int x, y;
  lf_at(pass, sub_x, sub_y, row, col, 2 * ca, 2 * cb, &x, &y);
  if (x >= 8 * k.mi_cols || y >= 8 * k.mi_rows) return e;
  int loop_col = ((x >> 3) >> sub_x) << sub_x;
  int loop_row = ((y >> 3) >> sub_y) << sub_y;
  uint32_t m = mi_at(loop_row, loop_col);
  int l = m & 63;
  if (l == 0) return e;
  int tx_sz = plane ? ((m >> 8) & 3) : ((m >> 6) & 3);
  int mi_size = (m >> 10) & 15;
  bool coded = (m >> 14) & 1;
  // num_8x8 wide / high by block size, as 2-bit fields of a constant.
  int w8 = 1 << ((0x3ea5400u >> (2 * mi_size)) & 3);
  int h8 = 1 << ((0x3b99100u >> (2 * mi_size)) & 3);
  int sb_size = sub == 0 ? mi_size : (mi_size > 6 ? mi_size : 6);
  if (sb_size != mi_size) {
    w8 = 1 << ((0x3ea5400u >> (2 * sb_size)) & 3);
    h8 = 1 << ((0x3b99100u >> (2 * sb_size)) & 3);
  }
  int block_mask = pass == 0 ? 8 * w8 - 1 : 8 * h8 - 1;
  lf_at(pass, sub_x, sub_y, row, col, ed, 2 * cb, &x, &y);
  if ((pass == 0 && x == 0) || (pass == 1 && y == 0)) return e;
  int across = pass == 0 ? x : y;
  bool is_block_edge = (across & block_mask) == 0;
  bool tx_edge = (ed & ((1 << tx_sz) - 1)) == 0;
  if (!is_block_edge && !(tx_edge && coded)) return e;
  bool is_32_edge = ed % 8 == 0;
  int base_size = (tx_sz == 0 && is_32_edge) ? 1 : (tx_sz < 2 ? tx_sz : 2);
  int filter_size = base_size;
  if ((pass == 0 && sub_x == 1 && base_size == 2 && (x >> 3) == k.mi_cols - 1) ||
      (pass == 1 && sub_y == 1 && base_size == 2 && (y >> 3) == k.mi_rows - 1))
    filter_size = 1;
  lf_at(pass, sub_x, sub_y, row, col, ed, rn, &x, &y);
  if ((rn & 1) && (x >= 8 * k.mi_cols || y >= 8 * k.mi_rows)) return e;
  bool is_tx_edge = tx_edge;
  if (pass == 1 && sub_x == 1 && (k.mi_cols & 1) && (ed & 1) && (x + 8) >= k.mi_cols * 8) is_tx_edge = false;
  if (!(is_block_edge || (is_tx_edge && coded))) return e;
  e.fs = (int8_t)filter_size;
  e.limit = k.limit[l];
  e.blimit = k.blimit[l];
  e.thresh = k.thresh[l];
  return e;
}

RV9_HD LfEdge lf_edge_entry(const LfParams& k, int plane, int pass, int row, int col, int ed, int rn) {
  return lf_edge_entry_at(k, LfMiFrame{k.lf_mi, k.mi_cols}, plane, pass, row, col, ed, rn);
}

// The loop-filter record of a block (the MiInfo fields the filter reads).
// `lvl` is LvlLookup[segment][ref][mode type] (8.8.1).
RV9_HD uint32_t lf_block_record(int mi_size, int tx_size, int flags, int segment_id, int y_mode, int ref0,
                                const uint8_t (*lvl)[4][2], int legacy_uv, int ss_x, int ss_y) {
  int mode_type = (y_mode == 10 || y_mode == 11 || y_mode == 13) ? 1 : 0;  // NEARESTMV, NEARMV, NEWMV
  int rf = ref0 > 0 ? ref0 : 0;
  int level = lvl[segment_id][rf][mode_type];
  int uv_tx = 0;
  if (mi_size >= 3) {
    // get_uv_tx_size: the chroma block's largest transform, with 4:2:0's
    // subsampling for a pre-final profile 1 stream.
    int ux = legacy_uv ? 1 : ss_x, uy = legacy_uv ? 1 : ss_y;
    // Chroma block width / height log2 in 4-sample units.
    int bw = ((0x3ea5400u >> (2 * mi_size)) & 3) + 1 - ux;  // log2(8x8 units) + 1 = log2(4x4 units)
    int bh = ((0x3b99100u >> (2 * mi_size)) & 3) + 1 - uy;
    int m = bw < bh ? bw : bh;  // largest square transform inside: log2 in 4-sample units
    if (m > 3) m = 3;
    uv_tx = tx_size < m ? tx_size : m;
  }
  bool coded = ref0 <= 0 || !(flags & 1);
  return lf_pack(level, tx_size, uv_tx, mi_size, coded);
}

// Vertical edges of one sample row of a superblock, left to right. `line`
// holds the row from 8 samples left of the superblock; `e` the plane's
// vertical-pass entries [edge][run].
RV9_HD void lf_vertical_row(int16_t* line, const LfEdge (*e)[16], int n_edges, int run, int bd) {
  for (int ed = 0; ed < n_edges; ++ed) {
    LfEdge f = e[ed][run];
    if (f.fs < 0) continue;
    int16_t* w = line + 4 * ed;
    int s[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) s[q] = w[q];
    lf_line(s, f.fs, f.limit, f.blimit, f.thresh, bd);
#pragma unroll
    for (int q = 1; q < 15; ++q) w[q] = (int16_t)s[q];
  }
}

// Horizontal edges of one sample column, top to bottom. `col` points at the
// column's sample 8 rows above the superblock; `pitch` is the row pitch;
// `rows` the rows available from there.
RV9_HD void lf_horizontal_col(int16_t* col, int pitch, int rows, const LfEdge (*e)[16], int n_edges, int run,
                              int bd) {
  for (int ed = 0; ed < n_edges; ++ed) {
    LfEdge f = e[ed][run];
    if (f.fs < 0) continue;
    int16_t* w = col + 4 * ed * pitch;
    const int avail = rows - 4 * ed;
    int s[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) s[q] = q < avail ? w[q * pitch] : 0;
    lf_line(s, f.fs, f.limit, f.blimit, f.thresh, bd);
#pragma unroll
    for (int q = 1; q < 15; ++q)
      if (q < avail) w[q * pitch] = (int16_t)s[q];
  }
}

}  // namespace rv9g

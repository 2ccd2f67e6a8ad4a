// MD5 (RFC 1321), for host and device: the digest of a decoded frame's packed
// planes (the bytes of the reference's Frame::packed(), whose per-frame MD5s
// are what the reference's tests compare, tests/common/mod.rs:151), computed
// where the frame is.
//
// The sine table is the RFC's definition, T[i] = floor(2^32 |sin(i + 1)|) for
// i = 0..63; md5_sine_table computes it on the host, and the caller hands it
// to md5_block (the device copy lives in constant memory). The four rounds'
// functions, message orders and rotations are the RFC's.
#pragma once
#include <math.h>
#include <stdint.h>

#ifdef __CUDACC__
#define RV9_MD5 __host__ __device__ __forceinline__
#else
#define RV9_MD5 static inline
#endif

namespace rv9g {

struct Md5State {
  uint32_t a, b, c, d;
};

static inline void md5_sine_table(uint32_t* t) {
  for (int i = 0; i < 64; ++i) t[i] = (uint32_t)floor(fabs(sin((double)(i + 1))) * 4294967296.0);
}

RV9_MD5 void md5_init(Md5State* h) {
  h->a = 0x67452301u;
  h->b = 0xefcdab89u;
  h->c = 0x98badcfeu;
  h->d = 0x10325476u;
}

RV9_MD5 uint32_t md5_rotl(uint32_t x, int s) { return (x << s) | (x >> (32 - s)); }

// The rotation of step i (RFC 1321 section 3.4: four per round).
RV9_MD5 int md5_shift(int i) {
  const int r = i >> 4, j = i & 3;
  if (r == 0) return j == 0 ? 7 : j == 1 ? 12 : j == 2 ? 17 : 22;
  if (r == 1) return j == 0 ? 5 : j == 1 ? 9 : j == 2 ? 14 : 20;
  if (r == 2) return j == 0 ? 4 : j == 1 ? 11 : j == 2 ? 16 : 23;
  return j == 0 ? 6 : j == 1 ? 10 : j == 2 ? 15 : 21;
}

// One 64-byte block, as 16 little-endian words.
RV9_MD5 void md5_block(Md5State* h, const uint32_t* w, const uint32_t* t) {
  uint32_t a = h->a, b = h->b, c = h->c, d = h->d;
#ifdef __CUDACC__
#pragma unroll
#endif
  for (int i = 0; i < 64; ++i) {
    uint32_t f;
    int g;
    if (i < 16) {
      f = (b & c) | (~b & d);
      g = i;
    } else if (i < 32) {
      f = (d & b) | (~d & c);
      g = (5 * i + 1) & 15;
    } else if (i < 48) {
      f = b ^ c ^ d;
      g = (3 * i + 5) & 15;
    } else {
      f = c ^ (b | ~d);
      g = (7 * i) & 15;
    }
    const uint32_t e = d;
    d = c;
    c = b;
    b = b + md5_rotl(a + f + t[i] + w[g], md5_shift(i));
    a = e;
  }
  h->a += a;
  h->b += b;
  h->c += c;
  h->d += d;
}

// Byte k of the padded message of `len` bytes whose bytes below len come
// from `data_byte` (RFC 1321 sections 3.1-3.2: 0x80, zeros, then the bit
// length, little-endian, in the last 8 bytes of the final block).
RV9_MD5 uint64_t md5_padded_bytes(uint64_t len) { return ((len + 8) / 64 + 1) * 64; }
RV9_MD5 uint8_t md5_pad_byte(uint64_t k, uint64_t len) {
  const uint64_t total = md5_padded_bytes(len);
  if (k == len) return 0x80;
  if (k >= total - 8) return (uint8_t)((len * 8) >> (8 * (k - (total - 8))));
  return 0;
}

// The 16-byte digest of the final state.
RV9_MD5 void md5_digest(const Md5State& h, uint8_t* out) {
  const uint32_t v[4] = {h.a, h.b, h.c, h.d};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) out[4 * i + j] = (uint8_t)(v[i] >> (8 * j));
}

}  // namespace rv9g

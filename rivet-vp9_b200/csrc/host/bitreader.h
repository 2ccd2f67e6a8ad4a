// Bit readers of the VP9 syntax: the plain f(n)/s(n) reader of the
// uncompressed header (spec 4.9, 9.1; reference src/bits.rs:13-90) and the
// boolean arithmetic decoder of spec 9.2 (reference src/bool_coder.rs:12-126).
#pragma once
#include <stddef.h>
#include <stdint.h>
#include <string.h>

namespace rv9 {

struct HeaderError {
  const char* msg;
};

// f(n) / s(n) reader, most significant bit first. Reading past the end throws
// HeaderError (the uncompressed header is cut short).
class BitReader {
 public:
  BitReader(const uint8_t* d, size_t n) : data_(d), len_(n), pos_(0) {}
  uint32_t bit() {
    size_t byte = pos_ >> 3;
    if (byte >= len_) throw HeaderError{"uncompressed header runs past the end of the frame"};
    uint32_t b = (data_[byte] >> (7 - (pos_ & 7))) & 1;
    ++pos_;
    return b;
  }
  uint32_t f(int n) {
    uint32_t x = 0;
    for (int i = 0; i < n; ++i) x = (x << 1) | bit();
    return x;
  }
  bool flag() { return bit() != 0; }
  int32_t s(int n) {
    int32_t v = (int32_t)f(n);
    return flag() ? -v : v;
  }
  void byte_align() { pos_ = (pos_ + 7) & ~(size_t)7; }
  size_t position() const { return pos_; }

 private:
  const uint8_t* data_;
  size_t len_;
  size_t pos_;
};

// Boolean decoder. `value` holds the decoder's current byte (BoolValue of the
// specification) in bits 63..56 followed by stream bits not yet consumed;
// `bits` counts the valid bits from bit 63 down. Bits past the end of the
// data read as zero.
class BoolDecoder {
 public:
  BoolDecoder() = default;
  // init_bool(sz). Returns false if the data is empty or the marker bit is 1.
  bool init(const uint8_t* d, size_t n) {
    p_ = d;
    end_ = d + n;
    start_ = d;
    value_ = 0;
    bits_ = 0;
    range_ = 255;
    if (n == 0) return false;
    fill();
    return !read(128);
  }

  // The decoder's state as plain values. Hot loops keep a copy in locals
  // (registers), so that their stores to byte arrays, which may alias
  // anything, do not force the state back to memory on every read.
  struct State {
    uint64_t value;
    uint32_t range;
    int bits;
    const uint8_t* p;
    const uint8_t* end;
  };
  State save() const { return State{value_, range_, bits_, p_, end_}; }
  void load(const State& s) {
    value_ = s.value;
    range_ = s.range;
    bits_ = s.bits;
    p_ = s.p;
  }

  static inline bool read(State& s, int prob) {
    uint32_t split = 1 + (((s.range - 1) * (uint32_t)prob) >> 8);
    uint64_t big = (uint64_t)split << 56;
    // Branch-free: the decoded bit is data, not control flow.
    const bool bit = s.value >= big;
    const uint64_t m = 0 - (uint64_t)bit;
    s.range = bit ? s.range - split : split;
    s.value -= big & m;
    int shift = __builtin_clz(s.range) - 24;
    s.range <<= shift;
    s.value <<= shift;
    s.bits -= shift;
    if (s.bits < 16) fill(s);
    return bit;
  }

  inline bool read(int prob) {
    State s = save();
    bool b = read(s, prob);
    load(s);
    return b;
  }

  uint32_t literal(int n) {
    uint32_t x = 0;
    for (int i = 0; i < n; ++i) x = (x << 1) | (uint32_t)read(128);
    return x;
  }

  // Tree decode (spec 9.3.3): `probs(node)` gives the probability of node
  // index n >> 1.
  template <class P>
  inline int tree(const int8_t* t, P probs) {
    int n = 0;
    do {
      n = t[n + (int)read(probs(n >> 1))];
    } while (n > 0);
    return -n;
  }

  // Whether the bits not yet read (the padding, spec 9.2.3) are all zero.
  bool padding_is_zero() const {
    if (value_ & ((1ull << 56) - 1)) return false;
    for (const uint8_t* q = p_; q < end_; ++q)
      if (*q) return false;
    return true;
  }

 private:
  static inline void fill(State& s) {
    if (s.end - s.p >= 8) {
      // Whole bytes that fit below the valid bits, from one big-endian load.
      // The part of the next byte that also lands is ORed in again, at the
      // same position, by the next fill.
      uint64_t w;
      memcpy(&w, s.p, 8);
      w = __builtin_bswap64(w);
      const int nbytes = (64 - s.bits) >> 3;
      s.value |= w >> s.bits;
      s.p += nbytes;
      s.bits += nbytes * 8;
      return;
    }
    while (s.bits <= 56) {
      if (s.p < s.end) {
        s.value |= (uint64_t)(*s.p++) << (56 - s.bits);
        s.bits += 8;
      } else {
        s.bits = 64;  // zeros from here on
        break;
      }
    }
  }
  inline void fill() {
    State s = save();
    fill(s);
    load(s);
  }
  const uint8_t* p_ = nullptr;
  const uint8_t* end_ = nullptr;
  const uint8_t* start_ = nullptr;
  uint64_t value_ = 0;
  int bits_ = 0;
  uint32_t range_ = 255;
};

}  // namespace rv9

// The tile, partition and block syntax of VP9 (spec 6.4) as a device parser:
// one thread decodes one tile column of one frame (its tile rows in turn),
// many columns of many frames at once. It writes the same records
// (rv9_records.h) as the host parser, byte for byte: a restatement of the
// decode direction of the host's tile syntax, which itself restates the
// reference decoder's parse (src/decoder/block.rs:368-1715, the bool decoder
// of src/bool_coder.rs:12-126, motion vector prediction of
// src/decoder/mvpred.rs).
//
// The code is plain C++ with __host__ __device__ qualifiers, so the same
// functions also run on the CPU, where a test holds their records to the host
// parser's on every test stream.
//
// What differs from the host parser is the form, for one GPU thread:
//   * a 64-bit arithmetic-decoder window (two 32-bit words), refilled 32
//     bits at a time (the decoded values do not depend on the window's width);
//   * the token cache and the coefficient probabilities in shared memory,
//     the probabilities of the current band in registers;
//   * the left contexts as 16-entry windows of the current superblock row
//     (they are cleared at each superblock row and never read outside it);
//   * tables in one device-resident struct (Tables), the scan position, the
//     two context neighbours and the band of a scan index in one 8-byte entry;
//   * errors as codes (the host's messages by code), outputs into buffers
//     sized for the worst case of the tile column, and no symbol counts: a
//     frame parses here only when nothing adapts from its counts.
#pragma once
#include <stdint.h>
#include <string.h>

#include "../../../include/rv9_records.h"
#include "../host/probs.h"

#if defined(__CUDACC__)
#define TP_HD __host__ __device__
#define TP_INL __host__ __device__ __forceinline__
#define TP_NOINL __host__ __device__ __noinline__
#else
#define TP_HD
#define TP_INL inline
#define TP_NOINL __attribute__((noinline))
#endif

namespace rv9g {
namespace tp {

#if !defined(__CUDACC__)
struct uint2 {
  uint32_t x, y;
};
#endif

enum Error : int32_t {
  TP_OK = 0,
  TP_EMPTY_TILE = 1,    // boolean-coded partition of size 0
  TP_MARKER = 2,        // boolean decoder marker bit is not 0
  TP_PARTITION = 3,     // invalid partition
  TP_CHROMA_BLOCK = 4,  // block size invalid for the chroma subsampling
  TP_CHROMA_SIZE = 5,   // invalid chroma block size
  TP_REF_SCALE = 6,     // reference frame scaled beyond 2:1 / 1:16
  TP_OVERFLOW = 7,      // an output ran past its capacity
};

// The host parser's message for each code.
inline const char* error_message(int32_t e) {
  switch (e) {
    case TP_EMPTY_TILE: return "boolean-coded partition of size 0";
    case TP_MARKER: return "boolean decoder marker bit is not 0";
    case TP_PARTITION: return "invalid partition";
    case TP_CHROMA_BLOCK: return "block size invalid for the chroma subsampling";
    case TP_CHROMA_SIZE: return "invalid chroma block size";
    case TP_REF_SCALE: return "reference frame scaled beyond 2:1 / 1:16";
    case TP_OVERFLOW: return "device parser output capacity exceeded";
    default: return "bitstream error";
  }
}

struct Mv {
  int32_t r, c;
};
TP_INL bool mv_eq(const Mv& a, const Mv& b) { return a.r == b.r && a.c == b.c; }

// Mode info per 8x8 position (the host parser's MiInfo, same layout).
struct Mi {
  uint8_t mi_size;
  uint8_t skip;
  uint8_t tx_size;
  uint8_t y_mode;
  uint8_t sub_modes[4];
  uint8_t segment_id;
  int8_t ref_frame[2];
  uint8_t interp_filter;
  Mv mv[2][4];
};

// The previous frame's motion vectors per 8x8 position (PrevMvs and
// PrevRefFrames of spec 8.10; the host parser's PrevMv, same layout).
struct PrevMv {
  int8_t ref_frame[2];
  Mv mv[2];
};

// One scan index of a transform size and scan order: the coefficient's
// position, the two positions whose token energies give its context (spec
// 6.4.24's above and left; reference block.rs:1656-1699) and its band.
struct alignas(8) ScanEnt {
  uint16_t pos, nb0, nb1;
  uint8_t band, pad;
};

// Every table the tile syntax reads, in one struct (uploaded once per
// device). Filled on the host from the specification tables.
struct Tables {
  ScanEnt scan[4][3][1024];  // [tx size][0 default, 1 DCT_ADST (column), 2 ADST_DCT (row)][scan index]
  uint8_t pareto[256][8];    // token-tree nodes 2..9 given node 1's probability
  uint8_t energy[12];
  uint8_t kf_partition[16][3];
  uint8_t kf_y_mode[10][10][9];
  uint8_t kf_uv_mode[10][9];
  int8_t mv_ref_blocks[13][8][2];
  uint8_t mode_2_counter[14];
  uint8_t idx_n_col_to_sub[4][2];
  uint8_t b_wl2[13], b_hl2[13], n4w[13], n4h[13], mi_wl2[13], n8w[13], n8h[13], size_group[13];
  uint8_t subsize[4][13];
  uint8_t ss_size[13][2][2];
  uint8_t max_tx[13];
  uint8_t tx_mode_biggest[5];
  uint8_t mode2txfm[14];
  uint8_t counter_to_ctx[19];
  int16_t extra_bits[11][3];
  uint8_t cat_probs[7][14];
  int8_t partition_tree[6], intra_mode_tree[18], tx32_tree[6], tx16_tree[4], tx8_tree[2];
  int8_t inter_mode_tree[6], interp_tree[4], mv_joint_tree[6], mv_class_tree[20], mv_fr_tree[6], token_tree[20];
};

// What the tile syntax reads of one frame's headers.
struct FrameIn {
  uint32_t mi_cols, mi_rows, sb64_cols, sb64_rows;
  uint8_t ss_x, ss_y, bit_depth, frame_is_intra;
  uint8_t tx_mode, reference_mode, interp_filter, allow_hp;
  int8_t comp_fixed_ref;
  int8_t comp_var_ref[2];
  uint8_t sign_bias[4];
  uint8_t lossless, legacy_uv, tile_cols_log2, tile_rows_log2;
  uint8_t ref_ok[3];
  uint8_t use_prev;  // motion vector candidates from the previous frame
  rv9::Probs probs;
  // The coefficient probabilities repacked: word k of a band holds node k's
  // probability for context c in byte c.
  uint64_t coef_pk[4][2][2][6][3];
};

// One tile of a column: its bytes and rows.
struct Span {
  uint64_t off;  // into the batch's packet bytes
  uint32_t size;
  uint32_t mi_row_start, mi_row_end;
  uint32_t index;  // the tile's number in bitstream order (row * columns + column)
};

// One tile column of one frame: the unit of work of one thread.
struct Chain {
  uint32_t frame;               // into the batch's FrameIn array
  uint32_t first_span, n_spans;
  uint32_t mi_col_start, mi_col_end;
  // Outputs: element offsets into the batch's record arrays, and capacities.
  uint64_t blocks_at, toks_at, coefs_at;
  uint32_t blocks_cap, toks_cap, coefs_cap;
  // Per-frame working memory: mode info (mi_rows x mi_cols) and the above
  // contexts, element offsets into the batch's arrays.
  uint64_t mi_at, above_at;
  uint64_t prev_at;  // the previous frame's PrevMv array (when use_prev)
};

struct ChainOut {
  uint32_t n_blocks, n_toks, n_coefs;
  int32_t err;         // Error
  uint32_t err_tile;   // the failing tile's number (when err)
  uint32_t bools;      // boolean decodes (for the throughput figure)
  uint32_t pad[2];
};

// Above contexts of a frame: per plane sb64_cols * 16 + 16 nonzero flags,
// then sb64_cols * 8 + 8 partition contexts.
TP_INL uint64_t above_bytes(uint32_t sb64_cols) { return 3ull * (sb64_cols * 16 + 16) + (sb64_cols * 8 + 8); }

// Worst-case outputs of a tile column mi_w x mi_h (8x8 units), over its
// superblocks (a transform block that starts inside the frame may reach past
// it, up to its superblock's edge): a block per 8x8, a transform block per
// 4x4 of each plane, a coefficient per sample.
TP_INL void chain_caps(uint32_t mi_w, uint32_t mi_h, uint32_t ss_x, uint32_t ss_y, uint32_t* blocks, uint32_t* toks,
                       uint32_t* coefs) {
  const uint64_t w4 = (uint64_t)((mi_w + 7) & ~7u) * 2, h4 = (uint64_t)((mi_h + 7) & ~7u) * 2;
  const uint64_t luma4 = w4 * h4, chroma4 = (w4 >> ss_x) * (h4 >> ss_y);
  *blocks = mi_w * mi_h;
  *toks = (uint32_t)(luma4 + 2 * chroma4);
  *coefs = (uint32_t)(16 * (luma4 + 2 * chroma4));
}


TP_INL int clz32(uint32_t x) {
#if defined(__CUDA_ARCH__)
  return __clz((int)x);
#else
  return __builtin_clz(x);
#endif
}

// Device intrinsics with their host equivalents.
// The top 32 bits of (hi:lo) << s, 0 <= s < 32.
TP_INL uint32_t funnel_l(uint32_t lo, uint32_t hi, int s) {
#if defined(__CUDA_ARCH__)
  return __funnelshift_l(lo, hi, s);
#else
  return s ? (hi << s) | (lo >> (32 - s)) : hi;
#endif
}
// Byte i of the result is byte (s >> 4i) & 7 of (y:x) (selector values 0-7).
TP_INL uint32_t byte_perm(uint32_t x, uint32_t y, uint32_t s) {
#if defined(__CUDA_ARCH__)
  return __byte_perm(x, y, s);
#else
  const uint64_t v = ((uint64_t)y << 32) | x;
  uint32_t r = 0;
  for (int i = 0; i < 4; ++i) r |= (uint32_t)((v >> (8 * ((s >> (4 * i)) & 7))) & 0xff) << (8 * i);
  return r;
#endif
}
// Read-only loads through the non-coherent cache on the device.
template <class T>
TP_INL T ro(const T* p) {
#if defined(__CUDA_ARCH__)
  return __ldg(p);
#else
  return *p;
#endif
}
// Four bytes at p, big-endian, when p + 4 <= the end of the data. On the
// device, from the two aligned words around them (the buffer holding the
// tile data has 16 bytes of padding past its end).
TP_INL uint32_t load_be32(const uint8_t* p) {
#if defined(__CUDA_ARCH__)
  const uint32_t a = (uint32_t)((uintptr_t)p & 3);
  const uint32_t* q = (const uint32_t*)(p - a);
  return __byte_perm(__ldg(q), __ldg(q + 1), 0x0123u + a * 0x1111u);
#else
  return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
#endif
}

// The parse kernel's shared memory (one tile column per CTA): the token
// cache and the frame's coefficient probabilities as 32-bit words. Declared
// here so that the parser's accesses are shared-memory accesses, which the
// compiler keeps apart from its global stores; the CPU build uses the
// TileParser's own arrays.
#if defined(__CUDACC__)
__shared__ uint8_t tp_tc_smem[1024];
__shared__ uint32_t tp_pkw_smem[576];
#endif
#if defined(__CUDA_ARCH__)
#define TP_TC(i) tp_tc_smem[i]
#define TP_PKW(i) tp_pkw_smem[i]
#else
#define TP_TC(i) tc[i]
#define TP_PKW(i) pkw[i]
#endif

// A scan entry in one 8-byte load.
TP_INL ScanEnt ld_scan(const ScanEnt* p) {
#if defined(__CUDA_ARCH__)
  const uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
  ScanEnt e;
  e.pos = (uint16_t)(v.x & 0xffff);
  e.nb0 = (uint16_t)(v.x >> 16);
  e.nb1 = (uint16_t)(v.y & 0xffff);
  e.band = (uint8_t)((v.y >> 16) & 0xff);
  e.pad = 0;
  return e;
#else
  return *p;
#endif
}

// The boolean decoder (spec 9.2). The window hi:lo holds the decoder's
// current byte in hi's bits 31..24 followed by stream bits not yet consumed;
// `bits` counts its valid bits from the top (24 or more between decodes, so
// that a decode, which shifts out at most 7, always compares 8 valid bits),
// and bits below them are zero. Stream bits are appended 32 at a time; bits
// past the end of the data read as zero.
struct Bool {
  uint32_t hi, lo, range;
  int bits;
  const uint8_t* p;
  const uint8_t* end;
  uint32_t count;

  // The last bytes of the data (fewer than 4), then zeros: out of line, so
  // that the decodes inlined everywhere stay small. Takes and returns values
  // only, so that the window stays in registers.
  static TP_NOINL uint32_t tail_word(const uint8_t* p, const uint8_t* end) {
    uint32_t w = 0;
    for (int k = 0; k < 4; ++k) w = (w << 8) | (p + k < end ? p[k] : 0u);
    return w;
  }
  // Appends 32 stream bits; bits <= 32.
  TP_INL void refill() {
    uint32_t w;
    if (end - p >= 4) {
      w = load_be32(p);
      p += 4;
    } else {
      w = tail_word(p, end);
      p = end;
    }
    if (bits < 32) hi |= w >> bits;
    lo = bits ? w << (32 - bits) : 0;
    bits += 32;
  }
  // init_bool(sz): false if the marker bit is 1.
  TP_INL bool init(const uint8_t* d, uint32_t n) {
    p = d;
    end = d + n;
    hi = lo = 0;
    bits = 0;
    range = 255;
    count = 0;
    refill();
    return !read(128);
  }
  TP_INL bool read(uint32_t prob) {
    const uint32_t split = 1 + (((range - 1) * prob) >> 8);
    const uint32_t big = split << 24;
    const bool bit = hi >= big;
    range = bit ? range - split : split;
    hi = bit ? hi - big : hi;
    const int shift = clz32(range) - 24;
    range <<= shift;
    hi = funnel_l(lo, hi, shift);
    lo <<= shift;
    bits -= shift;
    if (bits < 24) refill();
    ++count;
    return bit;
  }
  // Tree decode (spec 9.3.3): node n's probability is p[n >> 1].
  TP_INL int tree(const int8_t* t, const uint8_t* pr) {
    int n = 0;
    do {
      n = t[n + (int)read(pr[n >> 1])];
    } while (n > 0);
    return -n;
  }
};

// The state of the block being decoded (reference src/decoder/block.rs:51-76).
struct Blk {
  uint32_t mi_row, mi_col;
  uint8_t mi_size;
  bool avail_u, avail_l;
  bool skip;
  uint8_t tx_size;
  bool is_inter;
  uint8_t y_mode;
  uint8_t sub_modes[4];
  uint8_t uv_mode;
  int8_t ref_frame[2];
  uint8_t interp_filter;
  uint8_t mode_context[4];
  const Mi* above;
  const Mi* left;
  Mv block_mvs[2][4];
  Mv nearest_mv[2], near_mv[2], best_mv[2], mv[2];
};

// Motion vector candidate search state (spec 6.5.1).
struct Search {
  int count;
  Mv list[2];
  Mv cand_mv[2];
  int8_t cand_frame[2];
  TP_INL void add(int ref_list) {
    if (count >= 2) return;
    if (count > 0 && mv_eq(cand_mv[ref_list], list[0])) return;
    list[count++] = cand_mv[ref_list];
  }
};

TP_INL bool use_mv_hp(const Mv& mv) {
  const int32_t ar = mv.r < 0 ? -mv.r : mv.r, ac = mv.c < 0 ? -mv.c : mv.c;
  return (ar >> 3) < 8 && (ac >> 3) < 8;  // COMPANDED_MVREF_THRESH
}


// One tile column's syntax (the decode direction of the host parser's
// TileCoder).
struct TileParser {
  const Tables* T;
  const FrameIn* F;
  Mi* mi;  // the frame's mode info
  uint8_t* above_nz[3];
  uint8_t* above_part;
  const PrevMv* prev;  // null unless the frame uses the previous frame's vectors
  rv9_block* blocks;
  rv9_tok* toks;
  uint32_t* coefs;
  uint32_t n_blocks, n_toks, n_coefs, cap_blocks, cap_toks, cap_coefs;
  // Token cache (1024 entries) and the frame's coefficient probabilities as
  // 32-bit words: node k of band b of a (tx size, plane type, reference
  // type) at 36 * index + 6 b + 2 k (low word: contexts 0-3, high word: 4-5),
  // FrameIn::coef_pk. On the device both are the kernel's shared arrays
  // (TP_TC, TP_PKW).
  uint8_t* tc;
  const uint32_t* pkw;
  uint8_t left_nz[3][16];
  uint8_t left_part[8];
  uint32_t mi_row_start, mi_row_end, mi_col_start, mi_col_end;
  uint32_t mi_cols, mi_rows, ss_x, ss_y;
  int32_t err;
  uint32_t eob_total;
  Bool bd;
  Blk b;

  TP_INL Mi& mi_at(uint32_t r, uint32_t c) const { return mi[(size_t)r * mi_cols + c]; }
  TP_INL void fail(int32_t e) {
    if (!err) err = e;
  }

  // decode_tile (spec 6.4.2): the tile's superblocks in raster order.
  TP_HD void decode_tile() {
    for (uint32_t r = mi_row_start; r < mi_row_end && !err; r += 8) {
      memset(left_nz, 0, sizeof left_nz);
      memset(left_part, 0, sizeof left_part);
      for (uint32_t c = mi_col_start; c < mi_col_end && !err; c += 8) decode_superblock(r, c);
    }
  }

  // decode_partition (spec 6.4.3) from a superblock down, without recursion:
  // a split pushes its four quarters (the first on top) and has nothing left
  // to do after them, so an explicit stack visits the regions in the
  // recursion's order.
  TP_HD void decode_superblock(uint32_t r0, uint32_t c0) {
    uint32_t st_r[16], st_c[16];
    uint8_t st_b[16];
    int top = 0;
    st_r[0] = r0;
    st_c[0] = c0;
    st_b[0] = 12;  // BLOCK_64X64
    top = 1;
    while (top > 0 && !err) {
      --top;
      const uint32_t r = st_r[top], c = st_c[top];
      const uint8_t bsize = st_b[top];
      if (r >= mi_rows || c >= mi_cols) continue;
      const uint32_t num8x8 = T->n8w[bsize];
      const uint32_t half = num8x8 >> 1;
      const bool has_rows = (r + half) < mi_rows;
      const bool has_cols = (c + half) < mi_cols;
      const uint32_t bsl = T->mi_wl2[bsize];
      const uint32_t boffset = T->mi_wl2[12] - bsl;
      uint8_t above = 0, left = 0;
      for (uint32_t i = 0; i < num8x8; ++i) {
        above |= above_part[c + i];
        left |= left_part[(r + i) & 7];
      }
      const bool a = (above & (1 << boffset)) != 0;
      const bool l = (left & (1 << boffset)) != 0;
      const int ctx = (int)(bsl * 4 + (l ? 2 : 0) + (a ? 1 : 0));
      const uint8_t* probs = F->frame_is_intra ? T->kf_partition[ctx] : F->probs.partition[ctx];
      int partition;
      if (has_rows && has_cols)
        partition = bd.tree(T->partition_tree, probs);
      else if (has_cols)
        partition = bd.read(probs[1]) ? 3 /* SPLIT */ : 1 /* HORZ */;
      else if (has_rows)
        partition = bd.read(probs[2]) ? 3 : 2 /* VERT */;
      else
        partition = 3;
      const uint8_t subsize = T->subsize[partition][bsize];
      if (subsize == 14 /* BLOCK_INVALID */) {
        fail(TP_PARTITION);
        return;
      }
      if (subsize >= 3 /* BLOCK_8X8 */ && partition == 3) {
        // The quarters, the first one on top.
        st_r[top] = r + half; st_c[top] = c + half; st_b[top++] = subsize;
        st_r[top] = r + half; st_c[top] = c;        st_b[top++] = subsize;
        st_r[top] = r;        st_c[top] = c + half; st_b[top++] = subsize;
        st_r[top] = r;        st_c[top] = c;        st_b[top++] = subsize;
        continue;
      }
      if (subsize < 3 || partition == 0) {
        decode_block(r, c, subsize);
      } else if (partition == 1) {
        decode_block(r, c, subsize);
        if (has_rows) decode_block(r + half, c, subsize);
      } else {
        decode_block(r, c, subsize);
        if (has_cols) decode_block(r, c + half, subsize);
      }
      if (err) return;
      const uint8_t av = (uint8_t)(15 >> T->b_wl2[subsize]);
      const uint8_t lv = (uint8_t)(15 >> T->b_hl2[subsize]);
      for (uint32_t i = 0; i < num8x8; ++i) {
        above_part[c + i] = av;
        left_part[(r + i) & 7] = lv;
      }
    }
  }

  // One block: its mode info with the decoder's state in registers (the
  // mode-info functions are inlined here, and the block is decoded out of
  // line once rather than inlined at each of its callers), then its
  // residual and records.
  TP_NOINL void decode_block(uint32_t r, uint32_t c, uint8_t subsize) {
    if (err) return;
    if (ss_x + ss_y > 0 && subsize >= 3 && T->ss_size[subsize][ss_x][ss_y] == 14) {
      fail(TP_CHROMA_BLOCK);
      return;
    }
    memset(&b, 0, sizeof b);
    b.mi_row = r;
    b.mi_col = c;
    b.mi_size = subsize;
    b.avail_u = r > 0;
    b.avail_l = c > mi_col_start;
    b.above = b.avail_u ? &mi_at(r - 1, c) : nullptr;
    b.left = b.avail_l ? &mi_at(r, c - 1) : nullptr;
    b.ref_frame[0] = 0;   // INTRA_FRAME
    b.ref_frame[1] = -1;  // NONE
    {
      Bool rb = bd;
      if (F->frame_is_intra)
        intra_frame_mode_info(rb);
      else
        inter_frame_mode_info(rb);
      bd = rb;
    }
    eob_total = 0;
    if (n_blocks >= cap_blocks) {
      fail(TP_OVERFLOW);
      return;
    }
    const uint32_t bi = n_blocks++;
    const uint32_t tok0 = n_toks;
    const bool coded_skip = b.skip;
    residual();
    if (err) return;
    if (b.is_inter && subsize >= 3 && eob_total == 0) b.skip = true;
    rv9_block rb;
    rb.mi_row = (uint16_t)r;
    rb.mi_col = (uint16_t)c;
    rb.mi_size = subsize;
    rb.flags = (uint8_t)((b.skip ? RV9_BLK_SKIP : 0) | (b.is_inter ? RV9_BLK_INTER : 0) |
                         (b.avail_l ? RV9_BLK_AVAIL_L : 0) | (b.avail_u ? RV9_BLK_AVAIL_U : 0));
    rb.tx_size = b.tx_size;
    rb.segment_id = 0;
    rb.y_mode = b.y_mode;
    rb.uv_mode = b.uv_mode;
    rb.interp_filter = b.interp_filter;
    rb.coded_skip = coded_skip ? 1 : 0;
    for (int k = 0; k < 4; ++k) rb.sub_modes[k] = b.sub_modes[k];
    rb.ref_frame[0] = b.ref_frame[0];
    rb.ref_frame[1] = b.ref_frame[1];
    rb.n_tok = (uint16_t)(n_toks - tok0);
    rb.tok_start = tok0;
    for (int l = 0; l < 2; ++l)
      for (int k = 0; k < 4; ++k) {
        rb.mv[l][k][0] = b.block_mvs[l][k].r;
        rb.mv[l][k][1] = b.block_mvs[l][k].c;
      }
    blocks[bi] = rb;
    Mi info;
    info.mi_size = subsize;
    info.skip = b.skip;
    info.tx_size = b.tx_size;
    info.y_mode = b.y_mode;
    for (int k = 0; k < 4; ++k) info.sub_modes[k] = b.sub_modes[k];
    info.segment_id = 0;
    info.ref_frame[0] = b.ref_frame[0];
    info.ref_frame[1] = b.ref_frame[1];
    info.interp_filter = b.interp_filter;
    for (int l = 0; l < 2; ++l)
      for (int k = 0; k < 4; ++k) info.mv[l][k] = b.block_mvs[l][k];
    const uint32_t bh = T->n8h[subsize], bw = T->n8w[subsize];
    const uint32_t ye = r + bh < mi_rows ? r + bh : mi_rows, xe = c + bw < mi_cols ? c + bw : mi_cols;
    for (uint32_t y = r; y < ye; ++y)
      for (uint32_t x = c; x < xe; ++x) mi_at(y, x) = info;
  }

  // ---- Mode info (spec 6.4.5 - 6.4.17) ----

  TP_INL void intra_frame_mode_info(Bool& r) {
    read_skip(r);
    read_tx_size(r, true);
    b.ref_frame[0] = 0;
    b.ref_frame[1] = -1;
    b.is_inter = false;
    if (b.mi_size >= 3) {
      const uint8_t am = b.above ? b.above->sub_modes[2] : 0;
      const uint8_t lm = b.left ? b.left->sub_modes[1] : 0;
      const uint8_t mode = (uint8_t)r.tree(T->intra_mode_tree, T->kf_y_mode[am][lm]);
      b.y_mode = mode;
      for (int i = 0; i < 4; ++i) b.sub_modes[i] = mode;
    } else {
      const int n4w = T->n4w[b.mi_size], n4h = T->n4h[b.mi_size];
      uint8_t mode = 0;
      for (int idy = 0; idy < 2; idy += n4h)
        for (int idx = 0; idx < 2; idx += n4w) {
          const uint8_t am = idy > 0 ? b.sub_modes[idx] : (b.above ? b.above->sub_modes[2 + idx] : 0);
          const uint8_t lm = idx > 0 ? b.sub_modes[idy * 2] : (b.left ? b.left->sub_modes[1 + idy * 2] : 0);
          mode = (uint8_t)r.tree(T->intra_mode_tree, T->kf_y_mode[am][lm]);
          for (int y2 = 0; y2 < n4h; ++y2)
            for (int x2 = 0; x2 < n4w; ++x2) b.sub_modes[(idy + y2) * 2 + idx + x2] = mode;
        }
      b.y_mode = mode;
    }
    b.uv_mode = (uint8_t)r.tree(T->intra_mode_tree, T->kf_uv_mode[b.y_mode]);
  }

  TP_INL void read_skip(Bool& r) {
    const int ctx = (b.above ? b.above->skip : 0) + (b.left ? b.left->skip : 0);
    b.skip = r.read(F->probs.skip[ctx]);
  }

  TP_INL void read_tx_size(Bool& r, bool allow_select) {
    const uint8_t max_tx = T->max_tx[b.mi_size];
    if (allow_select && F->tx_mode == 4 /* TX_MODE_SELECT */ && b.mi_size >= 3) {
      uint8_t above = max_tx, left = max_tx;
      if (b.above && !b.above->skip) above = b.above->tx_size;
      if (b.left && !b.left->skip) left = b.left->tx_size;
      if (!b.avail_l) left = above;
      if (!b.avail_u) above = left;
      const int ctx = (above + left) > max_tx ? 1 : 0;
      const int8_t* tree = max_tx == 3 ? T->tx32_tree : max_tx == 2 ? T->tx16_tree : T->tx8_tree;
      b.tx_size = (uint8_t)r.tree(tree, F->probs.tx[max_tx][ctx]);
    } else {
      const uint8_t m = T->tx_mode_biggest[F->tx_mode];
      b.tx_size = max_tx < m ? max_tx : m;
    }
  }

  TP_INL void inter_frame_mode_info(Bool& r) {
    read_skip(r);
    read_is_inter(r);
    read_tx_size(r, !b.skip || !b.is_inter);
    if (b.is_inter)
      inter_block_mode_info(r);
    else
      intra_block_mode_info(r);
  }

  TP_INL void left_ref(int8_t out[2]) const {
    out[0] = b.left ? b.left->ref_frame[0] : 0;
    out[1] = b.left ? b.left->ref_frame[1] : -1;
  }
  TP_INL void above_ref(int8_t out[2]) const {
    out[0] = b.above ? b.above->ref_frame[0] : 0;
    out[1] = b.above ? b.above->ref_frame[1] : -1;
  }

  TP_INL void read_is_inter(Bool& r) {
    int8_t l[2], a[2];
    left_ref(l);
    above_ref(a);
    const bool left_intra = l[0] <= 0, above_intra = a[0] <= 0;
    const bool au = b.avail_u, al = b.avail_l;
    int ctx;
    if (au && al)
      ctx = (left_intra && above_intra) ? 3 : (left_intra || above_intra) ? 1 : 0;
    else if (au || al)
      ctx = 2 * (au ? above_intra : left_intra);
    else
      ctx = 0;
    b.is_inter = r.read(F->probs.is_inter[ctx]);
  }

  TP_INL void intra_block_mode_info(Bool& r) {
    b.ref_frame[0] = 0;
    b.ref_frame[1] = -1;
    if (b.mi_size >= 3) {
      const uint8_t mode = (uint8_t)r.tree(T->intra_mode_tree, F->probs.y_mode[T->size_group[b.mi_size]]);
      b.y_mode = mode;
      for (int i = 0; i < 4; ++i) b.sub_modes[i] = mode;
    } else {
      const int n4w = T->n4w[b.mi_size], n4h = T->n4h[b.mi_size];
      uint8_t mode = 0;
      for (int idy = 0; idy < 2; idy += n4h)
        for (int idx = 0; idx < 2; idx += n4w) {
          mode = (uint8_t)r.tree(T->intra_mode_tree, F->probs.y_mode[0]);
          for (int y2 = 0; y2 < n4h; ++y2)
            for (int x2 = 0; x2 < n4w; ++x2) b.sub_modes[(idy + y2) * 2 + idx + x2] = mode;
        }
      b.y_mode = mode;
    }
    b.uv_mode = (uint8_t)r.tree(T->intra_mode_tree, F->probs.uv_mode[b.y_mode]);
  }

  TP_INL void inter_block_mode_info(Bool& r) {
    read_ref_frames(r);
    for (int j = 0; j < 2; ++j)
      if (b.ref_frame[j] > 0) find_best_ref_mvs(j);
    const bool is_compound = b.ref_frame[1] > 0;
    if (b.mi_size >= 3) b.y_mode = (uint8_t)(10 /* NEARESTMV */ + read_inter_mode(r));
    if (F->interp_filter == 4 /* SWITCHABLE */) {
      int8_t l[2], a[2];
      left_ref(l);
      above_ref(a);
      const int left_interp = (b.avail_l && l[0] > 0) ? b.left->interp_filter : 3;
      const int above_interp = (b.avail_u && a[0] > 0) ? b.above->interp_filter : 3;
      int ctx;
      if (left_interp == above_interp)
        ctx = left_interp;
      else if (left_interp == 3 && above_interp != 3)
        ctx = above_interp;
      else if (left_interp != 3 && above_interp == 3)
        ctx = left_interp;
      else
        ctx = 3;
      b.interp_filter = (uint8_t)r.tree(T->interp_tree, F->probs.interp_filter[ctx]);
    } else {
      b.interp_filter = F->interp_filter;
    }
    const int nrefs = 1 + (is_compound ? 1 : 0);
    if (b.mi_size < 3) {
      const int n4w = T->n4w[b.mi_size], n4h = T->n4h[b.mi_size];
      for (int idy = 0; idy < 2; idy += n4h)
        for (int idx = 0; idx < 2; idx += n4w) {
          b.y_mode = (uint8_t)(10 + read_inter_mode(r));
          if (b.y_mode == 10 || b.y_mode == 11 /* NEARMV */)
            for (int j = 0; j < nrefs; ++j) append_sub8x8_mvs(idy * 2 + idx, j);
          assign_mv(r, is_compound);
          for (int y2 = 0; y2 < n4h; ++y2)
            for (int x2 = 0; x2 < n4w; ++x2) {
              const int blk = (idy + y2) * 2 + idx + x2;
              for (int rl = 0; rl < nrefs; ++rl) b.block_mvs[rl][blk] = b.mv[rl];
            }
        }
    } else {
      assign_mv(r, is_compound);
      for (int rl = 0; rl < nrefs; ++rl)
        for (int k = 0; k < 4; ++k) b.block_mvs[rl][k] = b.mv[rl];
    }
  }

  TP_INL int read_inter_mode(Bool& r) {
    return r.tree(T->inter_mode_tree, F->probs.inter_mode[b.mode_context[b.ref_frame[0]]]);
  }

  TP_INL void read_ref_frames(Bool& r) {
    int comp_mode;
    if (F->reference_mode == 2 /* REFERENCE_MODE_SELECT */)
      comp_mode = r.read(F->probs.comp_mode[comp_mode_ctx()]) ? 1 : 0;
    else
      comp_mode = F->reference_mode;
    if (comp_mode == 1 /* COMPOUND_REFERENCE */) {
      const int idx = F->sign_bias[F->comp_fixed_ref] ? 1 : 0;
      const bool v = r.read(F->probs.comp_ref[comp_ref_ctx()]);
      b.ref_frame[idx] = F->comp_fixed_ref;
      b.ref_frame[1 - idx] = F->comp_var_ref[v ? 1 : 0];
    } else {
      const bool p1 = r.read(F->probs.single_ref[single_ref_p1_ctx()][0]);
      if (p1) {
        const bool p2 = r.read(F->probs.single_ref[single_ref_p2_ctx()][1]);
        b.ref_frame[0] = p2 ? 3 : 2;
      } else {
        b.ref_frame[0] = 1;
      }
      b.ref_frame[1] = -1;
    }
  }

  TP_HD int comp_mode_ctx() const {
    const bool au = b.avail_u, al = b.avail_l;
    int8_t a[2], l[2];
    above_ref(a);
    left_ref(l);
    const bool a_single = a[1] <= -1, l_single = l[1] <= -1;
    const bool a_intra = a[0] <= 0, l_intra = l[0] <= 0;
    const int8_t fixed = F->comp_fixed_ref;
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

  TP_HD int comp_ref_ctx() const {
    const bool au = b.avail_u, al = b.avail_l;
    int8_t a[2], l[2];
    above_ref(a);
    left_ref(l);
    const bool a_single = a[1] <= -1, l_single = l[1] <= -1;
    const bool a_intra = a[0] <= 0, l_intra = l[0] <= 0;
    const int fix_ref_idx = F->sign_bias[F->comp_fixed_ref] ? 1 : 0;
    const int var_ref_idx = 1 - fix_ref_idx;
    const int8_t var1 = F->comp_var_ref[1], var0 = F->comp_var_ref[0], fixed = F->comp_fixed_ref;
    if (au && al) {
      if (a_intra && l_intra) return 2;
      if (l_intra) return a_single ? 1 + 2 * (a[0] != var1) : 1 + 2 * (a[var_ref_idx] != var1);
      if (a_intra) return l_single ? 1 + 2 * (l[0] != var1) : 1 + 2 * (l[var_ref_idx] != var1);
      const int8_t vrfa = a_single ? a[0] : a[var_ref_idx];
      const int8_t vrfl = l_single ? l[0] : l[var_ref_idx];
      if (vrfa == vrfl && var1 == vrfa) return 0;
      if (l_single && a_single) {
        if ((vrfa == fixed && vrfl == var0) || (vrfl == fixed && vrfa == var0)) return 4;
        if (vrfa == vrfl) return 3;
        return 1;
      }
      if (l_single || a_single) {
        const int8_t vrfc = l_single ? vrfa : vrfl;
        const int8_t rfs = a_single ? vrfa : vrfl;
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

  TP_HD int single_ref_p1_ctx() const {
    const bool au = b.avail_u, al = b.avail_l;
    int8_t a[2], l[2];
    above_ref(a);
    left_ref(l);
    const bool a_single = a[1] <= -1, l_single = l[1] <= -1;
    const bool a_intra = a[0] <= 0, l_intra = l[0] <= 0;
    const int8_t LF = 1;
    if (au && al) {
      if (a_intra && l_intra) return 2;
      if (l_intra) return a_single ? 4 * (a[0] == LF) : 1 + (a[0] == LF || a[1] == LF);
      if (a_intra) return l_single ? 4 * (l[0] == LF) : 1 + (l[0] == LF || l[1] == LF);
      if (a_single && l_single) return 2 * (a[0] == LF) + 2 * (l[0] == LF);
      if (!a_single && !l_single) return 1 + (a[0] == LF || a[1] == LF || l[0] == LF || l[1] == LF);
      const int8_t rfs = a_single ? a[0] : l[0];
      const int8_t crf1 = a_single ? l[0] : a[0];
      const int8_t crf2 = a_single ? l[1] : a[1];
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

  TP_HD int single_ref_p2_ctx() const {
    const bool au = b.avail_u, al = b.avail_l;
    int8_t a[2], l[2];
    above_ref(a);
    left_ref(l);
    const bool a_single = a[1] <= -1, l_single = l[1] <= -1;
    const bool a_intra = a[0] <= 0, l_intra = l[0] <= 0;
    const int8_t LF = 1, GF = 2, AF = 3;
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
      const int8_t rfs = a_single ? a[0] : l[0];
      const int8_t crf1 = a_single ? l[0] : a[0];
      const int8_t crf2 = a_single ? l[1] : a[1];
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

  TP_INL void assign_mv(Bool& r, bool is_compound) {
    b.mv[1] = Mv{0, 0};
    for (int i = 0; i < 1 + (is_compound ? 1 : 0); ++i) {
      switch (b.y_mode) {
        case 13 /* NEWMV */: b.mv[i] = read_mv(r, i); break;
        case 10: b.mv[i] = b.nearest_mv[i]; break;
        case 11: b.mv[i] = b.near_mv[i]; break;
        default: b.mv[i] = Mv{0, 0}; break;
      }
    }
  }

  TP_INL Mv read_mv(Bool& r, int rl) {
    const Mv best = b.best_mv[rl];
    const bool use_hp = F->allow_hp && use_mv_hp(best);
    int32_t diff[2] = {0, 0};
    const int joint = r.tree(T->mv_joint_tree, F->probs.mv_joint);
    if (joint == 2 /* HZVNZ */ || joint == 3 /* HNZVNZ */) diff[0] = read_mv_component(r, 0, use_hp);
    if (joint == 1 /* HNZVZ */ || joint == 3) diff[1] = read_mv_component(r, 1, use_hp);
    return Mv{best.r + diff[0], best.c + diff[1]};
  }

  TP_INL int32_t read_mv_component(Bool& r, int comp, bool use_hp) {
    const rv9::Probs& pr = F->probs;
    const bool sign = r.read(pr.mv_sign[comp]);
    const int cls = r.tree(T->mv_class_tree, pr.mv_class[comp]);
    int32_t mag;
    if (cls == 0) {
      const int c0 = r.read(pr.mv_class0_bit[comp]) ? 1 : 0;
      const int fr = r.tree(T->mv_fr_tree, pr.mv_class0_fr[comp][c0]);
      const int hp = use_hp ? (r.read(pr.mv_class0_hp[comp]) ? 1 : 0) : 1;
      mag = ((c0 << 3) | (fr << 1) | hp) + 1;
    } else {
      int32_t dd = 0;
      for (int i = 0; i < cls; ++i) dd |= (r.read(pr.mv_bits[comp][i]) ? 1 : 0) << i;
      const int32_t m0 = 2 << (cls + 2);
      const int fr = r.tree(T->mv_fr_tree, pr.mv_fr[comp]);
      const int hp = use_hp ? (r.read(pr.mv_hp[comp]) ? 1 : 0) : 1;
      mag = m0 + ((dd << 3) | (fr << 1) | hp) + 1;
    }
    return sign ? -mag : mag;
  }

  // ---- Motion vector prediction (spec 6.5; reference mvpred.rs) ----

  TP_INL bool is_inside(int32_t r, int32_t c) const {
    return r >= 0 && r < (int32_t)mi_rows && c >= (int32_t)mi_col_start && c < (int32_t)mi_col_end;
  }

  TP_INL void scale_mv(Search& s, int ref_list, int8_t ref_frame) const {
    const int8_t cand = s.cand_frame[ref_list];
    if (F->sign_bias[cand] != F->sign_bias[ref_frame]) {
      s.cand_mv[ref_list].r *= -1;
      s.cand_mv[ref_list].c *= -1;
    }
  }

  TP_INL int32_t clamp_mv_row(int32_t v, int32_t border) const {
    const int32_t bh = T->n8h[b.mi_size];
    const int32_t mi_row = (int32_t)b.mi_row;
    const int32_t to_top = -((mi_row * 8) * 8);
    const int32_t to_bottom = (((int32_t)mi_rows - bh - mi_row) * 8) * 8;
    const int32_t lo = to_top - border, hi = to_bottom + border;
    return v < lo ? lo : (v > hi ? hi : v);
  }

  TP_INL int32_t clamp_mv_col(int32_t v, int32_t border) const {
    const int32_t bw = T->n8w[b.mi_size];
    const int32_t mi_col = (int32_t)b.mi_col;
    const int32_t to_left = -((mi_col * 8) * 8);
    const int32_t to_right = (((int32_t)mi_cols - bw - mi_col) * 8) * 8;
    const int32_t lo = to_left - border, hi = to_right + border;
    return v < lo ? lo : (v > hi ? hi : v);
  }

  // The candidate searches of find_mv_refs on values already loaded: a
  // candidate's two reference frames and the motion vectors it offers.
  TP_INL static void same_add(Search& s, const int8_t rf[2], const Mv mv[2], int8_t ref_frame) {
    for (int j = 0; j < 2; ++j) {
      s.cand_mv[j] = mv[j];
      s.cand_frame[j] = rf[j];
      if (rf[j] == ref_frame) {
        s.add(j);
        return;
      }
    }
  }
  TP_INL void diff_add(Search& s, const int8_t rf[2], const Mv mv[2], int8_t ref_frame) const {
    s.cand_mv[0] = mv[0];
    s.cand_mv[1] = mv[1];
    s.cand_frame[0] = rf[0];
    s.cand_frame[1] = rf[1];
    const bool mvs_same = mv_eq(s.cand_mv[0], s.cand_mv[1]);
    if (s.cand_frame[0] > 0 && s.cand_frame[0] != ref_frame) {
      scale_mv(s, 0, ref_frame);
      s.add(0);
    }
    if (s.cand_frame[1] > 0 && s.cand_frame[1] != ref_frame && !mvs_same) {
      scale_mv(s, 1, ref_frame);
      s.add(1);
    }
  }

  // find_mv_refs( refFrame, block ) (spec 6.5.1). The eight neighbours' mode
  // info is loaded first, all loads at once (it sits in L2, written by this
  // thread earlier), then searched in the specification's order.
  TP_HD void find_mv_refs(int8_t ref_frame, int block, Mv out[2]) {
    Search s;
    s.count = 0;
    s.list[0] = s.list[1] = Mv{0, 0};
    s.cand_mv[0] = s.cand_mv[1] = Mv{0, 0};
    s.cand_frame[0] = s.cand_frame[1] = 0;
    const int8_t(*search)[2] = T->mv_ref_blocks[b.mi_size];
    const int32_t mi_row = (int32_t)b.mi_row, mi_col = (int32_t)b.mi_col;
    bool in[8];
    int8_t rf[8][2];
    Mv mv3[8][2];    // the neighbour's vectors of its last 4x4 (sub-block 3)
    Mv first[2][2];  // the first two neighbours' vectors of the sub-block next to `block`
    uint8_t ym[2];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int32_t r = mi_row + search[i][0], c = mi_col + search[i][1];
      in[i] = is_inside(r, c);
      rf[i][0] = rf[i][1] = 0;
      mv3[i][0] = mv3[i][1] = Mv{0, 0};
      if (in[i]) {
        const Mi& m = mi_at(r, c);
        rf[i][0] = m.ref_frame[0];
        rf[i][1] = m.ref_frame[1];
        mv3[i][0] = m.mv[0][3];
        mv3[i][1] = m.mv[1][3];
        if (i < 2) {
          ym[i] = m.y_mode;
          const int idx = block >= 0 ? T->idx_n_col_to_sub[block][search[i][1] == 0 ? 1 : 0] : 3;
          first[i][0] = m.mv[0][idx];
          first[i][1] = m.mv[1][idx];
        }
      }
    }
    int context_counter = 0;
    for (int i = 0; i < 2; ++i) {
      if (!in[i]) continue;
      context_counter += T->mode_2_counter[ym[i]];
      for (int j = 0; j < 2; ++j) {
        if (rf[i][j] == ref_frame) {
          s.cand_mv[j] = first[i][j];
          s.add(j);
          break;
        }
      }
    }
    for (int i = 2; i < 8; ++i)
      if (in[i]) same_add(s, rf[i], mv3[i], ref_frame);
    const bool use_prev = prev != nullptr;
    int8_t prf[2] = {0, 0};
    Mv pmv[2] = {{0, 0}, {0, 0}};
    if (use_prev) {
      const PrevMv& pv = prev[(size_t)mi_row * mi_cols + mi_col];
      prf[0] = pv.ref_frame[0];
      prf[1] = pv.ref_frame[1];
      pmv[0] = pv.mv[0];
      pmv[1] = pv.mv[1];
      same_add(s, prf, pmv, ref_frame);
    }
    for (int i = 0; i < 8; ++i)
      if (in[i]) diff_add(s, rf[i], mv3[i], ref_frame);
    if (use_prev) diff_add(s, prf, pmv, ref_frame);
    b.mode_context[ref_frame] = T->counter_to_ctx[context_counter];
    for (int i = 0; i < 2; ++i) {
      s.list[i].r = clamp_mv_row(s.list[i].r, 128 /* MV_BORDER */);
      s.list[i].c = clamp_mv_col(s.list[i].c, 128);
    }
    out[0] = s.list[0];
    out[1] = s.list[1];
  }

  // find_best_ref_mvs( refList ) (spec 6.5.12).
  TP_HD void find_best_ref_mvs(int ref_list) {
    Mv list[2];
    find_mv_refs(b.ref_frame[ref_list], -1, list);
    const int32_t border = (160 /* BORDERINPIXELS */ - 4 /* INTERP_EXTEND */) << 3;
    for (int i = 0; i < 2; ++i) {
      int32_t dr = list[i].r, dc = list[i].c;
      if (!F->allow_hp || !use_mv_hp(list[i])) {
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
  TP_HD void append_sub8x8_mvs(int block, int ref_list) {
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
      for (int idx = 1; idx >= 0 && dst < 2; --idx)
        if (!mv_eq(bm[idx], sub[0])) sub[dst++] = bm[idx];
    }
    for (int n = 0; n < 2 && dst < 2; ++n)
      if (!mv_eq(list[n], sub[0])) sub[dst++] = list[n];
    if (dst < 2) sub[dst] = Mv{0, 0};
    b.nearest_mv[ref_list] = sub[0];
    b.near_mv[ref_list] = sub[1];
  }

  // ---- Residual (spec 6.4.21 - 6.4.26) ----

  TP_INL uint8_t uv_tx_size() const {
    if (b.mi_size < 3) return 0;
    const int sx = F->legacy_uv ? 1 : (int)ss_x, sy = F->legacy_uv ? 1 : (int)ss_y;
    const uint8_t m = T->max_tx[T->ss_size[b.mi_size][sx][sy]];
    return b.tx_size < m ? b.tx_size : m;
  }

  TP_INL uint8_t tx_type(int plane, int tx_sz, int block_idx) const {
    if (plane > 0 || tx_sz == 3) return 0;
    if (tx_sz == 0) {
      if (F->lossless || b.is_inter) return 0;
      return T->mode2txfm[b.mi_size < 3 ? b.sub_modes[block_idx] : b.y_mode];
    }
    return T->mode2txfm[b.y_mode];
  }

  TP_HD void residual() {
    const uint8_t bsize = b.mi_size < 3 ? 3 : b.mi_size;
    for (int plane = 0; plane < 3; ++plane) {
      const int tx_sz = plane > 0 ? uv_tx_size() : b.tx_size;
      const int step = 1 << tx_sz;
      const int sx = plane > 0 ? (int)ss_x : 0, sy = plane > 0 ? (int)ss_y : 0;
      const uint8_t plane_sz = T->ss_size[bsize][sx][sy];
      if (plane_sz == 14) {
        fail(TP_CHROMA_SIZE);
        return;
      }
      const int n4w = T->n4w[plane_sz], n4h = T->n4h[plane_sz];
      const uint32_t base_x = (b.mi_col * 8) >> sx, base_y = (b.mi_row * 8) >> sy;
      if (b.is_inter && plane == 0) {
        const int n = 1 + (b.ref_frame[1] > 0 ? 1 : 0);
        for (int i = 0; i < n; ++i)
          if (!F->ref_ok[b.ref_frame[i] - 1]) {
            fail(TP_REF_SCALE);
            return;
          }
      }
      const uint32_t max_x = (mi_cols * 8) >> sx, max_y = (mi_rows * 8) >> sy;
      int block_idx = 0;
      uint8_t* an = above_nz[plane];
      uint8_t* ln = left_nz[plane];
      for (int y = 0; y < n4h; y += step) {
        for (int x = 0; x < n4w; x += step) {
          const uint32_t start_x = base_x + 4 * x, start_y = base_y + 4 * y;
          bool nonzero = false;
          if (start_x < max_x && start_y < max_y && !b.skip) {
            const int eob = tokens(plane, start_x, start_y, tx_sz, block_idx);
            if (err) return;
            nonzero = eob > 0;
          }
          for (int i = 0; i < step; ++i) {
            an[(start_x >> 2) + i] = nonzero;
            ln[((start_y >> 2) + i) & 15] = nonzero;
          }
          ++block_idx;
        }
      }
    }
  }

  // tokens() (spec 6.4.24): records the nonzero coefficients; returns eob.
  TP_HD int tokens(int plane, uint32_t start_x, uint32_t start_y, int tx_sz, int block_idx) {
    const int seg_eob = 16 << (tx_sz << 1);
    const int ttype = tx_type(plane, tx_sz, block_idx);
    const int ref_type = b.is_inter ? 1 : 0;
    const int ptype = plane > 0 ? 1 : 0;
    const int sx = plane > 0 ? (int)ss_x : 0, sy = plane > 0 ? (int)ss_y : 0;
    const uint32_t max_x4 = (2 * mi_cols) >> sx, max_y4 = (2 * mi_rows) >> sy;
    const uint32_t x4 = start_x >> 2, y4 = start_y >> 2;
    uint8_t above = 0, left = 0;
    const uint8_t* an = above_nz[plane];
    const uint8_t* ln = left_nz[plane];
    for (int i = 0; i < (1 << tx_sz); ++i) {
      if (x4 + i < max_x4) above |= an[x4 + i];
      if (y4 + i < max_y4) left |= ln[(y4 + i) & 15];
    }
    if (n_toks >= cap_toks || n_coefs + (uint32_t)seg_eob > cap_coefs) {
      fail(TP_OVERFLOW);
      return 0;
    }
    const int kind = ttype == 2 /* DCT_ADST */ ? 1 : ttype == 1 /* ADST_DCT */ ? 2 : 0;
    const ScanEnt* sc = T->scan[tx_sz][kind];
    const uint32_t pkb = 36 * ((tx_sz * 2 + ptype) * 2 + ref_type);
    const uint32_t bd_bits = F->bit_depth;
    const uint32_t coef0 = n_coefs;
    uint32_t* out = coefs + n_coefs;
    uint32_t n_out = 0;
    int c = 0;
    // The loop keeps the current scan index's entry `e`, its band's six
    // probability words `w` (in registers) and its context; and, loaded a
    // step ahead so that no load waits on the decode, the next entry `en`,
    // its band's words `wn` and the token energies of its two context
    // neighbours (t0, t1). A neighbour of `en` may be the current position,
    // whose energy is only known once its token is decoded: advance()
    // substitutes it. Bytes 6 and 7 of a band word are zero, so the selector
    // 0x7770 | ctx yields the context's probability byte alone.
    ScanEnt e = ld_scan(sc);
    ScanEnt en = ld_scan(sc + 1);
    uint32_t w[6], wn[6];
    auto band = [&](uint32_t* dst, uint32_t b) {
      const uint32_t o = pkb + 6 * b;
#pragma unroll
      for (int k = 0; k < 6; ++k) dst[k] = TP_PKW(o + k);
    };
    band(w, e.band);
    band(wn, en.band);
    uint32_t t0 = TP_TC(en.nb0), t1 = TP_TC(en.nb1);
    uint32_t ctx = above + left;
    // After the token at e.pos (energy `cur`, already stored) and ++c.
    auto advance = [&](uint32_t cur) {
      ctx = (1 + (en.nb0 == e.pos ? cur : t0) + (en.nb1 == e.pos ? cur : t1)) >> 1;
      e = en;
#pragma unroll
      for (int k = 0; k < 6; ++k) w[k] = wn[k];
      en = ld_scan(sc + (c + 1 < seg_eob ? c + 1 : c));
      band(wn, en.band);
      t0 = TP_TC(en.nb0);
      t1 = TP_TC(en.nb1);
    };
    Bool r = bd;
    while (true) {
      // more_coefs: read at the start and after every nonzero token.
      if (!r.read(byte_perm(w[0], w[1], 0x7770u | ctx))) break;
      // A run of zero tokens; after a zero token no more_coefs is read.
      bool done = false;
      while (!r.read(byte_perm(w[2], w[3], 0x7770u | ctx))) {
        TP_TC(e.pos) = 0;
        if (++c == seg_eob) {
          done = true;
          break;
        }
        advance(0);
      }
      if (done) break;
      int32_t coef;
      uint32_t energy;
      const uint32_t p2 = byte_perm(w[4], w[5], 0x7770u | ctx);
      if (!r.read(p2)) {
        coef = 1;  // ONE_TOKEN
        energy = 1;
      } else {
        // The rest of the token tree (TOKEN_TREE from node 4), its node
        // probabilities from one pareto row, walked as its fixed branches:
        // no table load waits between two decodes.
        const uint2 pp = ro(reinterpret_cast<const uint2*>(T->pareto[p2]));
        auto pr = [&](uint32_t k) { return byte_perm(pp.x, pp.y, k) & 0xffu; };
        int cat = 0;  // DCT_VAL_CATEGORY1..6 as 1..6; 0: TWO, THREE or FOUR
        if (!r.read(pr(0))) {
          if (!r.read(pr(1))) {
            coef = 2;  // TWO_TOKEN
            energy = 2;
          } else {
            coef = r.read(pr(2)) ? 4 : 3;  // FOUR_TOKEN : THREE_TOKEN
            energy = 3;
          }
        } else if (!r.read(pr(3))) {
          cat = r.read(pr(4)) ? 2 : 1;
          energy = 4;
        } else if (!r.read(pr(5))) {
          cat = r.read(pr(6)) ? 4 : 3;
          energy = 5;
        } else {
          cat = r.read(pr(7)) ? 6 : 5;
          energy = 5;
        }
        if (cat) {
          // The category's base value and extra bits (spec 9.3: extra_bits).
          const int num_extra = cat == 6 ? 14 : cat;
          coef = cat == 6 ? 67 : cat == 5 ? 35 : cat == 4 ? 19 : cat == 3 ? 11 : cat == 2 ? 7 : 5;
          if (cat == 6)
            for (int k = 0; k < (int)bd_bits - 8; ++k) coef += (int32_t)r.read(255) << (5 + (int)bd_bits - k);
          const uint8_t* probs = T->cat_probs[cat];
          for (int k = 0; k < num_extra; ++k) coef += (int32_t)r.read(ro(&probs[k])) << (num_extra - 1 - k);
        }
      }
      TP_TC(e.pos) = (uint8_t)energy;
      const bool sign = r.read(128);
      out[n_out++] = RV9_COEF_PACK(e.pos, sign ? -coef : coef);
      if (++c == seg_eob) break;
      advance(energy);
    }
    bd = r;
    n_coefs += n_out;
    if (c > 0) ++eob_total;
    rv9_tok t;
    t.x = (uint16_t)start_x;
    t.y = (uint16_t)start_y;
    t.plane = (uint8_t)plane;
    t.tx_size = (uint8_t)tx_sz;
    t.tx_type = (uint8_t)ttype;
    t.reserved = 0;
    t.eob = (uint16_t)c;
    t.n_coef = (uint16_t)n_out;
    t.coef_start = coef0;
    toks[n_toks++] = t;
    return c;
  }
};

// Decodes one tile column (its tiles in bitstream order) into the chain's
// outputs. `tc` is 1024 bytes of token cache; `pkw` the frame's coef_pk as
// 32-bit words; `data` the batch's packet bytes.
// Record indices (tok_start, coef_start) are relative to the chain's own
// arrays; the caller rebases them when it gathers a frame's columns.
TP_HD inline void parse_chain(const Tables* T, const FrameIn* frames, const Chain& ch, const Span* spans,
                              const uint8_t* data, Mi* mi_base, uint8_t* above_base, const PrevMv* prev_base,
                              rv9_block* blocks, rv9_tok* toks, uint32_t* coefs, uint8_t* tc, const uint32_t* pkw,
                              ChainOut* out) {
  const FrameIn* F = &frames[ch.frame];
  TileParser P;
  P.pkw = pkw;
  P.T = T;
  P.F = F;
  P.mi = mi_base + ch.mi_at;
  uint8_t* above = above_base + ch.above_at;
  const uint32_t n4w = F->sb64_cols * 16 + 16;
  for (int p = 0; p < 3; ++p) P.above_nz[p] = above + p * n4w;
  P.above_part = above + 3 * n4w;
  P.prev = F->use_prev ? prev_base + ch.prev_at : nullptr;
  P.blocks = blocks + ch.blocks_at;
  P.toks = toks + ch.toks_at;
  P.coefs = coefs + ch.coefs_at;
  P.n_blocks = P.n_toks = P.n_coefs = 0;
  P.cap_blocks = ch.blocks_cap;
  P.cap_toks = ch.toks_cap;
  P.cap_coefs = ch.coefs_cap;
  P.tc = tc;
  P.mi_col_start = ch.mi_col_start;
  P.mi_col_end = ch.mi_col_end;
  P.mi_cols = F->mi_cols;
  P.mi_rows = F->mi_rows;
  P.ss_x = F->ss_x;
  P.ss_y = F->ss_y;
  P.err = TP_OK;
  uint32_t err_tile = 0, bools = 0;
  for (uint32_t k = 0; k < ch.n_spans && !P.err; ++k) {
    const Span& s = spans[ch.first_span + k];
    P.mi_row_start = s.mi_row_start;
    P.mi_row_end = s.mi_row_end;
    err_tile = s.index;
    if (s.size == 0) {
      P.err = TP_EMPTY_TILE;
      break;
    }
    if (!P.bd.init(data + s.off, s.size)) {
      P.err = TP_MARKER;
      break;
    }
    P.decode_tile();
    bools += P.bd.count;
  }
  out->n_blocks = P.n_blocks;
  out->n_toks = P.n_toks;
  out->n_coefs = P.n_coefs;
  out->err = P.err;
  out->err_tile = P.err ? err_tile : 0;
  out->bools = bools;
}

}  // namespace tp
}  // namespace rv9g

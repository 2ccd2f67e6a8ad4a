// Device-side work descriptions of the reconstruction engine, shared by the
// host code that builds them and the kernels that consume them.
#pragma once
#include <stdint.h>

#include "../../../include/rv9_records.h"

namespace rv9g {

// One inter prediction region: a block's plane, or one 4x4 sub-block of a
// block below 8x8 (reference FrameDec::predict_inter calls,
// src/decoder/block.rs:1430-1446).
struct InterUnit {
  uint32_t block;    // index into the frame's rv9_block array
  uint16_t x, y;     // plane sample position
  uint8_t plane;
  uint8_t w4, h4;    // size in 4-sample units
  uint8_t block_idx; // sub-block (mv index) for blocks below 8x8
};

// One intra transform block: prediction from its reconstructed neighbours,
// then its residual (reference FrameDec::predict_intra + reconstruct).
struct IntraItem {
  uint32_t block;
  uint32_t tok;      // rv9_tok index, or 0xffffffff when there is no residual
  uint16_t x, y;
  uint8_t plane;
  uint8_t tx_size;
  uint8_t mode;
  uint8_t flags;     // 1 have_left, 2 have_above, 4 not_on_right
};

constexpr uint32_t NO_TOK = 0xffffffffu;

// One inter block's coded transform block: its residual is added to the
// block's prediction.
struct ResItem {
  uint32_t tok;
  uint32_t block;
};

struct PlanePtr {
  void* data;
  int32_t stride;     // samples
  int32_t width;      // visible width in samples (references: lastX + 1)
  int32_t height;
};

// Everything a frame's kernels read, passed by value.
struct KFrame {
  PlanePtr cur[3];          // the frame being reconstructed (SB-aligned planes)
  PlanePtr ref[3][3];       // [LAST, GOLDEN, ALTREF][plane]
  int64_t ref_xs[3], ref_ys[3];  // reference scale factors, 1/(1<<14)
  uint8_t* cells[3];        // intra pending map, one byte per 4x4 per plane
  int32_t cell_stride[3];
  int32_t mi_cols, mi_rows, sb64_cols, sb64_rows;
  int32_t width, height;    // frame luma size
  int32_t ss_x, ss_y, bit_depth, lossless, legacy_uv;
  int32_t dc_q[8][2], ac_q[8][2];  // [segment][plane > 0]
  const rv9_block* blocks;
  const rv9_tok* toks;
  const uint32_t* coefs;
  const InterUnit* units;  // regions of at most 16x16 first, then the rest
  int32_t n_units;
  int32_t n_units_small;
  const ResItem* res;       // inter blocks' transform blocks with coefficients, 4x4 first, then 8x8, 16x16, 32x32
  int32_t n_res_by_size[4];
  int32_t n_res;
  const IntraItem* intra;
  int32_t n_intra;
  // Intra jobs: one row of a block's transform blocks of one plane, items
  // [intra_jobs[j], intra_jobs[j + 1]); n_intra_jobs + 1 entries.
  const uint32_t* intra_jobs;
  int32_t n_intra_jobs;
  // Loop filter.
  uint32_t* lf_mi;          // per 8x8: packed level / tx sizes / block size / skip
  uint8_t lvl[8][4][2];
  uint8_t lf_limit[64], lf_blimit[64], lf_thresh[64];
  int32_t lf_on;
  uint32_t* sb_done;        // loop filter: per superblock row, epoch << 16 | superblocks done
  uint32_t epoch;
  int32_t* counters;        // [0] intra tickets, [1] lf tickets
  int32_t* error;           // nonzero: a device wait timed out (code)
  int32_t wait_limit;       // polls before a wavefront wait gives up
  // Failure injection for tests (0 in normal use): bit 0 leaves the first
  // intra job untaken, bit 1 the first loop-filter row, so that the jobs
  // that depend on it wait until wait_limit runs out. No access goes out of
  // bounds and every wait still ends.
  int32_t test_skip;
};

}  // namespace rv9g

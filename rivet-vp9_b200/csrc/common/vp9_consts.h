// Symbolic constants and decode trees of the VP9 specification (sections 3,
// 6, 7 and 9.3.1), shared by the host parser, the encoder and the kernels.
// Values follow the specification's numbering, which the reference crate
// uses as well (rivet-vp9 src/consts.rs).
#pragma once
#include <stdint.h>

namespace vp9 {

constexpr int KEY_FRAME = 0;

// Block sizes (7.4.3).
enum : uint8_t {
  BLOCK_4X4 = 0, BLOCK_4X8, BLOCK_8X4, BLOCK_8X8, BLOCK_8X16, BLOCK_16X8,
  BLOCK_16X16, BLOCK_16X32, BLOCK_32X16, BLOCK_32X32, BLOCK_32X64,
  BLOCK_64X32, BLOCK_64X64, BLOCK_INVALID = 14
};

enum : uint8_t { PARTITION_NONE = 0, PARTITION_HORZ, PARTITION_VERT, PARTITION_SPLIT };

// Intra modes then inter modes: one numbering for y_mode.
enum : uint8_t {
  DC_PRED = 0, V_PRED, H_PRED, D45_PRED, D135_PRED, D117_PRED, D153_PRED,
  D207_PRED, D63_PRED, TM_PRED, NEARESTMV, NEARMV, ZEROMV, NEWMV
};

enum : uint8_t { TX_4X4 = 0, TX_8X8, TX_16X16, TX_32X32 };
enum : uint8_t { ONLY_4X4 = 0, ALLOW_8X8, ALLOW_16X16, ALLOW_32X32, TX_MODE_SELECT };
enum : uint8_t { DCT_DCT = 0, ADST_DCT = 1, DCT_ADST = 2, ADST_ADST = 3 };

// Reference frames; NONE sorts below INTRA_FRAME.
constexpr int8_t NONE_FRAME = -1;
constexpr int8_t INTRA_FRAME = 0;
constexpr int8_t LAST_FRAME = 1;
constexpr int8_t GOLDEN_FRAME = 2;
constexpr int8_t ALTREF_FRAME = 3;

// Interpolation filters (7.2.7) in the numbering of the subpel filter table.
enum : uint8_t { EIGHTTAP = 0, EIGHTTAP_SMOOTH = 1, EIGHTTAP_SHARP = 2, BILINEAR = 3, SWITCHABLE = 4 };
constexpr uint8_t LITERAL_TO_TYPE[4] = {EIGHTTAP_SMOOTH, EIGHTTAP, EIGHTTAP_SHARP, BILINEAR};

enum : uint8_t { SINGLE_REFERENCE = 0, COMPOUND_REFERENCE = 1, REFERENCE_MODE_SELECT = 2 };
enum : uint8_t { MV_JOINT_ZERO = 0, MV_JOINT_HNZVZ, MV_JOINT_HZVNZ, MV_JOINT_HNZVNZ };

constexpr int ZERO_TOKEN = 0;
constexpr int DCT_VAL_CAT6 = 10;

constexpr int SEG_LVL_ALT_Q = 0;
constexpr int SEG_LVL_ALT_L = 1;
constexpr int SEG_LVL_REF_FRAME = 2;
constexpr int SEG_LVL_SKIP = 3;
constexpr int MAX_SEGMENTS = 8;

constexpr int MV_BORDER = 128;
constexpr int INTERP_EXTEND = 4;
constexpr int BORDERINPIXELS = 160;
constexpr int COMPANDED_MVREF_THRESH = 8;
constexpr int MAX_LOOP_FILTER = 63;
constexpr uint32_t MIN_TILE_WIDTH_B64 = 4;
constexpr uint32_t MAX_TILE_WIDTH_B64 = 64;

// Inter mode contexts.
enum : uint8_t {
  BOTH_ZERO = 0, ZERO_PLUS_PREDICTED = 1, BOTH_PREDICTED = 2, NEW_PLUS_NON_INTRA = 3,
  BOTH_NEW = 4, INTRA_PLUS_NON_INTRA = 5, BOTH_INTRA = 6, INVALID_CASE = 9
};

constexpr uint8_t COUNTER_TO_CONTEXT[19] = {
  BOTH_PREDICTED, NEW_PLUS_NON_INTRA, BOTH_NEW, ZERO_PLUS_PREDICTED, NEW_PLUS_NON_INTRA,
  INVALID_CASE, BOTH_ZERO, INVALID_CASE, INVALID_CASE, INTRA_PLUS_NON_INTRA,
  INTRA_PLUS_NON_INTRA, INVALID_CASE, INTRA_PLUS_NON_INTRA, INVALID_CASE, INVALID_CASE,
  INVALID_CASE, INVALID_CASE, INVALID_CASE, BOTH_INTRA};

constexpr uint8_t MAX_TXSIZE_LOOKUP[13] = {
  TX_4X4, TX_4X4, TX_4X4, TX_8X8, TX_8X8, TX_8X8, TX_16X16, TX_16X16, TX_16X16,
  TX_32X32, TX_32X32, TX_32X32, TX_32X32};

constexpr uint8_t TX_MODE_TO_BIGGEST_TX_SIZE[5] = {TX_4X4, TX_8X8, TX_16X16, TX_32X32, TX_32X32};

constexpr uint8_t I_ = BLOCK_INVALID;
// ss_size_lookup[bsize][subx][suby] (6.4.23).
constexpr uint8_t SS_SIZE_LOOKUP[13][2][2] = {
  {{BLOCK_4X4, I_}, {I_, I_}},
  {{BLOCK_4X8, BLOCK_4X4}, {I_, I_}},
  {{BLOCK_8X4, I_}, {BLOCK_4X4, I_}},
  {{BLOCK_8X8, BLOCK_8X4}, {BLOCK_4X8, BLOCK_4X4}},
  {{BLOCK_8X16, BLOCK_8X8}, {I_, BLOCK_4X8}},
  {{BLOCK_16X8, I_}, {BLOCK_8X8, BLOCK_8X4}},
  {{BLOCK_16X16, BLOCK_16X8}, {BLOCK_8X16, BLOCK_8X8}},
  {{BLOCK_16X32, BLOCK_16X16}, {I_, BLOCK_8X16}},
  {{BLOCK_32X16, I_}, {BLOCK_16X16, BLOCK_16X8}},
  {{BLOCK_32X32, BLOCK_32X16}, {BLOCK_16X32, BLOCK_16X16}},
  {{BLOCK_32X64, BLOCK_32X32}, {I_, BLOCK_16X32}},
  {{BLOCK_64X32, I_}, {BLOCK_32X32, BLOCK_32X16}},
  {{BLOCK_64X64, BLOCK_64X32}, {BLOCK_32X64, BLOCK_32X32}},
};

// subsize_lookup[partition][bsize] (10.2).
constexpr uint8_t SUBSIZE_LOOKUP[4][13] = {
  {BLOCK_4X4, BLOCK_4X8, BLOCK_8X4, BLOCK_8X8, BLOCK_8X16, BLOCK_16X8, BLOCK_16X16,
   BLOCK_16X32, BLOCK_32X16, BLOCK_32X32, BLOCK_32X64, BLOCK_64X32, BLOCK_64X64},
  {I_, I_, I_, BLOCK_8X4, I_, I_, BLOCK_16X8, I_, I_, BLOCK_32X16, I_, I_, BLOCK_64X32},
  {I_, I_, I_, BLOCK_4X8, I_, I_, BLOCK_8X16, I_, I_, BLOCK_16X32, I_, I_, BLOCK_32X64},
  {I_, I_, I_, BLOCK_4X4, I_, I_, BLOCK_8X8, I_, I_, BLOCK_16X16, I_, I_, BLOCK_32X32},
};

// mode2txfm_map (10.2).
constexpr uint8_t MODE2TXFM_MAP[14] = {
  DCT_DCT, ADST_DCT, DCT_ADST, DCT_DCT, ADST_ADST, ADST_DCT, DCT_ADST,
  DCT_ADST, ADST_DCT, ADST_ADST, DCT_DCT, DCT_DCT, DCT_DCT, DCT_DCT};

// extra_bits[token]: category, number of extra bits, base value (6.4.26).
constexpr int EXTRA_BITS[11][3] = {
  {0, 0, 0}, {0, 0, 1}, {0, 0, 2}, {0, 0, 3}, {0, 0, 4}, {1, 1, 5},
  {2, 2, 7}, {3, 3, 11}, {4, 4, 19}, {5, 5, 35}, {6, 14, 67}};

constexpr uint8_t CAT_PROBS[7][14] = {
  {0},
  {159},
  {165, 145},
  {173, 148, 140},
  {176, 155, 140, 135},
  {180, 157, 141, 134, 130},
  {254, 254, 254, 252, 249, 243, 230, 196, 177, 153, 140, 133, 130, 129},
};

// Decode trees (9.3.1): leaves are negated values, a leaf of value 0 is 0.
constexpr int8_t PARTITION_TREE[6] = {-PARTITION_NONE, 2, -PARTITION_HORZ, 4, -PARTITION_VERT, -PARTITION_SPLIT};
constexpr int8_t INTRA_MODE_TREE[18] = {
  -DC_PRED, 2, -TM_PRED, 4, -V_PRED, 6, 8, 12, -H_PRED, 10, -D135_PRED, -D117_PRED,
  -D45_PRED, 14, -D63_PRED, 16, -D153_PRED, -D207_PRED};
constexpr int8_t SEGMENT_TREE[14] = {2, 4, 6, 8, 10, 12, 0, -1, -2, -3, -4, -5, -6, -7};
constexpr int8_t TX_SIZE_32_TREE[6] = {-TX_4X4, 2, -TX_8X8, 4, -TX_16X16, -TX_32X32};
constexpr int8_t TX_SIZE_16_TREE[4] = {-TX_4X4, 2, -TX_8X8, -TX_16X16};
constexpr int8_t TX_SIZE_8_TREE[2] = {-TX_4X4, -TX_8X8};
// Values are y_mode - NEARESTMV.
constexpr int8_t INTER_MODE_TREE[6] = {-(ZEROMV - NEARESTMV), 2, -(NEARESTMV - NEARESTMV), 4,
                                       -(NEARMV - NEARESTMV), -(NEWMV - NEARESTMV)};
constexpr int8_t INTERP_FILTER_TREE[4] = {-EIGHTTAP, 2, -EIGHTTAP_SMOOTH, -EIGHTTAP_SHARP};
constexpr int8_t MV_JOINT_TREE[6] = {-MV_JOINT_ZERO, 2, -MV_JOINT_HNZVZ, 4, -MV_JOINT_HZVNZ, -MV_JOINT_HNZVNZ};
constexpr int8_t MV_CLASS_TREE[20] = {0, 2, -1, 4, 6, 8, -2, -3, 10, 12, -4, -5, -6, 14, 16, 18, -7, -8, -9, -10};
constexpr int8_t MV_FR_TREE[6] = {0, 2, -1, 4, -2, -3};
constexpr int8_t TOKEN_TREE[20] = {0, 2, -1, 4, 6, 10, -2, 8, -3, -4, 12, 14, -5, -6, 16, 18, -7, -8, -9, -10};
// small_token_tree (8.4.3), adapted from index 2.
constexpr int8_t SMALL_TOKEN_TREE[6] = {0, 0, 0, 4, -1, -2};
constexpr int8_t BINARY_TREE[2] = {0, -1};

}  // namespace vp9

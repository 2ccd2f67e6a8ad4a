/*
 * rv9_records.h — the parsed-frame records handed from the host parser to the
 * reconstruction engine (the host -> device seam of the VP9 decoder).
 *
 * The reference decoder (safewords/rivet-vp9) already splits parsing from
 * reconstruction in its pipelined mode: the parser records one superblock row
 * as a RowRec (src/decoder/block.rs:143-152) of Block records
 * (src/decoder/block.rs:51-76), TokRec entries (src/decoder/block.rs:133-137)
 * and (position, value) coefficient pairs, and FrameDec::replay
 * (src/decoder/block.rs:1405-1498) reconstructs from them. These structs carry
 * the same information for a whole frame, laid out flat for a single
 * host->device copy:
 *
 *   rv9_frame_desc  the header fields reconstruction needs (size, format,
 *                   quantiser, loop filter and segmentation parameters, the
 *                   sizes of the three active references);
 *   rv9_block       one per decoded block, in decode (bitstream) order;
 *   rv9_tok         one per transform block of a non-skipped block that lies
 *                   inside the frame's mode-info area, in the residual
 *                   syntax's order (plane, then raster within the block);
 *   coefficient     one uint32 per nonzero coefficient, in scan order:
 *                   bits 0..9 the raster position in the transform block,
 *                   bits 10..31 the signed token value (not dequantised).
 *
 * Plain C; no pointers inside the structs, so arrays of them can be copied to
 * the device as they are.
 */
#ifndef RV9_RECORDS_H
#define RV9_RECORDS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RV9_MAX_SEGMENTS 8

/* Segmentation parameters (reference: src/header.rs:38-47). */
typedef struct rv9_segmentation {
  uint8_t enabled;
  uint8_t update_map;
  uint8_t temporal_update;
  uint8_t abs_or_delta_update;
  uint8_t feature_enabled[RV9_MAX_SEGMENTS][4];
  int16_t feature_data[RV9_MAX_SEGMENTS][4];
} rv9_segmentation;

/* What reconstruction needs of a frame header (reference: FrameHeader,
 * src/header.rs:88-146, LoopFilter src/header.rs:16-22). */
typedef struct rv9_frame_desc {
  uint32_t width, height;         /* FrameWidth, FrameHeight */
  uint32_t mi_cols, mi_rows;      /* 8x8 units */
  uint32_t sb64_cols, sb64_rows;  /* 64x64 units */
  uint8_t ss_x, ss_y;             /* chroma subsampling */
  uint8_t bit_depth;              /* 8, 10, 12 */
  uint8_t lossless;               /* base_q_idx == 0 and no deltas: WHT */
  uint8_t legacy_uv;              /* pre-final profile 1 stream rules */
  uint8_t frame_is_intra;
  uint8_t show_frame;
  uint8_t tile_cols_log2;         /* tile columns: 1 << tile_cols_log2 */
  int32_t base_q_idx;
  int32_t delta_q_y_dc, delta_q_uv_dc, delta_q_uv_ac;
  uint8_t lf_level, lf_sharpness, lf_delta_enabled, reserved1;
  int8_t lf_ref_deltas[4];
  int8_t lf_mode_deltas[2];
  uint8_t reserved2[2];
  rv9_segmentation seg;
  /* Luma size of the LAST, GOLDEN and ALTREF references (inter frames). */
  uint32_t ref_width[3], ref_height[3];
  /* Output metadata (reference: Frame, src/frame.rs:115-137). */
  uint8_t color_space;            /* 0..7 as coded */
  uint8_t color_range;            /* 1: full swing */
  uint8_t reserved3[2];
  uint32_t render_width, render_height;
} rv9_frame_desc;

/* Block flags. */
#define RV9_BLK_SKIP 1u
#define RV9_BLK_INTER 2u
#define RV9_BLK_AVAIL_L 4u
#define RV9_BLK_AVAIL_U 8u

/* One decoded block: the Block fields replay reads (reference:
 * src/decoder/block.rs:51-76) and the MiInfo fields the loop filter reads
 * (src/decoder/block.rs:19-31). `skip` is the value after the residual syntax
 * (an inter block of 8x8 or more with no coefficients reads as skipped,
 * src/decoder/block.rs:548-551); `coded_skip` is the bitstream's, which
 * decides whether tokens were read. */
typedef struct rv9_block {
  uint16_t mi_row, mi_col;
  uint8_t mi_size;        /* BLOCK_* */
  uint8_t flags;          /* RV9_BLK_*; SKIP is the loop filter's skip */
  uint8_t tx_size;        /* luma TX_* */
  uint8_t segment_id;
  uint8_t y_mode;         /* intra mode, or NEARESTMV.. for inter blocks */
  uint8_t uv_mode;
  uint8_t interp_filter;  /* 0 regular, 1 smooth, 2 sharp, 3 bilinear */
  uint8_t coded_skip;     /* skip as read: no tokens follow */
  uint8_t sub_modes[4];   /* intra sub-8x8 modes, raster order */
  int8_t ref_frame[2];    /* INTRA_FRAME(0)/LAST(1)/GOLDEN(2)/ALTREF(3); -1 none */
  uint16_t n_tok;         /* rv9_tok records of this block */
  uint32_t tok_start;     /* first rv9_tok of this block */
  int32_t mv[2][4][2];    /* [ref list][4x4 sub-block][row, col], 1/8 sample */
} rv9_block;

/* One transform block of a non-skipped block (reference TokRec,
 * src/decoder/block.rs:133-137, with its position made explicit). */
typedef struct rv9_tok {
  uint16_t x, y;          /* top-left sample, plane coordinates */
  uint8_t plane;          /* 0 Y, 1 U, 2 V */
  uint8_t tx_size;        /* TX_* */
  uint8_t tx_type;        /* DCT_DCT, ADST_DCT, DCT_ADST, ADST_ADST */
  uint8_t reserved;
  uint16_t eob;           /* end of block: coefficients read */
  uint16_t n_coef;        /* nonzero coefficients recorded */
  uint32_t coef_start;    /* first coefficient word */
} rv9_tok;

/* Coefficient word helpers. */
#define RV9_COEF_POS(w) ((uint32_t)(w) & 1023u)
#define RV9_COEF_VAL(w) ((int32_t)(w) >> 10)
#define RV9_COEF_PACK(pos, val) (((uint32_t)(int32_t)(val) << 10) | ((uint32_t)(pos) & 1023u))

#ifdef __cplusplus
}
#endif

#endif /* RV9_RECORDS_H */

/*
 * rv9_encoder.h — the stream generator: a seeded synthetic video source and a
 * VP9 encoder for it (host CPU code).
 *
 * The reference crate ships an encoder (safewords/rivet-vp9 src/encoder/,
 * Encoder::encode src/encoder/mod.rs:276-349) whose output the benchmark
 * configurations are defined on. This is a project-written VP9 encoder that
 * produces streams of those shapes: key frame then inter frames, LAST and
 * GOLDEN references, variable partitions 64x64..8x8, every transform size
 * (TX_MODE_SELECT), all ten intra modes, NEARESTMV / NEARMV / ZEROMV / NEWMV,
 * per-block switchable regular / smooth / sharp filters, tile columns,
 * profiles 0-3 (8/10/12-bit, 4:2:0 .. 4:4:4). Its reconstruction is the
 * decoder's (closed loop): a fresh decoder's output equals the encoder's
 * reconstruction sample for sample.
 *
 * The synthetic source follows the benchmark definition: luma is a 2D sine
 * gradient (period 64 samples) panned per frame, plus moving rectangles of
 * uniform random level, plus uniform noise; chroma is a half-resolution
 * smooth gradient; all scaled to the bit depth.
 */
#ifndef RV9_ENCODER_H
#define RV9_ENCODER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rv9_gen_config {
  uint32_t width, height;
  uint32_t bit_depth;        /* 8, 10, 12 */
  uint32_t ss_x, ss_y;       /* chroma subsampling: (1,1) 4:2:0 ... (0,0) 4:4:4 */
  uint32_t frames;
  int32_t base_q_idx;        /* 1..255 */
  uint32_t tile_cols_log2;   /* raised to the minimum the width needs */
  uint32_t golden_interval;  /* a GOLDEN refresh every N frames (0: never) */
  uint32_t seed;
  int32_t pan_x, pan_y;      /* luma pan per frame, samples */
  uint32_t rectangles;       /* moving 32x24 rectangles */
  uint32_t noise;            /* uniform noise amplitude at 8 bits */
  uint32_t threads;          /* encoder threads (tile columns); 0 = cores */
  uint32_t color_space;      /* coded colour space: 0 = BT.709 (2), else the VP9 code (1 BT.601 ...) */
  /* 0: error-resilient frames (each parses on its own). 1: frames that are
   * not error-resilient, so inter frames read the previous frame's motion
   * vectors; they refresh no probability context, except that with
   * adapt_interval N > 0 frames N, 2N and 3N adapt their probabilities into
   * contexts 1, 2 and 3 (read by no other frame). */
  uint32_t non_resilient;
  uint32_t adapt_interval;
} rv9_gen_config;

/* Generates and encodes a stream: packets back to back into `out` (`cap`
 * bytes), packet sizes into `sizes` (`frames` entries). Returns 0, or -1 if
 * `out` is too small or the configuration is invalid. */
int rv9_gen_stream(const rv9_gen_config* cfg, uint8_t* out, size_t cap, size_t* sizes, size_t* total);

/* One source frame (uint16 samples, planes packed with stride == width). */
void rv9_gen_source_frame(const rv9_gen_config* cfg, uint32_t index, uint16_t* y, uint16_t* u, uint16_t* v);

/* The encoder's reconstruction of the last frame encoded by the last
 * rv9_gen_stream call on this thread, packed like a decoded Frame (u8 at 8
 * bits, little-endian u16 above). Returns its size in bytes. */
size_t rv9_gen_last_reconstruction(uint8_t* out, size_t cap);

#ifdef __cplusplus
}
#endif

#endif /* RV9_ENCODER_H */

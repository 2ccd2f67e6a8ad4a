// Frame contexts (the adaptive probability tables), symbol counts and the
// backward adaptation of spec 8.4 (reference src/probs.rs).
#pragma once
#include <stdint.h>
#include <string.h>

namespace rv9 {

typedef uint8_t CoefProbs[4][2][2][6][6][3];

struct Probs {
  uint8_t tx[4][2][3];  // [maxTxSize][ctx][node], row 0 unused
  CoefProbs coef;
  uint8_t skip[3];
  uint8_t inter_mode[7][3];
  uint8_t interp_filter[4][2];
  uint8_t is_inter[4];
  uint8_t comp_mode[5];
  uint8_t single_ref[5][2];
  uint8_t comp_ref[5];
  uint8_t y_mode[4][9];
  uint8_t uv_mode[10][9];
  uint8_t partition[16][3];
  uint8_t mv_joint[3];
  uint8_t mv_sign[2];
  uint8_t mv_class[2][10];
  uint8_t mv_class0_bit[2];
  uint8_t mv_bits[2][10];
  uint8_t mv_class0_fr[2][2][3];
  uint8_t mv_fr[2][3];
  uint8_t mv_class0_hp[2];
  uint8_t mv_hp[2];

  void set_default();
  // load_probs(ctx): everything but tx and skip (spec 7.1.2).
  void load_except_tx_skip(const Probs& from) {
    uint8_t t[4][2][3];
    uint8_t s[3];
    memcpy(t, tx, sizeof t);
    memcpy(s, skip, sizeof s);
    *this = from;
    memcpy(tx, t, sizeof t);
    memcpy(skip, s, sizeof s);
  }
  // load_probs2(ctx): tx and skip only.
  void load_tx_skip(const Probs& from) {
    memcpy(tx, from.tx, sizeof tx);
    memcpy(skip, from.skip, sizeof skip);
  }
};

typedef uint32_t CoefCount3[4][2][2][6][6][3];
typedef uint32_t CoefCount2[4][2][2][6][6][2];

struct Counts {
  uint32_t intra_mode[4][10];
  uint32_t uv_mode[10][10];
  uint32_t partition[16][4];
  uint32_t interp_filter[4][3];
  uint32_t inter_mode[7][4];
  uint32_t tx[4][2][4];
  uint32_t is_inter[4][2];
  uint32_t comp_mode[5][2];
  uint32_t single_ref[5][2][2];
  uint32_t comp_ref[5][2];
  uint32_t skip[3][2];
  uint32_t mv_joint[4];
  uint32_t mv_sign[2][2];
  uint32_t mv_class[2][11];
  uint32_t mv_class0_bit[2][2];
  uint32_t mv_class0_fr[2][2][4];
  uint32_t mv_class0_hp[2][2];
  uint32_t mv_bits[2][10][2];
  uint32_t mv_fr[2][4];
  uint32_t mv_hp[2][2];
  CoefCount3 token;
  CoefCount2 more_coefs;

  void clear() { memset(this, 0, sizeof *this); }
  // Adds another tile column's counts.
  void add(const Counts& o) {
    const uint32_t* s = (const uint32_t*)&o;
    uint32_t* d = (uint32_t*)this;
    for (size_t i = 0; i < sizeof(Counts) / 4; ++i) d[i] += s[i];
  }
};

// adapt_coef_probs (spec 8.4.3).
void adapt_coef_probs(Probs& p, const Counts& c, bool frame_is_intra, bool last_frame_was_key);
// adapt_noncoef_probs (spec 8.4.4).
void adapt_noncoef_probs(Probs& p, const Counts& c, bool interp_switchable, bool tx_mode_select,
                         bool allow_hp);

}  // namespace rv9

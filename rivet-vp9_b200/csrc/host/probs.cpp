// Default probabilities and backward adaptation (spec 8.4; reference
// src/probs.rs:38-342).
#include "probs.h"

#include "../common/vp9_consts.h"
#include "../common/vp9_tables.h"

namespace rv9 {
using namespace vp9;

void Probs::set_default() {
  memcpy(tx, vp9t_default_tx_probs, sizeof tx);
  memcpy(coef, vp9t_default_coef_probs, sizeof coef);
  memcpy(skip, vp9t_default_skip_prob, sizeof skip);
  memcpy(inter_mode, vp9t_default_inter_mode_probs, sizeof inter_mode);
  memcpy(interp_filter, vp9t_default_interp_filter_probs, sizeof interp_filter);
  memcpy(is_inter, vp9t_default_is_inter_prob, sizeof is_inter);
  memcpy(comp_mode, vp9t_default_comp_mode_prob, sizeof comp_mode);
  memcpy(single_ref, vp9t_default_single_ref_prob, sizeof single_ref);
  memcpy(comp_ref, vp9t_default_comp_ref_prob, sizeof comp_ref);
  memcpy(y_mode, vp9t_default_y_mode_probs, sizeof y_mode);
  memcpy(uv_mode, vp9t_default_uv_mode_probs, sizeof uv_mode);
  memcpy(partition, vp9t_default_partition_probs, sizeof partition);
  memcpy(mv_joint, vp9t_default_mv_joint_probs, sizeof mv_joint);
  memcpy(mv_sign, vp9t_default_mv_sign_prob, sizeof mv_sign);
  memcpy(mv_class, vp9t_default_mv_class_probs, sizeof mv_class);
  memcpy(mv_class0_bit, vp9t_default_mv_class0_bit_prob, sizeof mv_class0_bit);
  memcpy(mv_bits, vp9t_default_mv_bits_prob, sizeof mv_bits);
  memcpy(mv_class0_fr, vp9t_default_mv_class0_fr_probs, sizeof mv_class0_fr);
  memcpy(mv_fr, vp9t_default_mv_fr_probs, sizeof mv_fr);
  memcpy(mv_class0_hp, vp9t_default_mv_class0_hp_prob, sizeof mv_class0_hp);
  memcpy(mv_hp, vp9t_default_mv_hp_prob, sizeof mv_hp);
}

// merge_prob (spec 8.4.1).
static uint8_t merge_prob(uint8_t pre, uint32_t ct0, uint32_t ct1, uint32_t count_sat,
                          uint32_t max_update_factor) {
  uint32_t den = ct0 + ct1;
  uint32_t prob;
  if (den == 0) {
    prob = 128;
  } else {
    uint64_t p = ((uint64_t)ct0 * 256 + (den >> 1)) / den;
    prob = p < 1 ? 1 : (p > 255 ? 255 : (uint32_t)p);
  }
  uint32_t count = den < count_sat ? den : count_sat;
  uint32_t factor = max_update_factor * count / count_sat;
  uint32_t v = pre * (256 - factor) + prob * factor;
  return (uint8_t)((v + 128) >> 8);
}

// merge_probs (spec 8.4.2): adapts `probs` along `tree` from node `i`.
static uint32_t merge_probs(const int8_t* tree, int i, uint8_t* probs, const uint32_t* counts,
                            uint32_t count_sat, uint32_t upd) {
  int s = tree[i];
  uint32_t left = s <= 0 ? counts[-s] : merge_probs(tree, s, probs, counts, count_sat, upd);
  int r = tree[i + 1];
  uint32_t right = r <= 0 ? counts[-r] : merge_probs(tree, r, probs, counts, count_sat, upd);
  probs[i >> 1] = merge_prob(probs[i >> 1], left, right, count_sat, upd);
  return left + right;
}

static void adapt_probs(const int8_t* tree, uint8_t* probs, const uint32_t* counts) {
  merge_probs(tree, 0, probs, counts, 20, 128);
}

static void adapt_prob(uint8_t* prob, const uint32_t* counts) {
  *prob = merge_prob(*prob, counts[0], counts[1], 20, 128);
}

void adapt_coef_probs(Probs& p, const Counts& c, bool frame_is_intra, bool last_frame_was_key) {
  uint32_t uf = frame_is_intra ? 112 : (last_frame_was_key ? 128 : 112);
  for (int t = 0; t < 4; ++t)
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j)
        for (int k = 0; k < 6; ++k) {
          int max_l = k == 0 ? 3 : 6;
          for (int l = 0; l < max_l; ++l) {
            uint8_t* pr = p.coef[t][i][j][k][l];
            merge_probs(SMALL_TOKEN_TREE, 2, pr, c.token[t][i][j][k][l], 24, uf);
            merge_probs(BINARY_TREE, 0, pr, c.more_coefs[t][i][j][k][l], 24, uf);
          }
        }
}

void adapt_noncoef_probs(Probs& p, const Counts& c, bool interp_switchable, bool tx_mode_select,
                         bool allow_hp) {
  for (int i = 0; i < 4; ++i) adapt_prob(&p.is_inter[i], c.is_inter[i]);
  for (int i = 0; i < 5; ++i) adapt_prob(&p.comp_mode[i], c.comp_mode[i]);
  for (int i = 0; i < 5; ++i) adapt_prob(&p.comp_ref[i], c.comp_ref[i]);
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 2; ++j) adapt_prob(&p.single_ref[i][j], c.single_ref[i][j]);
  for (int i = 0; i < 7; ++i) adapt_probs(INTER_MODE_TREE, p.inter_mode[i], c.inter_mode[i]);
  for (int i = 0; i < 4; ++i) adapt_probs(INTRA_MODE_TREE, p.y_mode[i], c.intra_mode[i]);
  for (int i = 0; i < 10; ++i) adapt_probs(INTRA_MODE_TREE, p.uv_mode[i], c.uv_mode[i]);
  for (int i = 0; i < 16; ++i) adapt_probs(PARTITION_TREE, p.partition[i], c.partition[i]);
  for (int i = 0; i < 3; ++i) adapt_prob(&p.skip[i], c.skip[i]);
  if (interp_switchable)
    for (int i = 0; i < 4; ++i) adapt_probs(INTERP_FILTER_TREE, p.interp_filter[i], c.interp_filter[i]);
  if (tx_mode_select) {
    for (int i = 0; i < 2; ++i) {
      adapt_probs(TX_SIZE_8_TREE, p.tx[1][i], c.tx[1][i]);
      adapt_probs(TX_SIZE_16_TREE, p.tx[2][i], c.tx[2][i]);
      adapt_probs(TX_SIZE_32_TREE, p.tx[3][i], c.tx[3][i]);
    }
  }
  adapt_probs(MV_JOINT_TREE, p.mv_joint, c.mv_joint);
  for (int i = 0; i < 2; ++i) {
    adapt_prob(&p.mv_sign[i], c.mv_sign[i]);
    adapt_probs(MV_CLASS_TREE, p.mv_class[i], c.mv_class[i]);
    adapt_prob(&p.mv_class0_bit[i], c.mv_class0_bit[i]);
    for (int j = 0; j < 10; ++j) adapt_prob(&p.mv_bits[i][j], c.mv_bits[i][j]);
    for (int j = 0; j < 2; ++j) adapt_probs(MV_FR_TREE, p.mv_class0_fr[i][j], c.mv_class0_fr[i][j]);
    adapt_probs(MV_FR_TREE, p.mv_fr[i], c.mv_fr[i]);
    if (allow_hp) {
      adapt_prob(&p.mv_class0_hp[i], c.mv_class0_hp[i]);
      adapt_prob(&p.mv_hp[i], c.mv_hp[i]);
    }
  }
}

}  // namespace rv9

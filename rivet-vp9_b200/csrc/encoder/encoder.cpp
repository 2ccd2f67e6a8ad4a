// The stream generator: a seeded synthetic source and a closed-loop VP9
// encoder (see include/rv9_encoder.h). The block syntax is written by the
// decoder's own syntax code (TileCoder<EncCoder>, host/syntax.h) from this
// encoder's decisions, so what is written is what the parser reads; the
// reconstruction uses the kernels' arithmetic (recon_host.h), so what the
// encoder predicts from is what a decoder reconstructs.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <memory>
#include <thread>
#include <vector>

#include "../../../include/rv9_encoder.h"
#include "../host/syntax.h"
#include "recon_host.h"

namespace rv9enc {
using namespace vp9;
using rv9::Mv;

// ---------------------------------------------------------------------------
// Synthetic source.

static inline uint32_t hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

struct Rect {
  int x, y, vx, vy, level;
};

static std::vector<Rect> rectangles(const rv9_gen_config& c) {
  std::vector<Rect> r;
  uint32_t s = hash32(c.seed * 2654435761u + 12345u);
  auto next = [&]() {
    s = hash32(s + 0x9e3779b9u);
    return s;
  };
  for (uint32_t i = 0; i < c.rectangles; ++i) {
    Rect q;
    q.x = (int)(next() % std::max<uint32_t>(1, c.width));
    q.y = (int)(next() % std::max<uint32_t>(1, c.height));
    q.vx = (int)(next() % 9) - 4;
    q.vy = (int)(next() % 9) - 4;
    q.level = (int)(next() % 256);
    r.push_back(q);
  }
  return r;
}

static void source_frame(const rv9_gen_config& c, uint32_t t, uint16_t* py, uint16_t* pu, uint16_t* pv) {
  const int w = c.width, h = c.height, bd = c.bit_depth;
  const int maxv = (1 << bd) - 1;
  const double k = 2.0 * M_PI / 64.0;
  std::vector<Rect> rs = rectangles(c);
  const int ox = c.pan_x * (int)t, oy = c.pan_y * (int)t;
  std::vector<double> sx(w), sy(h);
  for (int x = 0; x < w; ++x) sx[x] = 40.0 * sin(k * (x + ox));
  for (int y = 0; y < h; ++y) sy[y] = 40.0 * sin(k * (y + oy));
  const int noise = (int)c.noise;
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      double v8 = 128.0 + sx[x] + sy[y];
      for (const Rect& r : rs) {
        int rx = ((r.x + r.vx * (int)t) % w + w) % w, ry = ((r.y + r.vy * (int)t) % h + h) % h;
        if (x >= rx && x < rx + 32 && y >= ry && y < ry + 24) v8 = r.level;
      }
      int v = (int)lround(v8 * (1 << (bd - 8)));
      if (noise) v += (int)(hash32(c.seed ^ (t * 0x01000193u) ^ (uint32_t)(y * 65537 + x)) % (2 * noise + 1)) - noise;
      py[(size_t)y * w + x] = (uint16_t)std::min(std::max(v, 0), maxv);
    }
  const int cw = (w + (int)c.ss_x) >> c.ss_x, ch = (h + (int)c.ss_y) >> c.ss_y;
  for (int y = 0; y < ch; ++y)
    for (int x = 0; x < cw; ++x) {
      double u8 = 128.0 + 30.0 * sin(2.0 * M_PI * (x + ox / 2) / 128.0) + 10.0 * cos(2.0 * M_PI * y / 96.0);
      double v8 = 128.0 + 30.0 * cos(2.0 * M_PI * (y + oy / 2) / 128.0) - 10.0 * sin(2.0 * M_PI * x / 80.0);
      pu[(size_t)y * cw + x] = (uint16_t)std::min(std::max((int)lround(u8 * (1 << (bd - 8))), 0), maxv);
      pv[(size_t)y * cw + x] = (uint16_t)std::min(std::max((int)lround(v8 * (1 << (bd - 8))), 0), maxv);
    }
}

// ---------------------------------------------------------------------------
// Forward transforms: the inverse of the decoder's 1D transforms, measured on
// unit vectors (the exact integer transform, 64-bit lane), inverted once.

struct ForwardTables {
  // inv[n-2][kind] : n0 x n0 (kind 0 DCT, 1 ADST), row-major.
  std::vector<double> inv[4][2];
  ForwardTables() {
    for (int n = 2; n <= 5; ++n)
      for (int kind = 0; kind < 2; ++kind) {
        if (n == 5 && kind == 1) continue;
        int n0 = 1 << n;
        std::vector<double> A((size_t)n0 * n0);
        const int64_t S = 1 << 16;
        for (int j = 0; j < n0; ++j) {
          rv9g::L64 t[32];
          for (int i = 0; i < n0; ++i) t[i] = rv9g::L64::load(i == j ? S : 0);
          switch (n) {
            case 2: rv9g::tx1d<2>(t, kind, 0); break;
            case 3: rv9g::tx1d<3>(t, kind, 0); break;
            case 4: rv9g::tx1d<4>(t, kind, 0); break;
            default: rv9g::tx1d<5>(t, kind, 0); break;
          }
          for (int i = 0; i < n0; ++i) A[(size_t)i * n0 + j] = (double)t[i].v / (double)S;
        }
        inv[n - 2][kind] = invert(A, n0);
      }
  }
  static std::vector<double> invert(std::vector<double> a, int n) {
    std::vector<double> r((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) r[(size_t)i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
      int piv = c;
      for (int i = c + 1; i < n; ++i)
        if (fabs(a[(size_t)i * n + c]) > fabs(a[(size_t)piv * n + c])) piv = i;
      for (int j = 0; j < n; ++j) {
        std::swap(a[(size_t)c * n + j], a[(size_t)piv * n + j]);
        std::swap(r[(size_t)c * n + j], r[(size_t)piv * n + j]);
      }
      double d = a[(size_t)c * n + c];
      for (int j = 0; j < n; ++j) {
        a[(size_t)c * n + j] /= d;
        r[(size_t)c * n + j] /= d;
      }
      for (int i = 0; i < n; ++i) {
        if (i == c) continue;
        double f = a[(size_t)i * n + c];
        if (f == 0) continue;
        for (int j = 0; j < n; ++j) {
          a[(size_t)i * n + j] -= f * a[(size_t)c * n + j];
          r[(size_t)i * n + j] -= f * r[(size_t)c * n + j];
        }
      }
    }
    return r;
  }
};

static const ForwardTables& fwd_tables() {
  static const ForwardTables t;
  return t;
}

// Coefficients X with A_col X A_row^T / 2^shift = R (the decoder's 2D
// inverse, before rounding).
static void forward_2d(const int32_t* res, int n, int tx_type, double* out) {
  const int n0 = 1 << n;
  const int row_kind = (tx_type == DCT_DCT || tx_type == ADST_DCT) ? 0 : 1;
  const int col_kind = (tx_type == DCT_DCT || tx_type == DCT_ADST) ? 0 : 1;
  const std::vector<double>& ic = fwd_tables().inv[n - 2][col_kind];
  const std::vector<double>& ir = fwd_tables().inv[n - 2][row_kind];
  const double scale = (double)(1 << std::min(n + 2, 6));
  double tmp[32 * 32];
  // tmp = inv_col * R
  for (int i = 0; i < n0; ++i)
    for (int j = 0; j < n0; ++j) {
      double s = 0;
      for (int k = 0; k < n0; ++k) s += ic[(size_t)i * n0 + k] * res[k * n0 + j];
      tmp[i * n0 + j] = s * scale;
    }
  // out = tmp * inv_row^T
  for (int i = 0; i < n0; ++i)
    for (int j = 0; j < n0; ++j) {
      double s = 0;
      for (int k = 0; k < n0; ++k) s += tmp[i * n0 + k] * ir[(size_t)j * n0 + k];
      out[i * n0 + j] = s;
    }
}

// ---------------------------------------------------------------------------
// The encoder.

static const uint16_t* scan_of(int tx_sz, int tx_type) { return rv9::syn::get_scan(tx_sz, tx_type); }

struct TxStore {
  int plane;
  uint32_t x, y;
  int32_t lv[1024];
};

struct FrameEnc;

struct TileHooks final : rv9::syn::EncHooks {
  FrameEnc* fe = nullptr;
  uint32_t col_start = 0, col_end = 0;
  std::vector<TxStore> tx;
  size_t tx_used = 0, cursor = 0;
  int partition(uint32_t r, uint32_t c, uint8_t bsize, bool has_rows, bool has_cols) override;
  void analyze(uint32_t r, uint32_t c, uint8_t bsize, rv9::syn::EncBlock* eb) override;
  int inter_mode(const rv9::syn::BlockState& b, const rv9::syn::EncBlock* eb) override;
  const int32_t* tx_coefs(const rv9::syn::EncBlock* eb, int plane, uint32_t x, uint32_t y, int tx_sz,
                          const uint16_t* scan, int* eob) override;
  void code_residual(uint32_t r, uint32_t c, uint8_t bsize, rv9::syn::EncBlock* eb);
  void choose_intra(uint32_t r, uint32_t c, uint8_t bsize, rv9::syn::EncBlock* eb);
  int64_t motion_search(uint32_t r, uint32_t c, uint8_t bsize, int ref, Mv* best, uint8_t* filter);
};

struct FrameEnc {
  rv9_gen_config cfg;
  const Picture16* src = nullptr;
  Picture16* rec = nullptr;
  const Picture16* refs[3] = {nullptr, nullptr, nullptr};
  bool golden_ok = false;
  bool intra = false;
  uint32_t mi_cols = 0, mi_rows = 0, frame_no = 0;
  int q = 0;
  int32_t dc_q[2], ac_q[2];
  std::vector<Mv> mv_field;        // per 8x8, the block's motion vector
  std::vector<int8_t> ref_field;   // per 8x8, its reference (0 intra)
};

static inline uint32_t hash3(uint32_t a, uint32_t b, uint32_t c) { return hash32(a * 73856093u ^ b * 19349663u ^ c); }

static int64_t block_variance(const Picture16& s, int x0, int y0, int w, int h) {
  x0 = std::min(x0, s.width - 1);
  y0 = std::min(y0, s.height - 1);
  w = std::min(w, s.width - x0);
  h = std::min(h, s.height - y0);
  int64_t sum = 0, sq = 0;
  for (int y = 0; y < h; ++y) {
    const uint16_t* row = s.p[0].row(y0 + y) + x0;
    for (int x = 0; x < w; ++x) {
      sum += row[x];
      sq += (int64_t)row[x] * row[x];
    }
  }
  int64_t n = (int64_t)w * h;
  return n ? (sq - sum * sum / n) / n : 0;
}

int TileHooks::partition(uint32_t r, uint32_t c, uint8_t bsize, bool has_rows, bool has_cols) {
  if (!has_rows || !has_cols || bsize == BLOCK_8X8) return bsize == BLOCK_8X8 ? PARTITION_NONE : PARTITION_SPLIT;
  const FrameEnc& f = *fe;
  int size = 8 * vp9t_num_8x8_wide[bsize];
  int64_t var = block_variance(*f.src, c * 8, r * 8, size, size) >> (2 * (f.cfg.bit_depth - 8));
  // Split where the content is busy, more readily at lower quantisers; a
  // hashed fraction of the decisions is flipped so every size occurs.
  int64_t thresh = (int64_t)(size == 64 ? 60 : size == 32 ? 150 : 400) * (f.q + 20) / 60;
  uint32_t hsh = hash3(r, c, f.frame_no * 131 + bsize);
  bool split = var > thresh;
  if ((hsh & 15) == 0) split = !split;
  if (split) return PARTITION_SPLIT;
  // Rectangular halves now and then, where the chroma format allows them.
  int sx = f.cfg.ss_x, sy = f.cfg.ss_y;
  if (((hsh >> 4) & 7) == 0 && SS_SIZE_LOOKUP[SUBSIZE_LOOKUP[PARTITION_HORZ][bsize]][sx][sy] != BLOCK_INVALID)
    return PARTITION_HORZ;
  if (((hsh >> 4) & 7) == 1 && SS_SIZE_LOOKUP[SUBSIZE_LOOKUP[PARTITION_VERT][bsize]][sx][sy] != BLOCK_INVALID)
    return PARTITION_VERT;
  return PARTITION_NONE;
}

static int uv_tx_of(int bsize, int tx_size, int ss_x, int ss_y) {
  if (bsize < BLOCK_8X8) return TX_4X4;
  int uv = SS_SIZE_LOOKUP[bsize][ss_x][ss_y];
  return std::min<int>(tx_size, MAX_TXSIZE_LOOKUP[uv]);
}

static int64_t sad_region(const Plane16& a, const Plane16& b, int x, int y, int w, int h) {
  int64_t s = 0;
  for (int i = 0; i < h; ++i) {
    const uint16_t* pa = a.row(y + i) + x;
    const uint16_t* pb = b.row(y + i) + x;
    for (int j = 0; j < w; ++j) s += std::abs((int)pa[j] - (int)pb[j]);
  }
  return s;
}

void TileHooks::choose_intra(uint32_t r, uint32_t c, uint8_t bsize, rv9::syn::EncBlock* eb) {
  FrameEnc& f = *fe;
  int max_tx = MAX_TXSIZE_LOOKUP[bsize];
  uint32_t hsh = hash3(r + 7, c + 3, f.frame_no);
  eb->tx_size = (uint8_t)((max_tx > 0 && (hsh % 10) < 3) ? max_tx - 1 : max_tx);
  int tx = eb->tx_size, size = 4 << tx;
  bool have_left = c > col_start, have_above = r > 0;
  int n4w = vp9t_num_4x4_wide[bsize];
  bool not_on_right = (1 << tx) < n4w;
  int max_x = (int)(f.mi_cols * 8) - 1, max_y = (int)(f.mi_rows * 8) - 1;
  int x0 = c * 8, y0 = r * 8;
  int ew = std::min(size, f.src->width - x0), eh = std::min(size, f.src->height - y0);
  int64_t best = INT64_MAX;
  int best_mode = DC_PRED;
  for (int mode = 0; mode < 10; ++mode) {
    intra_pred(f.rec->p[0], mode, x0, y0, tx, have_left, have_above, not_on_right, max_x, max_y, f.cfg.bit_depth);
    int64_t s = sad_region(f.rec->p[0], f.src->p[0], x0, y0, std::max(ew, 1), std::max(eh, 1));
    s += (mode != DC_PRED) * (int64_t)size;  // a small bias toward DC
    if (s < best) {
      best = s;
      best_mode = mode;
    }
  }
  eb->y_mode = (uint8_t)best_mode;
  for (int i = 0; i < 4; ++i) eb->sub_modes[i] = (uint8_t)best_mode;
  // Chroma mode: the best of DC, V, H, TM and the luma mode on U.
  int utx = uv_tx_of(bsize, tx, f.cfg.ss_x, f.cfg.ss_y), usize = 4 << utx;
  int ux0 = x0 >> f.cfg.ss_x, uy0 = y0 >> f.cfg.ss_y;
  int umax_x = (int)((f.mi_cols * 8) >> f.cfg.ss_x) - 1, umax_y = (int)((f.mi_rows * 8) >> f.cfg.ss_y) - 1;
  int uw = std::max(1, std::min(usize, f.src->pw(1) - ux0)), uh = std::max(1, std::min(usize, f.src->ph(1) - uy0));
  int pnw = vp9t_num_4x4_wide[SS_SIZE_LOOKUP[bsize][f.cfg.ss_x][f.cfg.ss_y]];
  best = INT64_MAX;
  int cands[5] = {DC_PRED, V_PRED, H_PRED, TM_PRED, best_mode};
  eb->uv_mode = DC_PRED;
  for (int m : cands) {
    intra_pred(f.rec->p[1], m, ux0, uy0, utx, have_left, have_above, (1 << utx) < pnw, umax_x, umax_y,
               f.cfg.bit_depth);
    int64_t s = sad_region(f.rec->p[1], f.src->p[1], ux0, uy0, uw, uh);
    if (s < best) {
      best = s;
      eb->uv_mode = (uint8_t)m;
    }
  }
}

// Integer diamond search then half- and quarter-sample refinement and the
// filter choice, on luma. Motion vectors in 1/8 samples, always even.
int64_t TileHooks::motion_search(uint32_t r, uint32_t c, uint8_t bsize, int ref, Mv* best_mv, uint8_t* filter) {
  FrameEnc& f = *fe;
  const Picture16& rp = *f.refs[ref - 1];
  const Picture16& s = *f.src;
  int w = 8 * vp9t_num_8x8_wide[bsize], h = 8 * vp9t_num_8x8_high[bsize];
  int x0 = c * 8, y0 = r * 8;
  int ew = std::max(1, std::min(w, s.width - x0)), eh = std::max(1, std::min(h, s.height - y0));
  auto sad_int = [&](int dx, int dy) {
    int64_t acc = 0;
    if (x0 + dx >= 0 && x0 + dx + ew <= rp.width && y0 + dy >= 0 && y0 + dy + eh <= rp.height) {
      // The window inside the reference: the same sums without the clamps.
      for (int i = 0; i < eh; ++i) {
        const uint16_t* ps = s.p[0].row(y0 + i) + x0;
        const uint16_t* pr = rp.p[0].row(y0 + i + dy) + x0 + dx;
        int32_t row = 0;  // at most 64 samples of 12 bits
        for (int j = 0; j < ew; ++j) row += std::abs((int)ps[j] - (int)pr[j]);
        acc += row;
      }
      return acc;
    }
    for (int i = 0; i < eh; ++i) {
      const uint16_t* ps = s.p[0].row(y0 + i) + x0;
      const uint16_t* pr = rp.p[0].row(std::min(std::max(y0 + i + dy, 0), rp.height - 1));
      for (int j = 0; j < ew; ++j) acc += std::abs((int)ps[j] - (int)pr[std::min(std::max(x0 + j + dx, 0), rp.width - 1)]);
    }
    return acc;
  };
  // Predictors: zero, left and above neighbours on the same reference.
  std::vector<Mv> preds = {{0, 0}};
  if (c > col_start && f.ref_field[(size_t)r * f.mi_cols + c - 1] == ref) preds.push_back(f.mv_field[(size_t)r * f.mi_cols + c - 1]);
  if (r > 0 && f.ref_field[(size_t)(r - 1) * f.mi_cols + c] == ref) preds.push_back(f.mv_field[(size_t)(r - 1) * f.mi_cols + c]);
  int bx = 0, by = 0;
  int64_t bs = INT64_MAX;
  for (const Mv& p : preds) {
    int dx = (p.c + (p.c >= 0 ? 4 : -4)) / 8, dy = (p.r + (p.r >= 0 ? 4 : -4)) / 8;
    int64_t v = sad_int(dx, dy);
    if (v < bs) {
      bs = v;
      bx = dx;
      by = dy;
    }
  }
  const int range = 48;
  for (int step = 8; step >= 1; step >>= 1) {
    bool moved = true;
    int iter = 0;
    while (moved && iter++ < 16) {
      moved = false;
      const int d[4][2] = {{step, 0}, {-step, 0}, {0, step}, {0, -step}};
      for (auto& o : d) {
        int nx = bx + o[0], ny = by + o[1];
        if (std::abs(nx) > range || std::abs(ny) > range) continue;
        int64_t v = sad_int(nx, ny);
        if (v < bs) {
          bs = v;
          bx = nx;
          by = ny;
          moved = true;
        }
      }
    }
  }
  // Subsample refinement with the real prediction (regular filter), then the
  // filter choice.
  Mv cur{by * 8, bx * 8};
  std::vector<uint16_t> pred((size_t)w * h);
  int64_t xs = 1 << 14;
  auto cost = [&](Mv mv, int filt) {
    RefPos p = ref_position(mv.r, mv.c, 0, x0, y0, r, c, bsize, f.mi_rows, f.mi_cols, f.cfg.ss_x, f.cfg.ss_y, xs, xs);
    inter_pred(rp.p[0], rp.width - 1, rp.height - 1, p, w, h, filt, f.cfg.bit_depth, pred.data(), w);
    int64_t acc = 0;
    for (int i = 0; i < eh; ++i) {
      const uint16_t* ps = s.p[0].row(y0 + i) + x0;
      for (int j = 0; j < ew; ++j) acc += std::abs((int)ps[j] - (int)pred[(size_t)i * w + j]);
    }
    return acc;
  };
  int64_t cb = cost(cur, EIGHTTAP);
  for (int step = 4; step >= 2; step >>= 1) {
    Mv base = cur;
    for (int dy = -step; dy <= step; dy += step)
      for (int dx = -step; dx <= step; dx += step) {
        if (!dx && !dy) continue;
        Mv m{base.r + dy, base.c + dx};
        int64_t v = cost(m, EIGHTTAP);
        if (v < cb) {
          cb = v;
          cur = m;
        }
      }
  }
  *filter = EIGHTTAP;
  if ((cur.r & 15) || (cur.c & 15)) {
    for (int filt : {EIGHTTAP_SMOOTH, EIGHTTAP_SHARP}) {
      int64_t v = cost(cur, filt);
      if (v < cb) {
        cb = v;
        *filter = (uint8_t)filt;
      }
    }
  } else if ((hash3(r, c, f.frame_no + 5) & 3) == 0) {
    // Whole-sample vectors predict the same with any filter: vary it.
    *filter = (uint8_t)(hash3(c, r, f.frame_no) % 3);
  }
  *best_mv = cur;
  return cb;
}

void TileHooks::analyze(uint32_t r, uint32_t c, uint8_t bsize, rv9::syn::EncBlock* eb) {
  FrameEnc& f = *fe;
  *eb = rv9::syn::EncBlock();
  tx_used = 0;
  cursor = 0;
  if (f.intra) {
    choose_intra(r, c, bsize, eb);
  } else {
    Mv mv;
    uint8_t filt;
    int64_t cost = motion_search(r, c, bsize, LAST_FRAME, &mv, &filt);
    int ref = LAST_FRAME;
    if (f.golden_ok) {
      Mv mv2;
      uint8_t filt2;
      int64_t c2 = motion_search(r, c, bsize, GOLDEN_FRAME, &mv2, &filt2);
      if (c2 < cost) {
        cost = c2;
        mv = mv2;
        filt = filt2;
        ref = GOLDEN_FRAME;
      }
    }
    // Intra where prediction from the references fails.
    int w = 8 * vp9t_num_8x8_wide[bsize];
    int64_t per_px = cost / (w * 8 * vp9t_num_8x8_high[bsize]);
    bool go_intra = per_px > (12 << (f.cfg.bit_depth - 8)) || (hash3(r, c, f.frame_no * 7) % 61) == 0;
    if (go_intra) {
      choose_intra(r, c, bsize, eb);
      eb->is_inter = false;
    } else {
      eb->is_inter = true;
      eb->ref_frame[0] = (int8_t)ref;
      eb->ref_frame[1] = NONE_FRAME;
      eb->mv[0] = mv;
      eb->interp_filter = filt;
      eb->y_mode = NEWMV;
      int max_tx = MAX_TXSIZE_LOOKUP[bsize];
      uint32_t hsh = hash3(r + 11, c + 5, f.frame_no);
      eb->tx_size = (uint8_t)((max_tx > 0 && (hsh % 10) < 3) ? max_tx - 1 : max_tx);
    }
  }
  code_residual(r, c, bsize, eb);
  // Remember the block's vector for its neighbours' searches.
  uint32_t bw = vp9t_num_8x8_wide[bsize], bh = vp9t_num_8x8_high[bsize];
  for (uint32_t y = r; y < std::min(r + bh, f.mi_rows); ++y)
    for (uint32_t x = c; x < std::min(c + bw, f.mi_cols); ++x) {
      f.mv_field[(size_t)y * f.mi_cols + x] = eb->mv[0];
      f.ref_field[(size_t)y * f.mi_cols + x] = eb->is_inter ? eb->ref_frame[0] : 0;
    }
}

// Prediction, transform, quantisation and reconstruction of a block, in the
// residual syntax's order (spec 6.4.21-6.4.23).
void TileHooks::code_residual(uint32_t r, uint32_t c, uint8_t bsize, rv9::syn::EncBlock* eb) {
  FrameEnc& f = *fe;
  const int bd = f.cfg.bit_depth;
  const int bsize8 = std::max<int>(bsize, BLOCK_8X8);
  bool any = false;
  for (int plane = 0; plane < 3; ++plane) {
    int tx_sz = plane ? uv_tx_of(bsize, eb->tx_size, f.cfg.ss_x, f.cfg.ss_y) : eb->tx_size;
    int step = 1 << tx_sz, n = 2 + tx_sz, n0 = 1 << n;
    int sx = plane ? f.cfg.ss_x : 0, sy = plane ? f.cfg.ss_y : 0;
    int psz = SS_SIZE_LOOKUP[bsize8][sx][sy];
    int n4w = vp9t_num_4x4_wide[psz], n4h = vp9t_num_4x4_high[psz];
    int base_x = (c * 8) >> sx, base_y = (r * 8) >> sy;
    Plane16& rec = f.rec->p[plane];
    const Plane16& src = f.src->p[plane];
    if (eb->is_inter) {
      const Picture16& rp = *f.refs[eb->ref_frame[0] - 1];
      RefPos p = ref_position(eb->mv[0].r, eb->mv[0].c, plane, base_x, base_y, r, c, bsize, f.mi_rows, f.mi_cols,
                              f.cfg.ss_x, f.cfg.ss_y, 1 << 14, 1 << 14);
      inter_pred(rp.p[plane], rp.pw(plane) - 1, rp.ph(plane) - 1, p, n4w * 4, n4h * 4, eb->interp_filter, bd,
                 rec.row(base_y) + base_x, rec.stride);
    }
    int max_x = (int)((f.mi_cols * 8) >> sx), max_y = (int)((f.mi_rows * 8) >> sy);
    int pw = f.src->pw(plane), ph = f.src->ph(plane);
    int mode_y = eb->y_mode;
    int block_idx = 0;
    for (int y = 0; y < n4h; y += step)
      for (int x = 0; x < n4w; x += step) {
        int xs = base_x + 4 * x, ys = base_y + 4 * y;
        if (xs < max_x && ys < max_y) {
          if (!eb->is_inter)
            intra_pred(rec, plane ? eb->uv_mode : mode_y, xs, ys, tx_sz, (c > col_start) || x > 0, r > 0 || y > 0,
                       x + step < n4w, max_x - 1, max_y - 1, bd);
          int tx_type = DCT_DCT;
          if (plane == 0 && !eb->is_inter && tx_sz != TX_32X32) tx_type = MODE2TXFM_MAP[mode_y];
          int32_t res[1024];
          for (int i = 0; i < n0; ++i)
            for (int j = 0; j < n0; ++j) {
              int sv = src.row(std::min(ys + i, ph - 1))[std::min(xs + j, pw - 1)];
              res[i * n0 + j] = sv - (int)rec.row(ys + i)[xs + j];
            }
          double coef[1024];
          forward_2d(res, n, tx_type, coef);
          if (tx_used == tx.size()) tx.emplace_back();
          TxStore& ts = tx[tx_used++];
          ts.plane = plane;
          ts.x = (uint32_t)xs;
          ts.y = (uint32_t)ys;
          const int pt = plane ? 1 : 0;
          int32_t dq[1024];
          bool nz = false;
          for (int i = 0; i < n0 * n0; ++i) {
            double q = (i == 0 ? f.dc_q[pt] : f.ac_q[pt]) / (tx_sz == TX_32X32 ? 2.0 : 1.0);
            double v = coef[i] / q;
            double a = fabs(v);
            int32_t l = (int32_t)(a + (i == 0 ? 0.5 : 0.35));
            l = std::min(l, 16000);
            ts.lv[i] = v < 0 ? -l : l;
            int64_t d = (int64_t)ts.lv[i] * (i == 0 ? f.dc_q[pt] : f.ac_q[pt]);
            if (tx_sz == TX_32X32) d /= 2;
            dq[i] = (int32_t)std::min<int64_t>(std::max<int64_t>(d, INT32_MIN), INT32_MAX);
            nz |= l != 0;
          }
          if (nz) {
            const uint16_t* sc = scan_of(tx_sz, tx_type);
            int eob = 0;
            for (int k = 0; k < n0 * n0; ++k)
              if (ts.lv[sc[k]] != 0) eob = k + 1;
            itx_add(dq, n, tx_type, eob, bd, rec.row(ys) + xs, rec.stride);
            any = true;
          }
        }
        ++block_idx;
      }
  }
  eb->skip = !any;
  if (eb->skip && eb->is_inter) eb->tx_size = MAX_TXSIZE_LOOKUP[bsize];
}

int TileHooks::inter_mode(const rv9::syn::BlockState& b, const rv9::syn::EncBlock* eb) {
  const Mv& mv = eb->mv[0];
  if (mv == b.nearest_mv[0]) return NEARESTMV;
  if (mv == b.near_mv[0]) return NEARMV;
  if (mv.r == 0 && mv.c == 0) return ZEROMV;
  return NEWMV;
}

const int32_t* TileHooks::tx_coefs(const rv9::syn::EncBlock*, int plane, uint32_t x, uint32_t y, int tx_sz,
                                   const uint16_t* scan, int* eob) {
  // The transform blocks come in analysis order.
  while (cursor < tx_used && !(tx[cursor].plane == plane && tx[cursor].x == x && tx[cursor].y == y)) ++cursor;
  const TxStore& ts = tx[cursor < tx_used ? cursor : 0];
  const int count = 16 << (2 * tx_sz);
  int e = 0;
  for (int k = 0; k < count; ++k)
    if (ts.lv[scan[k]] != 0) e = k + 1;
  *eob = e;
  ++cursor;
  return ts.lv;
}

// ---------------------------------------------------------------------------
// Headers.

struct BitWriter {
  std::vector<uint8_t> buf;
  size_t nbits = 0;
  void bit(uint32_t b) {
    if ((nbits & 7) == 0) buf.push_back(0);
    if (b) buf.back() |= (uint8_t)(0x80 >> (nbits & 7));
    ++nbits;
  }
  void f(uint32_t v, int n) {
    for (int i = n - 1; i >= 0; --i) bit((v >> i) & 1);
  }
};

struct Encoder {
  rv9_gen_config cfg;
  Picture16 refs[8];
  uint32_t frame_no = 0;
  Picture16 last_rec;
  std::vector<rv9::syn::PrevMv> prev_mvs;  // the last frame's, when frames are not error-resilient

  std::vector<uint8_t> encode(const Picture16& src);
};

std::vector<uint8_t> Encoder::encode(const Picture16& src) {
  const bool key = frame_no == 0;
  const bool golden = !key && cfg.golden_interval && (frame_no % cfg.golden_interval) == 0;
  const int q = golden ? std::max(1, cfg.base_q_idx * 3 / 4) : cfg.base_q_idx;
  const int profile = (cfg.bit_depth > 8 ? 2 : 0) + ((cfg.ss_x && cfg.ss_y) ? 0 : 1);
  const uint32_t mi_cols = (cfg.width + 7) >> 3, mi_rows = (cfg.height + 7) >> 3;
  const uint32_t sb64_cols = (mi_cols + 7) >> 3, sb64_rows = (mi_rows + 7) >> 3;
  uint32_t min_log2 = 0;
  while ((MAX_TILE_WIDTH_B64 << min_log2) < sb64_cols) ++min_log2;
  uint32_t max_log2 = 1;
  while ((sb64_cols >> max_log2) >= MIN_TILE_WIDTH_B64) ++max_log2;
  --max_log2;
  uint32_t tcl = std::min(std::max(cfg.tile_cols_log2, min_log2), std::max(max_log2, min_log2));
  const int lf_level = std::min(63, q * 10 / 48);
  const uint8_t refresh = key ? 0xff : (uint8_t)(golden ? 0x03 : 0x01);
  const bool nonres = cfg.non_resilient != 0;
  const uint32_t ai = cfg.adapt_interval;
  const bool adapt = nonres && !key && ai && frame_no % ai == 0 && frame_no / ai <= 3;
  const uint32_t ctx_idx = adapt ? frame_no / ai : 0;
  // Uncompressed header (spec 6.2).
  BitWriter w;
  w.f(2, 2);
  w.f(profile & 1, 1);
  w.f(profile >> 1, 1);
  if (profile == 3) w.f(0, 1);
  w.f(0, 1);  // show_existing_frame
  w.f(key ? 0 : 1, 1);
  w.f(1, 1);  // show_frame
  w.f(nonres ? 0 : 1, 1);  // error_resilient_mode
  if (key) {
    w.f(0x49, 8);
    w.f(0x83, 8);
    w.f(0x42, 8);
    if (profile >= 2) w.f(cfg.bit_depth == 12 ? 1 : 0, 1);
    w.f(cfg.color_space ? std::min<uint32_t>(cfg.color_space, 6) : 2, 3);  // BT.709 unless asked (7, sRGB, is not written)
    w.f(0, 1);  // studio swing
    if (profile == 1 || profile == 3) {
      w.f(cfg.ss_x, 1);
      w.f(cfg.ss_y, 1);
      w.f(0, 1);
    }
    w.f(cfg.width - 1, 16);
    w.f(cfg.height - 1, 16);
    w.f(0, 1);  // render size = frame size
  } else {
    if (nonres) w.f(0, 2);  // reset_frame_context
    w.f(refresh, 8);
    for (int i = 0; i < 3; ++i) {
      w.f((uint32_t)i, 3);  // LAST slot 0, GOLDEN slot 1, ALTREF slot 2
      w.f(0, 1);            // sign bias
    }
    w.f(1, 1);  // frame size from LAST
    w.f(0, 1);  // render size
    w.f(0, 1);  // allow_high_precision_mv
    w.f(1, 1);  // switchable interpolation filter
  }
  if (nonres) {
    w.f(adapt ? 1 : 0, 1);  // refresh_frame_context
    w.f(adapt ? 0 : 1, 1);  // frame_parallel_decoding_mode
  }
  w.f(ctx_idx, 2);  // frame_context_idx
  w.f((uint32_t)lf_level, 6);
  w.f(0, 3);  // sharpness
  w.f(1, 1);  // loop_filter_delta_enabled (the defaults)
  w.f(0, 1);  // no delta update
  w.f((uint32_t)q, 8);
  w.f(0, 1);
  w.f(0, 1);
  w.f(0, 1);  // no delta_q
  w.f(0, 1);  // segmentation off
  for (uint32_t i = min_log2; i < tcl; ++i) w.f(1, 1);
  if (tcl < max_log2) w.f(0, 1);
  w.f(0, 1);  // one tile row
  // Compressed header (spec 6.3): TX_MODE_SELECT, no probability updates.
  rv9::syn::BoolEncoder ch;
  ch.reset();
  ch.write(false, 128);  // marker
  ch.literal(ALLOW_32X32, 2);
  ch.literal(1, 1);  // tx_mode_select
  for (int i = 0; i < 12; ++i) ch.write(false, 252);  // tx probs
  for (int t = 0; t < 4; ++t) ch.literal(0, 1);       // coef probs
  for (int i = 0; i < 3; ++i) ch.write(false, 252);   // skip
  if (!key) {
    for (int i = 0; i < 21; ++i) ch.write(false, 252);  // inter mode
    for (int i = 0; i < 8; ++i) ch.write(false, 252);   // interp filter
    for (int i = 0; i < 4; ++i) ch.write(false, 252);   // is_inter
    for (int i = 0; i < 10; ++i) ch.write(false, 252);  // single ref
    for (int i = 0; i < 36; ++i) ch.write(false, 252);  // y mode
    for (int i = 0; i < 48; ++i) ch.write(false, 252);  // partition
    for (int i = 0; i < 3 + 2 * (1 + 10 + 1 + 10) + 2 * (6 + 3); ++i) ch.write(false, 252);  // mv
  }
  std::vector<uint8_t> comp = ch.finish();
  w.f((uint32_t)comp.size(), 16);
  std::vector<uint8_t> out = w.buf;
  out.insert(out.end(), comp.begin(), comp.end());
  // Tiles.
  rv9::syn::FrameHeader h;
  h.frame_is_intra = key;
  h.tx_mode = TX_MODE_SELECT;
  h.mi_cols = mi_cols;
  h.mi_rows = mi_rows;
  h.sb64_cols = sb64_cols;
  h.sb64_rows = sb64_rows;
  h.ss_x = cfg.ss_x;
  h.ss_y = cfg.ss_y;
  h.bit_depth = cfg.bit_depth;
  h.interpolation_filter = SWITCHABLE;
  h.reference_mode = SINGLE_REFERENCE;
  h.error_resilient_mode = !nonres;
  h.frame_parallel_decoding_mode = !adapt;
  h.tile_cols_log2 = tcl;
  h.tile_rows_log2 = 0;
  h.base_q_idx = q;
  rv9::syn::SegParams seg;
  rv9::Probs probs;
  probs.set_default();
  std::vector<rv9::MiInfo> mi((size_t)mi_rows * mi_cols);
  std::vector<uint8_t> an[3], ap(sb64_cols * 8 + 8, 0), asp(sb64_cols * 8 + 8, 0);
  for (auto& a : an) a.assign(sb64_cols * 16 + 16, 0);
  rv9::syn::FrameCtx fc;
  fc.h = &h;
  fc.seg = &seg;
  fc.probs = &probs;
  fc.prev_seg_ids = nullptr;
  fc.prev_seg_len = 0;
  fc.prev_mvs = nonres && !key && prev_mvs.size() == (size_t)mi_rows * mi_cols ? prev_mvs.data() : nullptr;
  fc.mi = mi.data();
  for (int p = 0; p < 3; ++p) fc.above_nonzero[p] = an[p].data();
  fc.above_partition = ap.data();
  fc.above_seg_pred = asp.data();
  fc.ref_scale_ok[0] = fc.ref_scale_ok[1] = fc.ref_scale_ok[2] = true;
  fc.count_coefs = false;
  Picture16 rec;
  rec.alloc(cfg.width, cfg.height, cfg.ss_x, cfg.ss_y, cfg.bit_depth);
  FrameEnc fe;
  fe.cfg = cfg;
  fe.src = &src;
  fe.rec = &rec;
  fe.intra = key;
  fe.golden_ok = !key && frame_no >= 1;
  fe.mi_cols = mi_cols;
  fe.mi_rows = mi_rows;
  fe.frame_no = frame_no;
  fe.q = q;
  int bd_idx = (cfg.bit_depth - 8) >> 1;
  fe.dc_q[0] = fe.dc_q[1] = vp9t_dc_qlookup[bd_idx][q];
  fe.ac_q[0] = fe.ac_q[1] = vp9t_ac_qlookup[bd_idx][q];
  fe.mv_field.assign((size_t)mi_rows * mi_cols, Mv{0, 0});
  fe.ref_field.assign((size_t)mi_rows * mi_cols, 0);
  if (!key)
    for (int i = 0; i < 3; ++i) fe.refs[i] = &refs[i];
  uint32_t tile_cols = 1u << tcl;
  std::vector<std::unique_ptr<rv9::syn::TileCoder<rv9::syn::EncCoder>>> tcs(tile_cols);
  std::vector<TileHooks> hooks(tile_cols);
  std::vector<rv9::syn::EncBlock> ebs(tile_cols);
  std::vector<std::vector<uint8_t>> tile_bytes(tile_cols);
  auto run = [&](uint32_t col) {
    auto& tc = tcs[col];
    tc.reset(new rv9::syn::TileCoder<rv9::syn::EncCoder>());
    tc->init(&fc);
    hooks[col].fe = &fe;
    hooks[col].col_start = rv9::syn::tile_offset(col, mi_cols, tcl);
    hooks[col].col_end = rv9::syn::tile_offset(col + 1, mi_cols, tcl);
    tc->enc_ = &hooks[col];
    tc->eb_ = &ebs[col];
    tc->mi_row_start = 0;
    tc->mi_row_end = mi_rows;
    tc->mi_col_start = hooks[col].col_start;
    tc->mi_col_end = hooks[col].col_end;
    rv9::syn::EncCoder coder;
    coder.be.reset();
    coder.be.write(false, 128);  // marker
    tc->decode_tile(coder);
    tile_bytes[col] = coder.be.finish();
  };
  unsigned nth = cfg.threads ? cfg.threads : std::max(1u, std::thread::hardware_concurrency());
  if (nth > 1 && tile_cols > 1) {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < std::min<unsigned>(nth, tile_cols); ++t)
      th.emplace_back([&, t]() {
        for (uint32_t col = t; col < tile_cols; col += std::min<unsigned>(nth, tile_cols)) run(col);
      });
    for (auto& t : th) t.join();
  } else {
    for (uint32_t col = 0; col < tile_cols; ++col) run(col);
  }
  for (uint32_t col = 0; col < tile_cols; ++col) {
    const std::vector<uint8_t>& tb = tile_bytes[col];
    if (col + 1 < tile_cols) {
      uint32_t n = (uint32_t)tb.size();
      out.push_back((uint8_t)(n >> 24));
      out.push_back((uint8_t)(n >> 16));
      out.push_back((uint8_t)(n >> 8));
      out.push_back((uint8_t)n);
    }
    out.insert(out.end(), tb.begin(), tb.end());
  }
  // Loop filter with the mode info as written, then the reference update.
  std::vector<rv9_block> blocks;
  for (uint32_t col = 0; col < tile_cols; ++col) blocks.insert(blocks.end(), tcs[col]->blocks.begin(), tcs[col]->blocks.end());
  rv9_frame_desc d;
  memset(&d, 0, sizeof d);
  d.width = cfg.width;
  d.height = cfg.height;
  d.mi_cols = mi_cols;
  d.mi_rows = mi_rows;
  d.sb64_cols = sb64_cols;
  d.sb64_rows = sb64_rows;
  d.ss_x = (uint8_t)cfg.ss_x;
  d.ss_y = (uint8_t)cfg.ss_y;
  d.bit_depth = (uint8_t)cfg.bit_depth;
  d.lf_level = (uint8_t)lf_level;
  d.lf_delta_enabled = 1;
  d.lf_ref_deltas[0] = 1;
  d.lf_ref_deltas[1] = 0;
  d.lf_ref_deltas[2] = -1;
  d.lf_ref_deltas[3] = -1;
  if (lf_level) loop_filter(rec, d, blocks.data(), blocks.size());
  for (int i = 0; i < 8; ++i)
    if ((refresh >> i) & 1) refs[i] = rec;
  last_rec = rec;
  if (nonres) {
    // PrevMvs / PrevRefFrames for the next frame (spec 8.10 step 2).
    prev_mvs.resize(mi.size());
    for (size_t i = 0; i < mi.size(); ++i) {
      prev_mvs[i].ref_frame[0] = mi[i].ref_frame[0];
      prev_mvs[i].ref_frame[1] = mi[i].ref_frame[1];
      prev_mvs[i].mv[0] = mi[i].mv[0][3];
      prev_mvs[i].mv[1] = mi[i].mv[1][3];
    }
  }
  ++frame_no;
  return out;
}

// ---------------------------------------------------------------------------
// Loop filter (the kernels' superblock procedure, sequential).

void loop_filter(Picture16& pic, const rv9_frame_desc& d, const rv9_block* blocks, size_t n_blocks) {
  using namespace rv9g;
  uint8_t lvl[8][4][2];
  uint8_t lim[64], blim[64], thr[64];
  int n_shift = d.lf_level >> 5;
  for (int seg = 0; seg < 8; ++seg)
    for (int rf = 0; rf < 4; ++rf)
      for (int mode = 0; mode < 2; ++mode) {
        int v = d.lf_level;
        if (d.lf_delta_enabled) {
          v += d.lf_ref_deltas[rf] * (1 << n_shift);
          if (rf > 0) v += d.lf_mode_deltas[mode] * (1 << n_shift);
        }
        lvl[seg][rf][mode] = (uint8_t)std::min(std::max(v, 0), 63);
      }
  int shift = d.lf_sharpness > 4 ? 2 : (d.lf_sharpness > 0 ? 1 : 0);
  for (int l = 0; l < 64; ++l) {
    int limit = l >> shift;
    if (d.lf_sharpness > 0) limit = std::min(limit, 9 - (int)d.lf_sharpness);
    limit = std::max(limit, 1);
    lim[l] = (uint8_t)limit;
    blim[l] = (uint8_t)(2 * (l + 2) + limit);
    thr[l] = (uint8_t)(l >> 4);
  }
  std::vector<uint32_t> lf_mi((size_t)d.mi_rows * d.mi_cols);
  for (size_t i = 0; i < n_blocks; ++i) {
    const rv9_block& b = blocks[i];
    uint32_t v = lf_block_record(b.mi_size, b.tx_size, (b.flags & RV9_BLK_SKIP) ? 1 : 0, b.segment_id, b.y_mode,
                                 b.ref_frame[0], lvl, d.legacy_uv, d.ss_x, d.ss_y);
    uint32_t w8 = vp9t_num_8x8_wide[b.mi_size], h8 = vp9t_num_8x8_high[b.mi_size];
    for (uint32_t y = b.mi_row; y < std::min(b.mi_row + h8, d.mi_rows); ++y)
      for (uint32_t x = b.mi_col; x < std::min(b.mi_col + w8, d.mi_cols); ++x) lf_mi[(size_t)y * d.mi_cols + x] = v;
  }
  LfParams P{(int)d.mi_cols, (int)d.mi_rows, d.ss_x, d.ss_y, lf_mi.data(), lim, blim, thr};
  std::vector<int16_t> px((size_t)3 * 72 * 80);
  LfEdge edges[3][2][16][16];
  for (uint32_t sr = 0; sr < d.sb64_rows; ++sr)
    for (uint32_t sc = 0; sc < d.sb64_cols; ++sc) {
      int row = sr * 8, col = sc * 8;
      for (int i = 0; i < 3 * 2 * 256; ++i) {
        int plane = i / 512, pass = (i >> 8) & 1, ed = (i >> 4) & 15, rn = i & 15;
        edges[plane][pass][ed][rn] = lf_edge_entry(P, plane, pass, row, col, ed, rn);
      }
      int rows_p[3], cols_p[3], x0s[3], y0s[3];
      for (int p = 0; p < 3; ++p) {
        int sxp = p ? d.ss_x : 0, syp = p ? d.ss_y : 0;
        rows_p[p] = 64 >> syp;
        cols_p[p] = 64 >> sxp;
        x0s[p] = (col * 8) >> sxp;
        y0s[p] = (row * 8) >> syp;
        int16_t* t = &px[(size_t)p * 72 * 80];
        for (int r = 0; r < rows_p[p] + 8; ++r)
          for (int c = 0; c < cols_p[p] + 8; ++c) {
            int gy = y0s[p] - 8 + r, gx = x0s[p] - 8 + c;
            if (gy >= 0 && gx >= 0 && (r >= 8 || c >= 8)) t[r * 80 + c] = (int16_t)pic.p[p].row(gy)[gx];
          }
      }
      for (int p = 0; p < 3; ++p)
        for (int r = 0; r < rows_p[p]; ++r)
          lf_vertical_row(&px[(size_t)p * 72 * 80 + (8 + r) * 80], edges[p][0], 16 >> (p ? d.ss_x : 0), r >> 2,
                          d.bit_depth);
      for (int p = 0; p < 3; ++p)
        for (int c = 0; c < cols_p[p]; ++c)
          lf_horizontal_col(&px[(size_t)p * 72 * 80 + 8 + c], 80, 72, edges[p][1], 16 >> (p ? d.ss_y : 0), c >> 2,
                            d.bit_depth);
      for (int p = 0; p < 3; ++p) {
        const int16_t* t = &px[(size_t)p * 72 * 80];
        for (int r = 0; r < rows_p[p] + 8; ++r)
          for (int c = 0; c < cols_p[p] + 8; ++c) {
            int gy = y0s[p] - 8 + r, gx = x0s[p] - 8 + c;
            if (gy >= 0 && gx >= 0 && (r >= 8 || c >= 8)) pic.p[p].row(gy)[gx] = (uint16_t)t[r * 80 + c];
          }
      }
    }
}

static thread_local std::vector<uint8_t> g_last_rec;

}  // namespace rv9enc

extern "C" {

void rv9_gen_source_frame(const rv9_gen_config* cfg, uint32_t index, uint16_t* y, uint16_t* u, uint16_t* v) {
  rv9enc::source_frame(*cfg, index, y, u, v);
}

int rv9_gen_stream(const rv9_gen_config* cfg, uint8_t* out, size_t cap, size_t* sizes, size_t* total) {
  using namespace rv9enc;
  if (!cfg || cfg->width == 0 || cfg->height == 0 || (cfg->bit_depth != 8 && cfg->bit_depth != 10 &&
                                                      cfg->bit_depth != 12) ||
      cfg->base_q_idx < 1 || cfg->base_q_idx > 255 || cfg->ss_x > 1 || cfg->ss_y > 1)
    return -1;
  Encoder enc;
  enc.cfg = *cfg;
  *total = 0;
  const int w = cfg->width, h = cfg->height;
  const int cw = (w + (int)cfg->ss_x) >> cfg->ss_x, chh = (h + (int)cfg->ss_y) >> cfg->ss_y;
  std::vector<uint16_t> py((size_t)w * h), pu((size_t)cw * chh), pv((size_t)cw * chh);
  Picture16 src;
  src.alloc(w, h, cfg->ss_x, cfg->ss_y, cfg->bit_depth);
  for (uint32_t t = 0; t < cfg->frames; ++t) {
    source_frame(*cfg, t, py.data(), pu.data(), pv.data());
    for (int y = 0; y < h; ++y) memcpy(src.p[0].row(y), &py[(size_t)y * w], w * 2);
    for (int y = 0; y < chh; ++y) {
      memcpy(src.p[1].row(y), &pu[(size_t)y * cw], cw * 2);
      memcpy(src.p[2].row(y), &pv[(size_t)y * cw], cw * 2);
    }
    std::vector<uint8_t> pkt = enc.encode(src);
    if (*total + pkt.size() > cap) return -1;
    memcpy(out + *total, pkt.data(), pkt.size());
    *total += pkt.size();
    sizes[t] = pkt.size();
  }
  // The last reconstruction, packed.
  const Picture16& r = enc.last_rec;
  size_t bps = cfg->bit_depth > 8 ? 2 : 1;
  g_last_rec.clear();
  for (int p = 0; p < 3; ++p)
    for (int y = 0; y < r.ph(p); ++y)
      for (int x = 0; x < r.pw(p); ++x) {
        uint16_t v = r.p[p].row(y)[x];
        g_last_rec.push_back((uint8_t)(v & 0xff));
        if (bps == 2) g_last_rec.push_back((uint8_t)(v >> 8));
      }
  return 0;
}

size_t rv9_gen_last_reconstruction(uint8_t* out, size_t cap) {
  size_t n = rv9enc::g_last_rec.size();
  if (out && cap >= n) memcpy(out, rv9enc::g_last_rec.data(), n);
  return n;
}

}  // extern "C"

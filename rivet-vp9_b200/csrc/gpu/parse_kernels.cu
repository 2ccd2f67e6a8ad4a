// Kernels of the device parser: the tile columns' syntax (one thread per
// column) and, per frame, the gather of its columns' records and the build of
// the reconstruction engine's work lists (one CTA per frame).
#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <mutex>

#include "device_parse.h"
#include "parse_plan.h"

namespace rv9g {

// ---- Tables, once per device ----

cudaError_t parse_tables(int device, const tp::Tables** out) {
  static std::mutex mu;
  static const tp::Tables* by_device[64] = {nullptr};
  if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(mu);
  if (!by_device[device]) {
    std::unique_ptr<tp::Tables> h(new tp::Tables);
    tp::fill_tables(h.get());
    void* d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(tp::Tables));
    if (e != cudaSuccess) return e;
    e = cudaMemcpy(d, h.get(), sizeof(tp::Tables), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFree(d);
      return e;
    }
    by_device[device] = (const tp::Tables*)d;
  }
  *out = by_device[device];
  return cudaSuccess;
}

// ---- Tile columns ----

// One tile column per CTA of one warp; its first thread parses (the syntax
// is one serial chain of boolean decodes), with the token cache in shared
// memory.
__global__ void __launch_bounds__(32, 1) k_parse_chains(const tp::Tables* __restrict__ T,
                                                     const tp::FrameIn* __restrict__ frames,
                                                     const tp::Chain* __restrict__ chains, uint32_t first,
                                                     const tp::Span* __restrict__ spans,
                                                     const uint8_t* __restrict__ data, tp::Mi* mi, uint8_t* above,
                                                     const tp::PrevMv* prev, rv9_block* blocks, rv9_tok* toks,
                                                     uint32_t* coefs, tp::ChainOut* outs) {
  static_assert(sizeof(((tp::FrameIn*)0)->coef_pk) == sizeof(tp::tp_pkw_smem), "probability words");
  const uint32_t i = first + blockIdx.x;
  const tp::Chain ch = chains[i];
  // The frame's coefficient probabilities into the parser's shared array
  // (the warp), then the first thread parses.
  const uint32_t* src = reinterpret_cast<const uint32_t*>(frames[ch.frame].coef_pk);
  for (uint32_t k = threadIdx.x; k < sizeof(tp::tp_pkw_smem) / 4; k += 32) tp::tp_pkw_smem[k] = src[k];
  __syncwarp();
  if (threadIdx.x != 0) return;
  tp::parse_chain(T, frames, ch, spans, data, mi, above, prev, blocks, toks, coefs, tp::tp_tc_smem, tp::tp_pkw_smem,
                  &outs[i]);
}

cudaError_t launch_parse_chains(const tp::Tables* T, const tp::FrameIn* frames, const tp::Chain* chains,
                                uint32_t first, uint32_t n, const tp::Span* spans, const uint8_t* data, tp::Mi* mi,
                                uint8_t* above, const tp::PrevMv* prev, rv9_block* blocks, rv9_tok* toks,
                                uint32_t* coefs, tp::ChainOut* outs, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_parse_chains<<<n, 32, 0, s>>>(T, frames, chains, first, spans, data, mi, above, prev, blocks, toks, coefs, outs);
  return cudaGetLastError();
}

__global__ void k_mi_to_prev(const tp::Mi* __restrict__ mi, tp::PrevMv* __restrict__ prev, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    tp::PrevMv p;
    p.ref_frame[0] = mi[i].ref_frame[0];
    p.ref_frame[1] = mi[i].ref_frame[1];
    p.mv[0] = mi[i].mv[0][3];
    p.mv[1] = mi[i].mv[1][3];
    prev[i] = p;
  }
}

cudaError_t launch_mi_to_prev(const tp::Mi* mi, tp::PrevMv* prev, uint32_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const uint32_t grid = (n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184;
  k_mi_to_prev<<<grid, 256, 0, s>>>(mi, prev, n);
  return cudaGetLastError();
}


// ---- Work lists, one CTA per frame ----

constexpr int kBuildThreads = 1024;
constexpr uint32_t kMaxDiag = 1024;
constexpr uint32_t kMaxChains = 64;

struct BuildSmem {
  uint32_t warp_tot[32][8];
  uint32_t carry[8];
  uint32_t tot[8];  // pass A's totals: small units, large units, residuals by size, intra items
  uint32_t res_base[4];
  uint32_t chain_b[kMaxChains + 1], chain_t[kMaxChains + 1], chain_c[kMaxChains + 1];
  uint32_t diag[kMaxDiag];
  unsigned long long kb[4];  // inter, inter residual, intra, inter output bytes
  int32_t err;
  uint32_t err_tile;
};

// Exclusive scan of eight counters over the CTA's 1024 threads in thread
// order, continuing from S.carry (which then holds the running totals).
__device__ __forceinline__ void cta_scan8(uint32_t (&v)[8], BuildSmem& S) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    uint32_t x = v[k];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
      if (lane >= d) x += y;
    }
    inc[k] = x;
  }
  if (lane == 31)
#pragma unroll
    for (int k = 0; k < 8; ++k) S.warp_tot[warp][k] = inc[k];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      uint32_t x = S.warp_tot[lane][k];
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
      }
      S.warp_tot[lane][k] = x;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] = S.carry[k] + (warp ? S.warp_tot[warp - 1][k] : 0) + inc[k] - v[k];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < 8; ++k) S.carry[k] += S.warp_tot[31][k];
  __syncthreads();
}

struct WalkOut {
  uint32_t small, large, res[4], intra;
  uint64_t kb_inter, kb_res, kb_intra, out_bytes;
};

// One block's prediction regions, residuals and intra items (the loops of
// Engine::build_work): counted, or (EMIT) written at the given positions.
template <bool EMIT>
__device__ void walk_block(const tp::Tables* __restrict__ T, const BuildFrame& F, const rv9_block& b, uint32_t bi,
                           const rv9_tok* __restrict__ toks, WalkOut& w, InterUnit* units, uint32_t small_at,
                           uint32_t large_at, ResItem* res, const uint32_t* res_at, IntraItem* intra,
                           uint32_t intra_at) {
  const bool is_inter = b.flags & RV9_BLK_INTER;
  const bool avail_l = b.flags & RV9_BLK_AVAIL_L, avail_u = b.flags & RV9_BLK_AVAIL_U;
  const int bsize = b.mi_size < 3 ? 3 : b.mi_size;
  const int nrefs = b.ref_frame[1] > 0 ? 2 : 1;
  const uint64_t bps = F.bit_depth > 8 ? 2 : 1;
  uint32_t tok = b.tok_start;
  for (int plane = 0; plane < 3; ++plane) {
    int tx_sz = b.tx_size;
    if (plane) {
      if (b.mi_size < 3) {
        tx_sz = 0;
      } else {
        const int sx = F.legacy_uv ? 1 : (int)F.ss_x, sy = F.legacy_uv ? 1 : (int)F.ss_y;
        const int m = T->max_tx[T->ss_size[b.mi_size][sx][sy]];
        tx_sz = b.tx_size < m ? b.tx_size : m;
      }
    }
    const int step = 1 << tx_sz;
    const int sx = plane ? (int)F.ss_x : 0, sy = plane ? (int)F.ss_y : 0;
    const int plane_sz = T->ss_size[bsize][sx][sy];
    const int n4w = T->n4w[plane_sz], n4h = T->n4h[plane_sz];
    const uint32_t base_x = ((uint32_t)b.mi_col * 8) >> sx, base_y = ((uint32_t)b.mi_row * 8) >> sy;
    if (is_inter) {
      if (b.mi_size < 3) {
        for (int y = 0; y < n4h; ++y)
          for (int x = 0; x < n4w; ++x) {
            if (EMIT)
              units[small_at + w.small] = InterUnit{bi, (uint16_t)(base_x + 4 * x), (uint16_t)(base_y + 4 * y),
                                                    (uint8_t)plane, 1, 1, (uint8_t)(y * n4w + x)};
            ++w.small;
          }
      } else if (n4w <= 4 && n4h <= 4) {
        if (EMIT)
          units[small_at + w.small] = InterUnit{bi, (uint16_t)base_x, (uint16_t)base_y, (uint8_t)plane,
                                                (uint8_t)n4w, (uint8_t)n4h, 0};
        ++w.small;
      } else {
        if (EMIT)
          units[large_at + w.large] = InterUnit{bi, (uint16_t)base_x, (uint16_t)base_y, (uint8_t)plane,
                                                (uint8_t)n4w, (uint8_t)n4h, 0};
        ++w.large;
      }
      const uint64_t out = (uint64_t)n4w * n4h * 16 * bps;
      w.kb_inter += out * (nrefs + 1);
      w.out_bytes += out;
    }
    const uint32_t max_x = (F.mi_cols * 8) >> sx, max_y = (F.mi_rows * 8) >> sy;
    int block_idx = 0;
    for (int y = 0; y < n4h; y += step)
      for (int x = 0; x < n4w; x += step) {
        const uint32_t start_x = base_x + 4 * x, start_y = base_y + 4 * y;
        if (start_x < max_x && start_y < max_y) {
          uint32_t t = NO_TOK;
          uint32_t n_coef = 0, tsz = 0;
          if (!b.coded_skip) {
            t = tok++;
            const rv9_tok tk = toks[t];
            if (tk.eob == 0) t = NO_TOK;
            n_coef = tk.n_coef;
            tsz = tk.tx_size & 3;
          }
          const uint64_t n0 = 4u << tx_sz;
          const uint64_t coef_bytes = t != NO_TOK ? sizeof(rv9_tok) + 4ull * n_coef : 0;
          if (is_inter) {
            if (t != NO_TOK) {
              if (EMIT) res[res_at[tsz] + w.res[tsz]] = ResItem{t, bi};
              ++w.res[tsz];
              w.kb_res += coef_bytes + 2 * n0 * n0 * bps;
            }
          } else {
            const int mode = plane ? b.uv_mode : (b.mi_size >= 3 ? b.y_mode : b.sub_modes[block_idx]);
            const uint8_t fl =
                (uint8_t)((avail_l || x > 0 ? 1 : 0) | (avail_u || y > 0 ? 2 : 0) | (x + step < n4w ? 4 : 0));
            if (EMIT)
              intra[intra_at + w.intra] = IntraItem{bi, t, (uint16_t)start_x, (uint16_t)start_y, (uint8_t)plane,
                                                    (uint8_t)tx_sz, (uint8_t)mode, fl};
            ++w.intra;
            w.kb_intra += (n0 * n0 + 3 * n0 + 1) * bps + coef_bytes;
          }
        }
        ++block_idx;
      }
  }
}

// A frame's records gathered from its tile columns (tok_start and
// coef_start rebased), then its work lists in Engine::build_work's order:
// inter regions of at most 16x16 first, then the larger ones; residuals by
// transform size; intra items by superblock anti-diagonal (column + 2 row),
// stable; intra jobs at each change of (block, plane, row). Within a bucket,
// bitstream order.
__global__ void __launch_bounds__(kBuildThreads) k_build_frames(
    const tp::Tables* __restrict__ T, const BuildFrame* __restrict__ frames, const tp::Chain* __restrict__ chains,
    const tp::ChainOut* __restrict__ outs, const rv9_block* __restrict__ cblocks, const rv9_tok* __restrict__ ctoks,
    const uint32_t* __restrict__ ccoefs, uint8_t* stage, uint32_t* scratch_base, BuildOut* results) {
  __shared__ BuildSmem S;
  const BuildFrame F = frames[blockIdx.x];
  BuildOut* R = &results[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t n_diag = F.sb64_cols + 2 * F.sb64_rows + 1;
  if (tid == 0) {
    S.err = 0;
    S.err_tile = 0;
    uint32_t nb = 0, nt = 0, nc = 0;
    uint64_t bools = 0;
    for (uint32_t c = 0; c < F.n_chains; ++c) {
      const tp::ChainOut o = outs[F.first_chain + c];
      S.chain_b[c] = nb;
      S.chain_t[c] = nt;
      S.chain_c[c] = nc;
      nb += o.n_blocks;
      nt += o.n_toks;
      nc += o.n_coefs;
      bools += o.bools;
      if (o.err && (!S.err || o.err_tile < S.err_tile)) {
        S.err = o.err;
        S.err_tile = o.err_tile;
      }
    }
    S.chain_b[F.n_chains] = nb;
    S.chain_t[F.n_chains] = nt;
    S.chain_c[F.n_chains] = nc;
    if (!S.err && (F.n_chains > kMaxChains || n_diag > kMaxDiag || nb > F.cap_blocks || nt > F.cap_items)) {
      S.err = tp::TP_OVERFLOW;
      S.err_tile = 0;
    }
    for (int k = 0; k < 8; ++k) S.carry[k] = 0;
    for (int k = 0; k < 4; ++k) S.kb[k] = 0;
    R->err = S.err;
    R->err_tile = S.err_tile;
    R->n_blocks = nb;
    R->n_toks = nt;
    R->n_coefs = nc;
    R->bools = bools;
  }
  __syncthreads();
  if (S.err) return;
  uint8_t* base = stage + F.base;
  rv9_block* blocks = (rv9_block*)(base + F.o_blocks);
  rv9_tok* toks = (rv9_tok*)(base + F.o_toks);
  uint32_t* coefs = (uint32_t*)(base + F.o_coefs);
  InterUnit* units = (InterUnit*)(base + F.o_units);
  ResItem* res = (ResItem*)(base + F.o_res);
  IntraItem* intra = (IntraItem*)(base + F.o_intra);
  uint32_t* jobs = (uint32_t*)(base + F.o_jobs);
  uint32_t* scr = scratch_base + F.scratch_at;
  const uint32_t nb = S.chain_b[F.n_chains];

  // Gather.
  for (uint32_t c = 0; c < F.n_chains; ++c) {
    const tp::Chain& ch = chains[F.first_chain + c];
    const uint32_t b0 = S.chain_b[c], bn = S.chain_b[c + 1] - b0;
    const uint32_t t0 = S.chain_t[c], tn = S.chain_t[c + 1] - t0;
    const uint32_t c0 = S.chain_c[c], cn = S.chain_c[c + 1] - c0;
    for (uint32_t i = tid; i < bn; i += kBuildThreads) {
      rv9_block b = cblocks[ch.blocks_at + i];
      b.tok_start += t0;
      blocks[b0 + i] = b;
    }
    for (uint32_t i = tid; i < tn; i += kBuildThreads) {
      rv9_tok t = ctoks[ch.toks_at + i];
      t.coef_start += c0;
      toks[t0 + i] = t;
    }
    for (uint32_t i = tid; i < cn; i += kBuildThreads) coefs[c0 + i] = ccoefs[ch.coefs_at + i];
  }
  __syncthreads();

  // Pass A: each block's counts, scanned in frame order.
  uint64_t kb_inter = 0, kb_res = 0, kb_intra = 0, out_bytes = 0;
  for (uint32_t chunk = 0; chunk < nb; chunk += kBuildThreads) {
    const uint32_t bi = chunk + tid;
    uint32_t v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (bi < nb) {
      const rv9_block b = blocks[bi];
      WalkOut w = {};
      walk_block<false>(T, F, b, bi, toks, w, nullptr, 0, 0, nullptr, nullptr, nullptr, 0);
      v[0] = w.small;
      v[1] = w.large;
      for (int z = 0; z < 4; ++z) v[2 + z] = w.res[z];
      v[6] = w.intra;
      kb_inter += w.kb_inter;
      kb_res += w.kb_res;
      kb_intra += w.kb_intra;
      out_bytes += w.out_bytes;
      scr[bi * 8 + 6] = w.intra;
      scr[bi * 8 + 7] = ((uint32_t)b.mi_col >> 3) + 2 * ((uint32_t)b.mi_row >> 3);
    }
    cta_scan8(v, S);
    if (bi < nb)
      for (int k = 0; k < 6; ++k) scr[bi * 8 + k] = v[k];
  }
  atomicAdd(&S.kb[0], (unsigned long long)kb_inter);
  atomicAdd(&S.kb[1], (unsigned long long)kb_res);
  atomicAdd(&S.kb[2], (unsigned long long)kb_intra);
  atomicAdd(&S.kb[3], (unsigned long long)out_bytes);
  if (tid == 0) {
    for (int k = 0; k < 8; ++k) {
      S.tot[k] = S.carry[k];
      S.carry[k] = 0;
    }
    S.res_base[0] = 0;
    for (int z = 1; z < 4; ++z) S.res_base[z] = S.res_base[z - 1] + S.tot[1 + z];
  }
  for (uint32_t g = tid; g < n_diag; g += kBuildThreads) S.diag[g] = 0;
  __syncthreads();

  // Intra items by anti-diagonal: a block's place within its diagonal is the
  // sum of the intra items of the blocks before it on that diagonal (warp 0,
  // 32 blocks at a time); then the diagonals' starts.
  if (warp == 0) {
    for (uint32_t chunk = 0; chunk < nb; chunk += 32) {
      const uint32_t bi = chunk + lane;
      const bool valid = bi < nb;
      const uint32_t g = valid ? scr[bi * 8 + 7] : 0xffffffffu;
      const uint32_t cnt = valid ? scr[bi * 8 + 6] : 0;
      const uint32_t peers = __match_any_sync(0xffffffffu, g);
      const uint32_t below = peers & ((1u << lane) - 1);
      uint32_t pre = 0;
      for (int k = 0; k < 32; ++k) {
        const uint32_t x = __shfl_sync(0xffffffffu, cnt, k);
        if ((below >> k) & 1) pre += x;
      }
      const uint32_t rel = valid ? S.diag[g] + pre : 0;
      __syncwarp();
      if (valid) {
        scr[bi * 8 + 6] = rel;
        if (lane == 31 - __clz(peers)) S.diag[g] = rel + cnt;
      }
      __syncwarp();
    }
  }
  __syncthreads();
  if (tid == 0) {
    uint32_t acc = 0;
    for (uint32_t g = 0; g < n_diag; ++g) {
      const uint32_t t = S.diag[g];
      S.diag[g] = acc;
      acc += t;
    }
  }
  __syncthreads();

  // Pass B: the lists.
  for (uint32_t bi = tid; bi < nb; bi += kBuildThreads) {
    const rv9_block b = blocks[bi];
    const uint32_t* o = scr + bi * 8;
    uint32_t res_at[4];
    for (int z = 0; z < 4; ++z) res_at[z] = S.res_base[z] + o[2 + z];
    WalkOut w = {};
    walk_block<true>(T, F, b, bi, toks, w, units, o[0], S.tot[0] + o[1], res, res_at, intra, S.diag[o[7]] + o[6]);
  }
  __syncthreads();

  // Intra jobs.
  const uint32_t n_intra = S.tot[6];
  for (uint32_t chunk = 0; chunk < n_intra; chunk += kBuildThreads) {
    const uint32_t i = chunk + tid;
    uint32_t v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    bool start = false;
    if (i < n_intra) {
      const IntraItem a = intra[i];
      if (i == 0) {
        start = true;
      } else {
        const IntraItem p = intra[i - 1];
        start = a.block != p.block || a.plane != p.plane || a.y != p.y;
      }
    }
    v[0] = start ? 1 : 0;
    cta_scan8(v, S);
    if (start) jobs[v[0]] = i;
  }
  if (tid == 0) {
    const uint32_t n_jobs = S.carry[0];
    jobs[n_jobs] = n_intra;
    const uint32_t nt = S.chain_t[F.n_chains], nc = S.chain_c[F.n_chains];
    const uint64_t bps = F.bit_depth > 8 ? 2 : 1;
    R->n_units_small = S.tot[0];
    R->n_units = S.tot[0] + S.tot[1];
    uint32_t n_res = 0;
    for (int z = 0; z < 4; ++z) {
      R->n_res_by_size[z] = S.tot[2 + z];
      n_res += S.tot[2 + z];
    }
    R->n_res = n_res;
    R->n_intra = n_intra;
    R->n_intra_jobs = n_jobs;
    for (int k = 0; k < K_COUNT; ++k) R->kbytes[k] = 0;
    R->kbytes[K_INTER] = S.kb[0];
    R->kbytes[K_INTER_RES] = S.kb[1];
    R->kbytes[K_INTRA] = S.kb[2];
    const uint64_t mi_w = (uint64_t)F.mi_cols * 8, mi_h = (uint64_t)F.mi_rows * 8;
    const uint64_t area = (mi_w * mi_h + 2 * (mi_w >> F.ss_x) * (mi_h >> F.ss_y)) * bps;
    if (F.lf_on) {
      R->kbytes[K_LF] = 2 * area;
      R->kbytes[K_PREP] = (uint64_t)nb * sizeof(rv9_block) + (uint64_t)F.mi_cols * F.mi_rows * 4;
    }
    R->kbytes[K_PREP] += (uint64_t)n_intra * sizeof(IntraItem);
    R->total_bytes = (uint64_t)nb * sizeof(rv9_block) + (uint64_t)nt * sizeof(rv9_tok) + (uint64_t)nc * 4 +
                     (S.kb[0] - S.kb[3]) + area;
  }
}

cudaError_t launch_build_frames(const BuildFrame* frames, uint32_t n, const tp::Chain* chains,
                                const tp::ChainOut* outs, const rv9_block* blocks, const rv9_tok* toks,
                                const uint32_t* coefs, uint8_t* stage, uint32_t* scratch, BuildOut* results,
                                cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return e;
  const tp::Tables* T = nullptr;
  if ((e = parse_tables(device, &T)) != cudaSuccess) return e;
  k_build_frames<<<n, kBuildThreads, 0, s>>>(T, frames, chains, outs, blocks, toks, coefs, stage, scratch, results);
  return cudaGetLastError();
}

}  // namespace rv9g

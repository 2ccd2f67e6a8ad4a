// Host side of the reconstruction engine: the device frame pool and reference
// slots (the reference's RefFrame / refs[8], src/decoder/mod.rs:65-75,
// 399-415), the work lists derived from a parsed frame's records (the loops of
// FrameDec::replay, src/decoder/block.rs:1405-1498), the quantiser and
// loop-filter tables (src/decoder/recon.rs:219-264,
// src/decoder/loopfilter.rs:15-47,135-170), and the launch of one frame.
#include "engine.h"

#include <string.h>

#include <algorithm>

#include "../common/vp9_consts.h"
#include "../common/vp9_tables.h"

namespace rv9g {
using namespace vp9;

const char* const kKernelNames[K_COUNT] = {"k_prep", "k_inter", "k_inter_res", "k_intra", "k_lf"};

#define CK(call)                                                 \
  do {                                                           \
    cudaError_t e_ = (call);                                     \
    if (e_ != cudaSuccess) {                                     \
      *err = std::string(#call) + ": " + cudaGetErrorString(e_); \
      return rv9::ST_DEVICE;                                     \
    }                                                            \
  } while (0)

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }


// Waits, when it goes out of scope, for the streams of engines[0..n): a run
// over several engines' streams that returns early (an error part-way
// through) leaves none of its launches running behind it.
struct StreamsDrain {
  Engine* const* engines;
  size_t n;
  ~StreamsDrain() {
    for (size_t j = 0; j < n; ++j) cudaStreamSynchronize(engines[j]->stream());
  }
};

Engine::~Engine() {
  if (stream_) cudaStreamSynchronize(stream_);
  for (DevFrame* f : pool_) {
    cudaFree(f->base);
    delete f;
  }
  for (int i = 0; i < 2; ++i) {
    cudaFree(d_stage_[i]);
    cudaFreeHost(h_stage_[i]);
    if (stage_ev_[i]) cudaEventDestroy(stage_ev_[i]);
  }
  cudaFree(d_lf_mi_);
  cudaFree(d_sb_done_);
  cudaFree(d_counters_);
  cudaFreeHost(h_error_);
  for (cudaEvent_t e : kev_) cudaEventDestroy(e);
  if (aux_.side) cudaStreamSynchronize(aux_.side);
  if (aux_.fork) cudaEventDestroy(aux_.fork);
  if (aux_.join) cudaEventDestroy(aux_.join);
  if (aux_.side) cudaStreamDestroy(aux_.side);
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  if (stream_) cudaStreamDestroy(stream_);
  cudaFree(batch_d_);
  cudaFreeHost(batch_h_);
  cudaFree(d_digest_);
}

bool Engine::init(int device, std::string* err, bool side_stream) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    *err = std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "none found");
    return false;
  }
  if (device < 0) cudaGetDevice(&device);
  device_ = device;
  if ((e = cudaSetDevice(device)) != cudaSuccess) {
    *err = cudaGetErrorString(e);
    return false;
  }
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  if (prop.major < 10) {
    *err = "the kernels are built for sm_100a (B200); device is sm_" + std::to_string(prop.major) +
           std::to_string(prop.minor);
    return false;
  }
  n_sm_ = prop.multiProcessorCount;
  if ((e = kernels_init_device(device)) != cudaSuccess) {
    *err = std::string("setting up the kernels on the device: ") + cudaGetErrorString(e);
    return false;
  }
  if ((e = cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreate(&ev0_)) != cudaSuccess || (e = cudaEventCreate(&ev1_)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&stage_ev_[0], cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&stage_ev_[1], cudaEventDisableTiming)) != cudaSuccess ||
      (side_stream && (e = cudaStreamCreateWithFlags(&aux_.side, cudaStreamNonBlocking)) != cudaSuccess) ||
      (e = cudaEventCreateWithFlags(&aux_.fork, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&aux_.join, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaMalloc(&d_counters_, 64)) != cudaSuccess || (e = cudaMallocHost(&h_error_, 64)) != cudaSuccess) {
    *err = cudaGetErrorString(e);
    return false;
  }
  *h_error_ = 0;
  int16_t f[4][16][8];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 16; ++b)
      for (int c = 0; c < 8; ++c) f[a][b][c] = (int16_t)vp9t_subpel_filters[a][b][c];
  if ((e = upload_filters(&f[0][0][0])) != cudaSuccess || (e = upload_md5_table()) != cudaSuccess) {
    *err = std::string("loading the kernels: ") + cudaGetErrorString(e);
    return false;
  }
  cudaMemset(d_counters_, 0, 64);
  return true;
}

size_t Engine::packed_bytes(const DevFrame* f) {
  size_t cw = (f->width + f->ss_x) >> f->ss_x, ch = (f->height + f->ss_y) >> f->ss_y;
  return ((size_t)f->width * f->height + 2 * cw * ch) * f->bps();
}

DevFrame* Engine::alloc_frame(const rv9_frame_desc& d, cudaStream_t stream) {
  uint32_t aw = d.sb64_cols * 64, ah = d.sb64_rows * 64;
  // A frame no slot holds is free: every use of it is queued on the stream
  // before the work that overwrites it.
  for (DevFrame* f : pool_) {
    if (f->refs == 0 && f->aw == aw && f->ah == ah && f->ss_x == d.ss_x && f->ss_y == d.ss_y &&
        f->bit_depth == d.bit_depth)
      return f;
  }
  if (fixed_) return nullptr;  // sequence_run_fixed allocates nothing
  DevFrame* f = new DevFrame;
  f->aw = aw;
  f->ah = ah;
  f->ss_x = d.ss_x;
  f->ss_y = d.ss_y;
  f->bit_depth = d.bit_depth;
  size_t bps = f->bps();
  size_t off = 0;
  size_t plane_off[3], cell_off[3];
  for (int p = 0; p < 3; ++p) {
    int w = p ? (int)(aw >> d.ss_x) : (int)aw, h = p ? (int)(ah >> d.ss_y) : (int)ah;
    f->stride[p] = w;
    f->pheight[p] = h;
    plane_off[p] = off;
    off += align256((size_t)w * h * bps);
  }
  for (int p = 0; p < 3; ++p) {
    f->cell_stride[p] = f->stride[p] / 4;
    cell_off[p] = off;
    off += align256((size_t)f->cell_stride[p] * (f->pheight[p] / 4));
  }
  f->bytes = off;
  if (cudaMalloc(&f->base, off) != cudaSuccess) {
    delete f;
    return nullptr;
  }
  for (int p = 0; p < 3; ++p) {
    f->planes[p] = (uint8_t*)f->base + plane_off[p];
    f->cells[p] = (uint8_t*)f->base + cell_off[p];
  }
  // Zeroed on the stream whose launches use the frame first (the cell map
  // must read zero before that frame's preparation kernel marks it).
  if (cudaMemsetAsync(f->base, 0, off, stream) != cudaSuccess) {
    cudaFree(f->base);
    delete f;
    return nullptr;
  }
  pool_.push_back(f);
  return f;
}

void Engine::reset_slots() {
  for (int i = 0; i < 8; ++i) {
    if (slots_[i]) --slots_[i]->refs;
    slots_[i] = nullptr;
  }
}

static int uv_tx_size(const rv9_frame_desc& d, const rv9_block& b) {
  if (b.mi_size < BLOCK_8X8) return TX_4X4;
  int sx = d.legacy_uv ? 1 : d.ss_x, sy = d.legacy_uv ? 1 : d.ss_y;
  int uv = SS_SIZE_LOOKUP[b.mi_size][sx][sy];
  return std::min<int>(b.tx_size, MAX_TXSIZE_LOOKUP[uv]);
}

// The work lists (the prediction regions and residuals of inter blocks, and
// the intra transform blocks in bitstream order, replay's loop structure) and
// the frame's staged bytes, written where `reserve` says. Algorithmic bytes
// per kernel: inter 1 sample per predicted sample and reference plus the
// output; a residual its coefficient words plus reading and writing its
// samples; intra its samples out plus (3 n + 1) edge samples plus its
// coefficients; the loop filter reading and writing the mode-info area once;
// all at 1 byte per sample at 8 bits, 2 above.
//
// The lists come out already in launch order, each bucketed as it is built
// (no sort): inter regions of at most 16x16 first (one warp each), then the
// larger ones (one CTA each); residuals by transform size (the residual
// kernel packs 8, 4, 2 or 1 of them per warp); intra items by superblock
// anti-diagonal. Within a bucket, bitstream order.
bool Engine::build_work(const rv9::ParsedFrame& pf, FrameWork* fw, const StageReserve& reserve) {
  const rv9_frame_desc& d = pf.desc;
  fw->desc = d;
  fw->show_existing = pf.show_existing;
  fw->show_slot = pf.show_slot;
  fw->show_frame = pf.show_frame;
  fw->refresh_mask = pf.refresh_mask;
  for (int i = 0; i < 3; ++i) fw->ref_slot[i] = pf.ref_slot[i];
  memset(fw->kbytes, 0, sizeof fw->kbytes);
  fw->total_bytes = 0;
  if (pf.show_existing) return true;
  units_small_.clear();
  units_large_.clear();
  for (auto& r : res_by_size_) r.clear();
  intra_.clear();
  intra_diag_.clear();
  const uint64_t bps = d.bit_depth > 8 ? 2 : 1;
  uint64_t out_bytes = 0;  // inter outputs, to take out of the reference bytes
  for (uint32_t bi = 0; bi < pf.blocks.size(); ++bi) {
    const rv9_block& b = pf.blocks[bi];
    const bool is_inter = b.flags & RV9_BLK_INTER;
    const bool avail_l = b.flags & RV9_BLK_AVAIL_L, avail_u = b.flags & RV9_BLK_AVAIL_U;
    const int bsize = std::max<int>(b.mi_size, BLOCK_8X8);
    const int nrefs = b.ref_frame[1] > INTRA_FRAME ? 2 : 1;
    // Superblock anti-diagonal (column + 2 row): every superblock an intra
    // block reads from (left, above, above-left; its above-right samples
    // stop at its own block's right edge, src/decoder/recon.rs:57-66) lies
    // on an earlier one. Column + row would also be safe, and measured 5 %
    // slower: it hands out the jobs of superblocks farther down before
    // those of the rows above them are done.
    const uint16_t diag = (uint16_t)((b.mi_col >> 3) + 2 * (b.mi_row >> 3));
    uint32_t tok = b.tok_start;
    for (int plane = 0; plane < 3; ++plane) {
      int tx_sz = plane ? uv_tx_size(d, b) : b.tx_size;
      int step = 1 << tx_sz;
      int sx = plane ? d.ss_x : 0, sy = plane ? d.ss_y : 0;
      int plane_sz = SS_SIZE_LOOKUP[bsize][sx][sy];
      int n4w = vp9t_num_4x4_wide[plane_sz], n4h = vp9t_num_4x4_high[plane_sz];
      int base_x = (b.mi_col * 8) >> sx, base_y = (b.mi_row * 8) >> sy;
      if (is_inter) {
        if (b.mi_size < BLOCK_8X8) {
          for (int y = 0; y < n4h; ++y)
            for (int x = 0; x < n4w; ++x)
              units_small_.push_back(InterUnit{bi, (uint16_t)(base_x + 4 * x), (uint16_t)(base_y + 4 * y),
                                               (uint8_t)plane, 1, 1, (uint8_t)(y * n4w + x)});
        } else {
          (n4w <= 4 && n4h <= 4 ? units_small_ : units_large_)
              .push_back(InterUnit{bi, (uint16_t)base_x, (uint16_t)base_y, (uint8_t)plane, (uint8_t)n4w,
                                   (uint8_t)n4h, 0});
        }
        const uint64_t out = (uint64_t)n4w * n4h * 16 * bps;
        fw->kbytes[K_INTER] += out * (nrefs + 1);
        out_bytes += out;
      }
      int max_x = (int)((d.mi_cols * 8) >> sx), max_y = (int)((d.mi_rows * 8) >> sy);
      int block_idx = 0;
      for (int y = 0; y < n4h; y += step)
        for (int x = 0; x < n4w; x += step) {
          int start_x = base_x + 4 * x, start_y = base_y + 4 * y;
          if (start_x < max_x && start_y < max_y) {
            uint32_t t = NO_TOK;
            if (!b.coded_skip) {
              t = tok++;
              if (pf.toks[t].eob == 0) t = NO_TOK;
            }
            const uint64_t n0 = 4u << tx_sz;
            const uint64_t coef_bytes = t != NO_TOK ? sizeof(rv9_tok) + 4ull * pf.toks[t].n_coef : 0;
            if (is_inter) {
              if (t != NO_TOK) {
                res_by_size_[pf.toks[t].tx_size & 3].push_back(ResItem{t, bi});
                fw->kbytes[K_INTER_RES] += coef_bytes + 2 * n0 * n0 * bps;
              }
            } else {
              int mode = plane ? b.uv_mode : (b.mi_size >= BLOCK_8X8 ? b.y_mode : b.sub_modes[block_idx]);
              uint8_t fl = (uint8_t)((avail_l || x > 0 ? 1 : 0) | (avail_u || y > 0 ? 2 : 0) | (x + step < n4w ? 4 : 0));
              intra_.push_back(IntraItem{bi, t, (uint16_t)start_x, (uint16_t)start_y, (uint8_t)plane, (uint8_t)tx_sz,
                                         (uint8_t)mode, fl});
              intra_diag_.push_back(diag);
              fw->kbytes[K_INTRA] += (n0 * n0 + 3 * n0 + 1) * bps + coef_bytes;
            }
          }
          ++block_idx;
        }
    }
  }
  const uint64_t mi_w = (uint64_t)d.mi_cols * 8, mi_h = (uint64_t)d.mi_rows * 8;
  const uint64_t area = (mi_w * mi_h + 2 * (mi_w >> d.ss_x) * (mi_h >> d.ss_y)) * bps;
  if (d.lf_level) {
    fw->kbytes[K_LF] = 2 * area;
    fw->kbytes[K_PREP] = pf.blocks.size() * sizeof(rv9_block) + (uint64_t)d.mi_cols * d.mi_rows * 4;
  }
  fw->kbytes[K_PREP] += intra_.size() * sizeof(IntraItem);
  // The frame's algorithmic bytes: records read once, reference samples
  // predicted from, and the reconstructed samples written once.
  const uint64_t ref_bytes = fw->kbytes[K_INTER] - out_bytes;
  fw->total_bytes = pf.blocks.size() * sizeof(rv9_block) + pf.toks.size() * sizeof(rv9_tok) +
                    pf.coefs.size() * 4 + ref_bytes + area;
  // Intra items by anti-diagonal: a counting sort, stable.
  if (!intra_.empty()) {
    size_t n_diag = (size_t)(d.sb64_cols + 2 * d.sb64_rows) + 1;
    diag_start_.assign(n_diag + 1, 0);
    for (uint16_t g : intra_diag_) ++diag_start_[g + 1];
    for (size_t g = 0; g < n_diag; ++g) diag_start_[g + 1] += diag_start_[g];
    sorted_intra_.resize(intra_.size());
    for (size_t i = 0; i < intra_.size(); ++i) sorted_intra_[diag_start_[intra_diag_[i]]++] = intra_[i];
    intra_.swap(sorted_intra_);
  }
  // Jobs: one row of transform blocks of one block and plane (contiguous in
  // this order), done by one warp in turn. Each depends on its left
  // neighbour anyway, so a row loses no parallelism by staying on one warp.
  intra_jobs_.clear();
  for (size_t i = 0; i < intra_.size(); ++i)
    if (i == 0 || intra_[i].block != intra_[i - 1].block || intra_[i].plane != intra_[i - 1].plane ||
        intra_[i].y != intra_[i - 1].y)
      intra_jobs_.push_back((uint32_t)i);
  fw->n_intra_jobs = (uint32_t)intra_jobs_.size();
  intra_jobs_.push_back((uint32_t)intra_.size());
  // The staged layout: each array at a 256-byte boundary.
  size_t n_res = 0;
  for (int z = 0; z < 4; ++z) {
    fw->n_res_by_size[z] = (uint32_t)res_by_size_[z].size();
    n_res += res_by_size_[z].size();
  }
  const size_t n_units = units_small_.size() + units_large_.size();
  size_t rel = 0;
  auto place = [&](size_t bytes) {
    size_t o = rel;
    rel = align256(rel + bytes);
    return o;
  };
  const size_t r_blocks = place(pf.blocks.size() * sizeof(rv9_block));
  const size_t r_toks = place(pf.toks.size() * sizeof(rv9_tok));
  const size_t r_coefs = place(pf.coefs.size() * 4);
  const size_t r_units = place(n_units * sizeof(InterUnit));
  const size_t r_res = place(n_res * sizeof(ResItem));
  const size_t r_intra = place(intra_.size() * sizeof(IntraItem));
  const size_t r_jobs = place(intra_jobs_.size() * 4);
  size_t base = 0;
  uint8_t* dst = reserve(rel, &base);
  if (!dst) return false;
  auto copy = [&](size_t r, const void* src, size_t bytes) {
    if (bytes) memcpy(dst + r, src, bytes);
  };
  // Zero padding after each array, so that the staged bytes depend on the
  // frame alone.
  const size_t ends[7][2] = {{r_blocks, pf.blocks.size() * sizeof(rv9_block)},
                             {r_toks, pf.toks.size() * sizeof(rv9_tok)},
                             {r_coefs, pf.coefs.size() * 4},
                             {r_units, n_units * sizeof(InterUnit)},
                             {r_res, n_res * sizeof(ResItem)},
                             {r_intra, intra_.size() * sizeof(IntraItem)},
                             {r_jobs, intra_jobs_.size() * 4}};
  for (const auto& e : ends) {
    const size_t end = e[0] + e[1];
    memset(dst + end, 0, align256(end) - end);
  }
  copy(r_blocks, pf.blocks.data(), pf.blocks.size() * sizeof(rv9_block));
  copy(r_toks, pf.toks.data(), pf.toks.size() * sizeof(rv9_tok));
  copy(r_coefs, pf.coefs.data(), pf.coefs.size() * 4);
  copy(r_units, units_small_.data(), units_small_.size() * sizeof(InterUnit));
  copy(r_units + units_small_.size() * sizeof(InterUnit), units_large_.data(),
       units_large_.size() * sizeof(InterUnit));
  size_t r = r_res;
  for (int z = 0; z < 4; ++z) {
    copy(r, res_by_size_[z].data(), res_by_size_[z].size() * sizeof(ResItem));
    r += res_by_size_[z].size() * sizeof(ResItem);
  }
  copy(r_intra, intra_.data(), intra_.size() * sizeof(IntraItem));
  copy(r_jobs, intra_jobs_.data(), intra_jobs_.size() * 4);
  fw->o_blocks = base + r_blocks;
  fw->o_toks = base + r_toks;
  fw->o_coefs = base + r_coefs;
  fw->o_units = base + r_units;
  fw->o_res = base + r_res;
  fw->o_intra = base + r_intra;
  fw->o_intra_jobs = base + r_jobs;
  fw->bytes = rel;
  fw->n_blocks = (uint32_t)pf.blocks.size();
  fw->n_toks = (uint32_t)pf.toks.size();
  fw->n_coefs = (uint32_t)pf.coefs.size();
  fw->n_units = (uint32_t)n_units;
  fw->n_units_small = (uint32_t)units_small_.size();
  fw->n_res = (uint32_t)n_res;
  fw->n_intra = (uint32_t)intra_.size();
  return true;
}

void Engine::hook(void* ctx, int kernel, int phase) {
  Engine* e = (Engine*)ctx;
  if (!((e->event_mask >> kernel) & 1)) return;
  if (e->kev_used_ == e->kev_.size()) {
    cudaEvent_t ev;
    cudaEventCreate(&ev);
    e->kev_.push_back(ev);
    e->kev_kernel_.push_back(0);
  }
  size_t i = e->kev_used_++;
  e->kev_kernel_[i] = kernel;
  cudaEventRecord(e->kev_[i], e->stream_);
  if (phase == 0 && e->cur_fw_) e->kstats[kernel].bytes += e->cur_fw_->kbytes[kernel];
}

void Engine::collect_kernel_events() {
  cudaStreamSynchronize(stream_);
  for (size_t i = 0; i + 1 < kev_used_; i += 2) {
    float ms = 0;
    cudaEventElapsedTime(&ms, kev_[i], kev_[i + 1]);
    KernelStat& s = kstats[kev_kernel_[i]];
    s.ms += ms;
    s.launches += 1;
  }
  kev_used_ = 0;
}

rv9::Status Engine::prepare_frame(const FrameWork& fw, const uint8_t* d_base, cudaStream_t stream, KFrame* kf,
                                  DevFrame** out, std::string* err) {
  *out = nullptr;
  if (fw.show_existing) {
    if (!slots_[fw.show_slot]) {
      *err = "show_existing_frame of an empty slot";
      return rv9::ST_BITSTREAM;
    }
    return rv9::ST_OK;
  }
  const rv9_frame_desc& d = fw.desc;
  DevFrame* cur = alloc_frame(d, stream);
  if (!cur) {
    *err = "out of device memory for a frame";
    return rv9::ST_DEVICE;
  }
  cur->width = d.width;
  cur->height = d.height;
  cur->color_space = d.color_space;
  cur->color_range = d.color_range;
  cur->render_w = d.render_width;
  cur->render_h = d.render_height;
  size_t mi_len = (size_t)d.mi_cols * d.mi_rows;
  if (fixed_) {
    // Already checked against the array's size; zero the two tickets and
    // the done flags (flags then compare against epoch 1). The error word
    // (the third counter) is cleared once per run, before its first frame,
    // so that a wait that gave up in any frame stays reported.
    size_t flags = align256((size_t)d.sb64_cols * d.sb64_rows * 4);
    CK(cudaMemsetAsync(fixed_, 0, 2 * sizeof(int32_t), stream));
    CK(cudaMemsetAsync(fixed_ + 256, 0, flags, stream));
  } else if (mi_len > lf_mi_cap_) {
    CK(cudaStreamSynchronize(stream));
    cudaFree(d_lf_mi_);
    CK(cudaMalloc(&d_lf_mi_, mi_len * 4));
    lf_mi_cap_ = mi_len;
  }
  size_t n_sb = (size_t)d.sb64_cols * d.sb64_rows;
  if (!fixed_ && n_sb > sb_cap_) {
    CK(cudaStreamSynchronize(stream));
    cudaFree(d_sb_done_);
    CK(cudaMalloc(&d_sb_done_, n_sb * 4));
    CK(cudaMemsetAsync(d_sb_done_, 0, n_sb * 4, stream));
    sb_cap_ = n_sb;
  }
  // The loop filter's progress words carry the epoch's low 16 bits: clear
  // them when those wrap, so that no stale word can match.
  if (!fixed_ && ((++epoch_) & 0xffff) == 0) {
    CK(cudaMemsetAsync(d_sb_done_, 0, sb_cap_ * 4, stream));
    ++epoch_;
  }
  KFrame& k = *kf;
  memset(&k, 0, sizeof k);
  for (int p = 0; p < 3; ++p) {
    k.cur[p].data = cur->planes[p];
    k.cur[p].stride = cur->stride[p];
    k.cur[p].width = cur->stride[p];
    k.cur[p].height = cur->pheight[p];
    k.cells[p] = cur->cells[p];
    k.cell_stride[p] = cur->cell_stride[p];
  }
  if (!d.frame_is_intra) {
    for (int i = 0; i < 3; ++i) {
      DevFrame* r = slots_[fw.ref_slot[i]];
      if (!r) {
        *err = "reference to an empty slot";
        return rv9::ST_BITSTREAM;
      }
      for (int p = 0; p < 3; ++p) {
        k.ref[i][p].data = r->planes[p];
        k.ref[i][p].stride = r->stride[p];
        k.ref[i][p].width = p ? (int)((r->width + d.ss_x) >> d.ss_x) : (int)r->width;
        k.ref[i][p].height = p ? (int)((r->height + d.ss_y) >> d.ss_y) : (int)r->height;
      }
      // xScale / yScale (spec 8.5.2.3; reference src/decoder/mod.rs:503-511).
      k.ref_xs[i] = ((int64_t)r->width << 14) / d.width;
      k.ref_ys[i] = ((int64_t)r->height << 14) / d.height;
    }
  }
  k.mi_cols = d.mi_cols;
  k.mi_rows = d.mi_rows;
  k.sb64_cols = d.sb64_cols;
  k.sb64_rows = d.sb64_rows;
  k.width = d.width;
  k.height = d.height;
  k.ss_x = d.ss_x;
  k.ss_y = d.ss_y;
  k.bit_depth = d.bit_depth;
  k.lossless = d.lossless;
  k.legacy_uv = d.legacy_uv;
  // Quantiser per segment (reference qindex + reconstruct's lookups).
  int bd_idx = (d.bit_depth - 8) >> 1;
  auto cq = [](int v) { return std::min(std::max(v, 0), 255); };
  for (int seg = 0; seg < 8; ++seg) {
    int q = d.base_q_idx;
    if (d.seg.enabled && d.seg.feature_enabled[seg][SEG_LVL_ALT_Q]) {
      int data = d.seg.feature_data[seg][SEG_LVL_ALT_Q];
      if (!d.seg.abs_or_delta_update) data += d.base_q_idx;
      q = cq(data);
    }
    k.dc_q[seg][0] = vp9t_dc_qlookup[bd_idx][cq(q + d.delta_q_y_dc)];
    k.ac_q[seg][0] = vp9t_ac_qlookup[bd_idx][cq(q)];
    k.dc_q[seg][1] = vp9t_dc_qlookup[bd_idx][cq(q + d.delta_q_uv_dc)];
    k.ac_q[seg][1] = vp9t_ac_qlookup[bd_idx][cq(q + d.delta_q_uv_ac)];
  }
  k.blocks = (const rv9_block*)(d_base + fw.o_blocks);
  k.toks = (const rv9_tok*)(d_base + fw.o_toks);
  k.coefs = (const uint32_t*)(d_base + fw.o_coefs);
  k.units = (const InterUnit*)(d_base + fw.o_units);
  k.n_units = (int32_t)fw.n_units;
  k.n_units_small = (int32_t)fw.n_units_small;
  k.res = (const ResItem*)(d_base + fw.o_res);
  k.n_res = (int32_t)fw.n_res;
  for (int z = 0; z < 4; ++z) k.n_res_by_size[z] = (int32_t)fw.n_res_by_size[z];
  k.intra = (const IntraItem*)(d_base + fw.o_intra);
  k.n_intra = (int32_t)fw.n_intra;
  k.intra_jobs = (const uint32_t*)(d_base + fw.o_intra_jobs);
  k.n_intra_jobs = (int32_t)fw.n_intra_jobs;
  // Loop filter levels and limits (8.8.1).
  k.lf_on = d.lf_level != 0;
  if (k.lf_on) {
    int n_shift = d.lf_level >> 5;
    for (int seg = 0; seg < 8; ++seg) {
      int lvl_seg = d.lf_level;
      if (d.seg.enabled && d.seg.feature_enabled[seg][SEG_LVL_ALT_L]) {
        int data = d.seg.feature_data[seg][SEG_LVL_ALT_L];
        lvl_seg = d.seg.abs_or_delta_update ? data : data + d.lf_level;
        lvl_seg = std::min(std::max(lvl_seg, 0), MAX_LOOP_FILTER);
      }
      for (int rf = 0; rf < 4; ++rf)
        for (int mode = 0; mode < 2; ++mode) {
          int v = lvl_seg;
          if (d.lf_delta_enabled) {
            v = lvl_seg + d.lf_ref_deltas[rf] * (1 << n_shift);
            if (rf > 0) v += d.lf_mode_deltas[mode] * (1 << n_shift);
          }
          k.lvl[seg][rf][mode] = (uint8_t)std::min(std::max(v, 0), MAX_LOOP_FILTER);
        }
    }
    int shift = d.lf_sharpness > 4 ? 2 : (d.lf_sharpness > 0 ? 1 : 0);
    for (int l = 0; l < 64; ++l) {
      int limit = l >> shift;
      if (d.lf_sharpness > 0) limit = std::min(limit, 9 - (int)d.lf_sharpness);
      limit = std::max(limit, 1);
      k.lf_limit[l] = (uint8_t)limit;
      k.lf_blimit[l] = (uint8_t)(2 * (l + 2) + limit);
      k.lf_thresh[l] = (uint8_t)(l >> 4);
    }
  }
  if (fixed_) {
    size_t flags = align256(n_sb * 4);
    k.counters = (int32_t*)fixed_;
    k.error = k.counters + 2;
    k.sb_done = (uint32_t*)(fixed_ + 256);
    k.lf_mi = (uint32_t*)(fixed_ + 256 + flags);
    k.epoch = 1;
  } else {
    k.lf_mi = d_lf_mi_;
    k.sb_done = d_sb_done_;
    k.epoch = epoch_;
    k.counters = d_counters_;
    k.error = d_counters_ + 2;
  }
  k.wait_limit = wait_limit_;
  k.test_skip = (int32_t)test_skip_;
  *out = cur;
  return rv9::ST_OK;
}

void Engine::commit_frame(const FrameWork& fw, DevFrame* cur, DevFrame** shown) {
  *shown = nullptr;
  if (fw.show_existing) {
    *shown = slots_[fw.show_slot];
    return;
  }
  ++frames;
  alg_bytes += fw.total_bytes;
  // Reference update (8.10 step 1).
  for (int i = 0; i < 8; ++i)
    if ((fw.refresh_mask >> i) & 1) {
      if (slots_[i]) --slots_[i]->refs;
      slots_[i] = cur;
      ++cur->refs;
    }
  if (fw.show_frame) *shown = cur;
}

rv9::Status Engine::run_frame(const FrameWork& fw, const uint8_t* d_base, bool per_kernel, DevFrame** shown,
                              std::string* err) {
  *shown = nullptr;
  KFrame k;
  DevFrame* cur = nullptr;
  rv9::Status st = prepare_frame(fw, d_base, stream_, &k, &cur, err);
  if (st != rv9::ST_OK) return st;
  if (!cur) {
    commit_frame(fw, nullptr, shown);
    return sink_frame(*shown, stream_, err);
  }
  if (!fixed_) CK(cudaMemsetAsync(d_counters_, 0, 8, stream_));
  int L = 0;
  cur_fw_ = &fw;
  TuneParams tune;
  if (tune_override_) {
    tune = *tune_override_;
  } else {
    auto it = tuned_.find(geometry_key(fw.desc));
    if (it != tuned_.end()) tune = it->second;
  }
  // Captured graphs keep every launch on the one stream: replays of graphs
  // with the fork's branches measured slower than without them.
  CK(launch_frame(k, (int)fw.n_blocks, stream_, n_sm_, &L, per_kernel ? &Engine::hook : nullptr, this, tune,
                  capturing_ ? nullptr : &aux_));
  cur_fw_ = nullptr;
  // The device's error word, read at the next sync.
  CK(cudaMemcpyAsync(h_error_ + 1, k.error, 4, cudaMemcpyDeviceToHost, stream_));
  launches += L;
  commit_frame(fw, cur, shown);
  return sink_frame(*shown, stream_, err);
}

rv9::Status Engine::recon(const rv9::ParsedFrame& pf, DevFrame** shown, std::string* err) {
  FrameWork fw;
  if (pf.show_existing) {
    build_work(pf, &fw, StageReserve());
    return run_frame(fw, nullptr, false, shown, err);
  }
  // The frame's bytes go straight into the pinned buffer of this turn (its
  // previous copy done), then one copy to the device.
  int s = stage_;
  stage_ ^= 1;
  CK(cudaEventSynchronize(stage_ev_[s]));
  cudaError_t alloc_err = cudaSuccess;
  auto reserve = [&](size_t n, size_t* base) -> uint8_t* {
    *base = 0;
    if (n > h_stage_cap_[s]) {
      size_t cap = std::max(n, h_stage_cap_[s] * 3 / 2);
      cudaFreeHost(h_stage_[s]);
      h_stage_[s] = nullptr;
      h_stage_cap_[s] = 0;
      if ((alloc_err = cudaMallocHost(&h_stage_[s], cap)) != cudaSuccess) return nullptr;
      h_stage_cap_[s] = cap;
    }
    return h_stage_[s];
  };
  if (!build_work(pf, &fw, reserve)) {
    *err = std::string("pinned staging buffer: ") + cudaGetErrorString(alloc_err);
    return rv9::ST_DEVICE;
  }
  if (fw.bytes > stage_cap_[s]) {
    size_t cap = std::max(fw.bytes, stage_cap_[s] * 3 / 2);
    CK(cudaStreamSynchronize(stream_));
    cudaFree(d_stage_[s]);
    d_stage_[s] = nullptr;
    stage_cap_[s] = 0;
    CK(cudaMalloc(&d_stage_[s], cap));
    stage_cap_[s] = cap;
  }
  CK(cudaMemcpyAsync(d_stage_[s], h_stage_[s], fw.bytes, cudaMemcpyHostToDevice, stream_));
  CK(cudaEventRecord(stage_ev_[s], stream_));
  return run_frame(fw, d_stage_[s], false, shown, err);
}

rv9::Status Engine::download_async(DevFrame* f, uint8_t* dst, std::string* err) {
  return download_on(f, dst, stream_, err);
}

void Engine::digest_add(DevFrame* f, Md5Jobs* jobs, int* n) {
  if (!d_digest_ || digest_n_ >= digest_cap_) return;
  Md5Job& j = jobs->job[(*n)++];
  const size_t bps = f->bps();
  for (int p = 0; p < 3; ++p) {
    j.plane[p] = (const uint8_t*)f->planes[p];
    j.stride[p] = (int64_t)f->stride[p] * (int64_t)bps;
    j.row_bytes[p] = (uint32_t)((p ? (f->width + f->ss_x) >> f->ss_x : f->width) * bps);
    j.rows[p] = p ? (f->height + f->ss_y) >> f->ss_y : f->height;
  }
  j.out = d_digest_ + 16 * digest_n_++;
}

rv9::Status Engine::set_digests(size_t cap, std::string* err) {
  if (d_digest_) {
    CK(cudaDeviceSynchronize());
    cudaFree(d_digest_);
    d_digest_ = nullptr;
  }
  digest_cap_ = 0;
  digest_n_ = 0;
  if (cap) {
    CK(cudaMalloc(&d_digest_, cap * 16));
    digest_cap_ = cap;
  }
  return rv9::ST_OK;
}

size_t Engine::digests(uint8_t* out, size_t cap) const {
  const size_t n = std::min(cap, digest_n_);
  if (n && d_digest_ && cudaMemcpy(out, d_digest_, n * 16, cudaMemcpyDefault) != cudaSuccess) return 0;
  return digest_n_;
}

rv9::Status Engine::sink_frame(DevFrame* shown, cudaStream_t stream, std::string* err, Md5Jobs* jobs, int* n_jobs) {
  if (!shown || capturing_) return rv9::ST_OK;
  if (d_digest_) {
    if (jobs) {
      digest_add(shown, jobs, n_jobs);
      if (*n_jobs == kMd5JobsPerLaunch) {
        CK(launch_md5(*jobs, *n_jobs, stream));
        *n_jobs = 0;
      }
    } else {
      Md5Jobs one;
      int n = 0;
      digest_add(shown, &one, &n);
      CK(launch_md5(one, n, stream));
    }
  }
  if (!sink_) return rv9::ST_OK;
  const size_t nb = packed_bytes(shown);
  if (sink_used_ + nb > sink_cap_) {
    ++sink_dropped_;
    return rv9::ST_OK;
  }
  rv9::Status st = download_on(shown, sink_ + sink_used_, stream, err);
  if (st != rv9::ST_OK) return st;
  sink_used_ += nb;
  ++sink_frames_;
  return rv9::ST_OK;
}

rv9::Status Engine::download_on(DevFrame* f, uint8_t* dst, cudaStream_t stream, std::string* err) {
  size_t bps = f->bps();
  size_t off = 0;
  for (int p = 0; p < 3; ++p) {
    size_t w = p ? (f->width + f->ss_x) >> f->ss_x : f->width;
    size_t h = p ? (f->height + f->ss_y) >> f->ss_y : f->height;
    CK(cudaMemcpy2DAsync(dst + off, w * bps, f->planes[p], (size_t)f->stride[p] * bps, w * bps, h,
                         cudaMemcpyDefault, stream));
    off += w * h * bps;
  }
  return rv9::ST_OK;
}

rv9::Status Engine::sync(std::string* err) {
  CK(cudaStreamSynchronize(stream_));
  if (h_error_[1]) {
    int code = h_error_[1];
    h_error_[1] = 0;
    *err = code == 1 ? "intra wavefront wait timed out" : "loop filter wait timed out";
    // Leave the cell maps and counters consistent for what follows.
    for (DevFrame* f : pool_) cudaMemsetAsync(f->cells[0], 0, (uint8_t*)f->base + f->bytes - f->cells[0], stream_);
    cudaMemsetAsync(d_counters_, 0, 64, stream_);
    cudaStreamSynchronize(stream_);
    return rv9::ST_DEVICE;
  }
  return rv9::ST_OK;
}

rv9::Status Engine::sequence_load(const std::vector<rv9::ParsedFrame>& frames, Sequence* seq, std::string* err) {
  std::vector<uint8_t> host;
  seq->frames.resize(frames.size());
  seq->luma_samples = 0;
  auto reserve = [&](size_t n, size_t* base) -> uint8_t* {
    *base = host.size();
    host.resize(*base + n);
    return host.data() + *base;
  };
  for (size_t i = 0; i < frames.size(); ++i) {
    build_work(frames[i], &seq->frames[i], reserve);
    const rv9::ParsedFrame& pf = frames[i];
    if (pf.show_existing || pf.show_frame) {
      // Visible luma of the shown frame (show_existing shows a slot of the
      // same stream: the size of the frame last shown is a fair stand-in).
      seq->luma_samples += pf.show_existing ? 0 : (uint64_t)pf.desc.width * pf.desc.height;
    }
  }
  seq->bytes = host.size();
  CK(cudaMalloc(&seq->d_data, std::max<size_t>(host.size(), 256)));
  CK(cudaMemcpy(seq->d_data, host.data(), host.size(), cudaMemcpyHostToDevice));
  return rv9::ST_OK;
}

rv9::Status Engine::sequence_run(const Sequence& seq, bool per_kernel, float* ms, std::string* err) {
  reset_slots();
  CK(cudaEventRecord(ev0_, stream_));
  for (const FrameWork& fw : seq.frames) {
    DevFrame* shown = nullptr;
    rv9::Status st = run_frame(fw, seq.d_data, per_kernel, &shown, err);
    if (st != rv9::ST_OK) return st;
  }
  CK(cudaEventRecord(ev1_, stream_));
  rv9::Status st = sync(err);
  if (st != rv9::ST_OK) return st;
  CK(cudaEventElapsedTime(ms, ev0_, ev1_));
  device_ms += *ms;
  if (per_kernel) collect_kernel_events();
  return rv9::ST_OK;
}

rv9::Status Engine::autotune(const Sequence& seq, TuneParams* best, float* best_ms, float* default_ms,
                             std::string* err) {
  *best = TuneParams();
  *best_ms = *default_ms = 0;
  if (seq.frames.empty()) return rv9::ST_OK;
  const FrameWork* first = nullptr;
  for (const FrameWork& fw : seq.frames)
    if (!fw.show_existing) {
      first = &fw;
      break;
    }
  if (!first) return rv9::ST_OK;
  // The sequence's time with given shapes: the best of three runs after one
  // untimed run.
  auto time_with = [&](const TuneParams& tp, float* out) -> rv9::Status {
    tune_override_ = &tp;
    float ms = 0, bestr = 0;
    rv9::Status st = rv9::ST_OK;
    for (int r = 0; r < 4 && st == rv9::ST_OK; ++r) {
      st = sequence_run(seq, false, &ms, err);
      device_ms -= ms;
      if (r == 1 || (r > 1 && ms < bestr)) bestr = ms;
    }
    tune_override_ = nullptr;
    *out = bestr;
    return st;
  };
  rv9::Status st = time_with(TuneParams(), default_ms);
  if (st != rv9::ST_OK) return st;
  *best_ms = *default_ms;
  const int grains[] = {1, 2, 4, 8, 16};
  const int threads[] = {64, 128, 256};
  for (int g : grains)
    for (int t : threads) {
      TuneParams tp;
      tp.intra_ctas_per_sm_x4 = g;
      tp.inter_threads = t;
      float ms = 0;
      st = time_with(tp, &ms);
      if (st != rv9::ST_OK) return st;
      if (ms < *best_ms) {
        *best_ms = ms;
        *best = tp;
      }
    }
  {
    // The best shape with the inter fork switched.
    TuneParams tp = *best;
    tp.inter_fork = !tp.inter_fork;
    float ms = 0;
    st = time_with(tp, &ms);
    if (st != rv9::ST_OK) return st;
    if (ms < *best_ms) {
      *best_ms = ms;
      *best = tp;
    }
  }
  for (const FrameWork& fw : seq.frames)
    if (!fw.show_existing) tuned_[geometry_key(fw.desc)] = *best;
  return rv9::ST_OK;
}

rv9::Status Engine::autotune_concurrent(Engine* const* engines, const Sequence* const* seqs, size_t n,
                                        TuneParams* best, float* best_ms, float* default_ms, std::string* err) {
  *best = TuneParams();
  *best_ms = *default_ms = 0;
  if (n == 0) return rv9::ST_OK;
  // The batch's time with given shapes: the better of two runs after one
  // untimed run.
  auto time_with = [&](const TuneParams& tp, float* out) -> rv9::Status {
    for (size_t j = 0; j < n; ++j) engines[j]->tune_override_ = &tp;
    float ms = 0, bestr = 0;
    rv9::Status st = rv9::ST_OK;
    for (int r = 0; r < 3 && st == rv9::ST_OK; ++r) {
      st = run_concurrent(engines, seqs, n, false, &ms, err);
      if (r == 1 || (r > 1 && ms < bestr)) bestr = ms;
    }
    for (size_t j = 0; j < n; ++j) engines[j]->tune_override_ = nullptr;
    *out = bestr;
    return st;
  };
  rv9::Status st = time_with(TuneParams(), default_ms);
  if (st != rv9::ST_OK) return st;
  *best_ms = *default_ms;
  const int grains[] = {1, 2, 4, 8, 16};
  const int threads[] = {64, 128, 256};
  for (int g : grains)
    for (int t : threads) {
      TuneParams tp;
      tp.intra_ctas_per_sm_x4 = g;
      tp.inter_threads = t;
      float ms = 0;
      st = time_with(tp, &ms);
      if (st != rv9::ST_OK) return st;
      if (ms < *best_ms) {
        *best_ms = ms;
        *best = tp;
      }
    }
  {
    // The best shape with the inter fork switched.
    TuneParams tp = *best;
    tp.inter_fork = !tp.inter_fork;
    float ms = 0;
    st = time_with(tp, &ms);
    if (st != rv9::ST_OK) return st;
    if (ms < *best_ms) {
      *best_ms = ms;
      *best = tp;
    }
  }
  for (size_t j = 0; j < n; ++j)
    for (const FrameWork& fw : seqs[j]->frames)
      if (!fw.show_existing) engines[j]->tuned_[geometry_key(fw.desc)] = *best;
  return rv9::ST_OK;
}

rv9::Status Engine::sequence_graph(const Sequence& seq, std::string* err) {
  if (seq.graph) return rv9::ST_OK;
  float ms = 0;
  rv9::Status st = sequence_run(seq, false, &ms, err);
  if (st != rv9::ST_OK) return st;
  device_ms -= ms;
  uint64_t frames0 = frames, launches0 = launches, bytes0 = alg_bytes;
  CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaMemsetAsync(d_sb_done_, 0, sb_cap_ * 4, stream_);
  reset_slots();
  capturing_ = true;
  for (size_t i = 0; e == cudaSuccess && st == rv9::ST_OK && i < seq.frames.size(); ++i) {
    DevFrame* shown = nullptr;
    st = run_frame(seq.frames[i], seq.d_data, false, &shown, err);
  }
  capturing_ = false;
  if (e == cudaSuccess) e = cudaMemsetAsync(d_sb_done_, 0, sb_cap_ * 4, stream_);
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(stream_, &g);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess && st == rv9::ST_OK) e = cudaGraphInstantiate(&seq.graph, g, 0);
  if (g) cudaGraphDestroy(g);
  // The capture ran the host side once; the replays account for themselves.
  seq.graph_launches = launches - launches0;
  frames = frames0;
  launches = launches0;
  alg_bytes = bytes0;
  for (int i = 0; i < 8; ++i) seq.graph_slots[i] = slots_[i];
  if (st != rv9::ST_OK) return st;
  if (e != cudaSuccess) {
    seq.graph = nullptr;
    *err = std::string("capturing the sequence: ") + cudaGetErrorString(e);
    return rv9::ST_DEVICE;
  }
  return rv9::ST_OK;
}

// After a replay the reference slots are those the captured run left.
static void adopt_slots(DevFrame** slots, DevFrame* const* from) {
  for (int i = 0; i < 8; ++i) {
    if (slots[i]) --slots[i]->refs;
    slots[i] = from[i];
    if (slots[i]) ++slots[i]->refs;
  }
}

rv9::Status Engine::sequence_replay(const Sequence& seq, float* ms, std::string* err) {
  rv9::Status st = sequence_graph(seq, err);
  if (st != rv9::ST_OK) return st;
  CK(cudaEventRecord(ev0_, stream_));
  CK(cudaGraphLaunch(seq.graph, stream_));
  CK(cudaEventRecord(ev1_, stream_));
  st = sync(err);
  if (st != rv9::ST_OK) return st;
  CK(cudaEventElapsedTime(ms, ev0_, ev1_));
  adopt_slots(slots_, seq.graph_slots);
  device_ms += *ms;
  frames += seq.frames.size();
  launches += seq.graph_launches;
  for (const FrameWork& fw : seq.frames) alg_bytes += fw.total_bytes;
  return rv9::ST_OK;
}

rv9::Status Engine::run_concurrent(Engine* const* engines, const Sequence* const* seqs, size_t n, bool per_kernel,
                                   float* ms, std::string* err, bool graphs) {
  if (n == 0) {
    *ms = 0;
    return rv9::ST_OK;
  }
  Engine* e0 = engines[0];
  for (size_t j = 0; j < n; ++j) {
    if (engines[j]->device_ != e0->device_) {
      *err = "decoders on different devices";
      return rv9::ST_INVALID_INPUT;
    }
    for (size_t i = 0; i < j; ++i)
      if (engines[i] == engines[j]) {
        *err = "a decoder appears twice";
        return rv9::ST_INVALID_INPUT;
      }
  }
  if (graphs)
    for (size_t j = 0; j < n; ++j) {
      rv9::Status st = engines[j]->sequence_graph(*seqs[j], err);
      if (st != rv9::ST_OK) return st;
    }
  StreamsDrain drain{engines, n};
  // Every stream starts after the start event on engines[0]'s stream.
  CK(cudaEventRecord(e0->ev0_, e0->stream_));
  for (size_t j = 0; j < n; ++j) {
    if (!graphs) engines[j]->reset_slots();
    if (j) CK(cudaStreamWaitEvent(engines[j]->stream_, e0->ev0_, 0));
  }
  if (graphs) {
    for (size_t j = 0; j < n; ++j) {
      CK(cudaGraphLaunch(seqs[j]->graph, engines[j]->stream_));
      adopt_slots(engines[j]->slots_, seqs[j]->graph_slots);
      engines[j]->frames += seqs[j]->frames.size();
      engines[j]->launches += seqs[j]->graph_launches;
      for (const FrameWork& fw : seqs[j]->frames) engines[j]->alg_bytes += fw.total_bytes;
    }
    per_kernel = false;
  } else {
    size_t most = 0;
    for (size_t j = 0; j < n; ++j) most = std::max(most, seqs[j]->frames.size());
    for (size_t i = 0; i < most; ++i)
      for (size_t j = 0; j < n; ++j) {
        if (i >= seqs[j]->frames.size()) continue;
        DevFrame* shown = nullptr;
        rv9::Status st = engines[j]->run_frame(seqs[j]->frames[i], seqs[j]->d_data, per_kernel, &shown, err);
        if (st != rv9::ST_OK) return st;
      }
  }
  // engines[0]'s stream waits for every other stream's end.
  for (size_t j = 1; j < n; ++j) {
    CK(cudaEventRecord(engines[j]->ev1_, engines[j]->stream_));
    CK(cudaStreamWaitEvent(e0->stream_, engines[j]->ev1_, 0));
  }
  CK(cudaEventRecord(e0->ev1_, e0->stream_));
  rv9::Status first = rv9::ST_OK;
  for (size_t j = 0; j < n; ++j) {
    rv9::Status st = engines[j]->sync(err);
    if (first == rv9::ST_OK) first = st;
  }
  if (first != rv9::ST_OK) return first;
  CK(cudaEventElapsedTime(ms, e0->ev0_, e0->ev1_));
  for (size_t j = 0; j < n; ++j) {
    engines[j]->device_ms += *ms / n;
    if (per_kernel) engines[j]->collect_kernel_events();
  }
  return rv9::ST_OK;
}

rv9::Status Engine::reserve_scratch(const Sequence& seq, std::string* err) {
  size_t mi = 0, sb = 0;
  for (const FrameWork& fw : seq.frames)
    if (!fw.show_existing) {
      mi = std::max(mi, (size_t)fw.desc.mi_cols * fw.desc.mi_rows);
      sb = std::max(sb, (size_t)fw.desc.sb64_cols * fw.desc.sb64_rows);
    }
  if (mi <= lf_mi_cap_ && sb <= sb_cap_) return rv9::ST_OK;
  CK(cudaStreamSynchronize(stream_));
  if (mi > lf_mi_cap_) {
    cudaFree(d_lf_mi_);
    d_lf_mi_ = nullptr;
    lf_mi_cap_ = 0;
    CK(cudaMalloc(&d_lf_mi_, mi * 4));
    lf_mi_cap_ = mi;
  }
  if (sb > sb_cap_) {
    cudaFree(d_sb_done_);
    d_sb_done_ = nullptr;
    sb_cap_ = 0;
    CK(cudaMalloc(&d_sb_done_, sb * 4));
    CK(cudaMemsetAsync(d_sb_done_, 0, sb * 4, stream_));
    CK(cudaStreamSynchronize(stream_));
    sb_cap_ = sb;
  }
  return rv9::ST_OK;
}

size_t Engine::step_table_bytes(size_t n) { return 2 * batch_table_bytes((int)n); }

rv9::Status Engine::launch_step(Engine* const* engines, const FrameWork* const* fws, const uint8_t* const* bases,
                                size_t n, cudaStream_t s, const TuneParams& tune, uint8_t* h_tables,
                                uint8_t* d_tables, size_t* table_bytes, DevFrame** shown, int* launches,
                                std::string* err) {
  *table_bytes = 0;
  Md5Jobs jobs;
  int n_jobs = 0;
  std::vector<KFrame> ks;
  std::vector<int> nb;
  std::vector<DevFrame*> curs;
  std::vector<size_t> who;
  const int n_sm = n ? engines[0]->n_sm_ : 0;
  for (int c = 0; c < 2; ++c) {
    ks.clear();
    nb.clear();
    curs.clear();
    who.clear();
    for (size_t q = 0; q < n; ++q) {
      const FrameWork& fw = *fws[q];
      // Kernels are typed by sample size: 8-bit frames (and frames that only
      // show an existing one) in the first launch set, deeper ones in the second.
      if ((fw.show_existing ? 0 : (fw.desc.bit_depth > 8 ? 1 : 0)) != c) continue;
      Engine* e = engines[q];
      KFrame k;
      DevFrame* cur = nullptr;
      rv9::Status st = e->prepare_frame(fw, bases[q], s, &k, &cur, err);
      if (st != rv9::ST_OK) return st;
      if (!cur) {
        e->commit_frame(fw, nullptr, &shown[q]);
        st = e->sink_frame(shown[q], s, err, &jobs, &n_jobs);
        if (st != rv9::ST_OK) return st;
        continue;
      }
      ks.push_back(k);
      nb.push_back((int)fw.n_blocks);
      curs.push_back(cur);
      who.push_back(q);
    }
    if (ks.empty()) continue;
    const int nf = (int)ks.size();
    BatchTotals tot;
    batch_fill(ks.data(), nb.data(), nf, h_tables + *table_bytes, &tot, n_sm, tune);
    const size_t bytes = batch_table_bytes(nf);
    CK(cudaMemcpyAsync(d_tables + *table_bytes, h_tables + *table_bytes, bytes, cudaMemcpyHostToDevice, s));
    CK(launch_batch(d_tables + *table_bytes, nf, tot, c == 1, s, n_sm, tune, launches));
    *table_bytes += bytes;
    for (int f = 0; f < nf; ++f) {
      Engine* e = engines[who[f]];
      e->commit_frame(*fws[who[f]], curs[f], &shown[who[f]]);
      // The frame's error word, for sync() and error_word().
      CK(cudaMemcpyAsync(e->h_error_ + 1, e->d_counters_ + 2, 4, cudaMemcpyDeviceToHost, s));
      rv9::Status st = e->sink_frame(shown[who[f]], s, err, &jobs, &n_jobs);
      if (st != rv9::ST_OK) return st;
    }
  }
  CK(launch_md5(jobs, n_jobs, s));
  return rv9::ST_OK;
}

rv9::Status Engine::stage(const rv9::ParsedFrame& pf, cudaStream_t s, FrameWork* fw, const uint8_t** d_base,
                          std::string* err) {
  *d_base = nullptr;
  if (pf.show_existing) {
    build_work(pf, fw, StageReserve());
    return rv9::ST_OK;
  }
  // As recon(): the frame's bytes straight into the pinned buffer of this
  // turn (its previous copy done), then one copy to the device, on `s`.
  int b = stage_;
  stage_ ^= 1;
  CK(cudaEventSynchronize(stage_ev_[b]));
  cudaError_t alloc_err = cudaSuccess;
  auto reserve = [&](size_t bytes, size_t* base) -> uint8_t* {
    *base = 0;
    if (bytes > h_stage_cap_[b]) {
      size_t cap = std::max(bytes, h_stage_cap_[b] * 3 / 2);
      cudaFreeHost(h_stage_[b]);
      h_stage_[b] = nullptr;
      h_stage_cap_[b] = 0;
      if ((alloc_err = cudaMallocHost(&h_stage_[b], cap)) != cudaSuccess) return nullptr;
      h_stage_cap_[b] = cap;
    }
    return h_stage_[b];
  };
  if (!build_work(pf, fw, reserve)) {
    *err = std::string("pinned staging buffer: ") + cudaGetErrorString(alloc_err);
    return rv9::ST_DEVICE;
  }
  if (fw->bytes > stage_cap_[b]) {
    size_t cap = std::max(fw->bytes, stage_cap_[b] * 3 / 2);
    CK(cudaStreamSynchronize(s));
    cudaFree(d_stage_[b]);
    d_stage_[b] = nullptr;
    stage_cap_[b] = 0;
    CK(cudaMalloc(&d_stage_[b], cap));
    stage_cap_[b] = cap;
  }
  CK(cudaMemcpyAsync(d_stage_[b], h_stage_[b], fw->bytes, cudaMemcpyHostToDevice, s));
  CK(cudaEventRecord(stage_ev_[b], s));
  *d_base = d_stage_[b];
  return rv9::ST_OK;
}

rv9::Status Engine::run_batched(Engine* const* engines, const Sequence* const* seqs, size_t n, int groups,
                                float* ms, std::string* err) {
  *ms = 0;
  if (n == 0) return rv9::ST_OK;
  Engine* e0 = engines[0];
  for (size_t j = 0; j < n; ++j) {
    if (engines[j]->device_ != e0->device_) {
      *err = "decoders on different devices";
      return rv9::ST_INVALID_INPUT;
    }
    for (size_t i = 0; i < j; ++i)
      if (engines[i] == engines[j]) {
        *err = "a decoder appears twice";
        return rv9::ST_INVALID_INPUT;
      }
  }
  const size_t G = std::min<size_t>(std::max(groups, 1), n);
  size_t most = 0;
  for (size_t j = 0; j < n; ++j) {
    rv9::Status st = engines[j]->reserve_scratch(*seqs[j], err);
    if (st != rv9::ST_OK) return st;
    CK(cudaStreamSynchronize(engines[j]->stream_));
    engines[j]->reset_slots();
    most = std::max(most, seqs[j]->frames.size());
  }
  // Every step of the run has its own region of the tables, so that no
  // copy waits for an earlier step's launches.
  size_t total = 0;
  for (size_t i = 0; i < most; ++i)
    for (size_t g = 0; g < G; ++g) {
      size_t cnt = 0;
      for (size_t j = g; j < n; j += G)
        if (i < seqs[j]->frames.size()) ++cnt;
      if (cnt) total += step_table_bytes(cnt);
    }
  if (total > e0->batch_cap_) {
    cudaFree(e0->batch_d_);
    cudaFreeHost(e0->batch_h_);
    e0->batch_d_ = e0->batch_h_ = nullptr;
    e0->batch_cap_ = 0;
    CK(cudaMalloc(&e0->batch_d_, total));
    CK(cudaMallocHost(&e0->batch_h_, total));
    e0->batch_cap_ = total;
  }
  StreamsDrain drain{engines, G};
  // Each group's stream starts after the start event on engines[0]'s.
  CK(cudaEventRecord(e0->ev0_, e0->stream_));
  for (size_t g = 1; g < G; ++g) CK(cudaStreamWaitEvent(engines[g]->stream_, e0->ev0_, 0));
  std::vector<Engine*> step_engines;
  std::vector<const FrameWork*> step_fws;
  std::vector<const uint8_t*> step_bases;
  std::vector<DevFrame*> shown;
  size_t off = 0;
  int L = 0;
  for (size_t i = 0; i < most; ++i)
    for (size_t g = 0; g < G; ++g) {
      step_engines.clear();
      step_fws.clear();
      step_bases.clear();
      for (size_t j = g; j < n; j += G) {
        if (i >= seqs[j]->frames.size()) continue;
        step_engines.push_back(engines[j]);
        step_fws.push_back(&seqs[j]->frames[i]);
        step_bases.push_back(seqs[j]->d_data);
      }
      if (step_engines.empty()) continue;
      shown.assign(step_engines.size(), nullptr);
      size_t used = 0;
      rv9::Status st = launch_step(step_engines.data(), step_fws.data(), step_bases.data(), step_engines.size(),
                                   engines[g]->stream_, e0->batch_tune_, e0->batch_h_ + off, e0->batch_d_ + off,
                                   &used, shown.data(), &L, err);
      if (st != rv9::ST_OK) return st;
      off += used;
    }
  // engines[0]'s stream waits for every group's end.
  for (size_t g = 1; g < G; ++g) {
    CK(cudaEventRecord(engines[g]->ev1_, engines[g]->stream_));
    CK(cudaStreamWaitEvent(e0->stream_, engines[g]->ev1_, 0));
  }
  CK(cudaEventRecord(e0->ev1_, e0->stream_));
  CK(cudaStreamSynchronize(e0->stream_));
  e0->launches += L;
  // Each decoder's error word (its frames' waits), as sync() reports it.
  rv9::Status first = rv9::ST_OK;
  for (size_t j = 0; j < n; ++j) {
    CK(cudaMemcpy(engines[j]->h_error_ + 1, engines[j]->d_counters_ + 2, 4, cudaMemcpyDeviceToHost));
    rv9::Status st = engines[j]->sync(err);
    if (first == rv9::ST_OK) first = st;
  }
  if (first != rv9::ST_OK) return first;
  CK(cudaEventElapsedTime(ms, e0->ev0_, e0->ev1_));
  for (size_t j = 0; j < n; ++j) engines[j]->device_ms += *ms / n;
  return rv9::ST_OK;
}

rv9::Status Engine::autotune_batched(Engine* const* engines, const Sequence* const* seqs, size_t n, int* groups,
                                    TuneParams* best, float* best_ms, float* default_ms, std::string* err) {
  *groups = 1;
  *best = TuneParams();
  *best_ms = *default_ms = 0;
  if (n == 0) return rv9::ST_OK;
  Engine* e0 = engines[0];
  // The batch's time with given shapes: the better of two runs after one
  // untimed run.
  auto time_with = [&](int g, const TuneParams& tp, float* out) -> rv9::Status {
    e0->batch_tune_ = tp;
    float ms = 0, bestr = 0;
    rv9::Status st = rv9::ST_OK;
    for (int r = 0; r < 3 && st == rv9::ST_OK; ++r) {
      st = run_batched(engines, seqs, n, g, &ms, err);
      if (r == 1 || (r > 1 && ms < bestr)) bestr = ms;
    }
    *out = bestr;
    return st;
  };
  rv9::Status st = time_with(1, TuneParams(), default_ms);
  if (st != rv9::ST_OK) return st;
  *best_ms = *default_ms;
  const int group_counts[] = {1, 2, 4, 8};
  const int grains[] = {2, 4, 8};
  for (int g : group_counts) {
    if ((size_t)g > n) break;
    for (int gr : grains) {
      if (g == 1 && gr == TuneParams().intra_ctas_per_sm_x4) continue;  // the defaults, timed above
      TuneParams tp;
      tp.intra_ctas_per_sm_x4 = gr;
      float ms = 0;
      st = time_with(g, tp, &ms);
      if (st != rv9::ST_OK) return st;
      if (ms < *best_ms) {
        *best_ms = ms;
        *best = tp;
        *groups = g;
      }
    }
  }
  e0->batch_tune_ = *best;
  return rv9::ST_OK;
}

static rv9_frame_desc geometry_desc(uint32_t width, uint32_t height, uint32_t ss_x, uint32_t ss_y, uint32_t bd) {
  rv9_frame_desc d;
  memset(&d, 0, sizeof d);
  d.width = width;
  d.height = height;
  d.mi_cols = (width + 7) >> 3;
  d.mi_rows = (height + 7) >> 3;
  d.sb64_cols = (d.mi_cols + 7) >> 3;
  d.sb64_rows = (d.mi_rows + 7) >> 3;
  d.ss_x = ss_x;
  d.ss_y = ss_y;
  d.bit_depth = bd;
  return d;
}

size_t Engine::footprint(uint32_t width, uint32_t height, uint32_t ss_x, uint32_t ss_y, uint32_t bit_depth,
                         int n_frames, size_t stage_bytes) {
  rv9_frame_desc d = geometry_desc(width, height, ss_x, ss_y, bit_depth);
  uint32_t aw = d.sb64_cols * 64, ah = d.sb64_rows * 64;
  size_t bps = bit_depth > 8 ? 2 : 1, frame = 0;
  for (int p = 0; p < 3; ++p) {
    size_t w = p ? (aw >> ss_x) : aw, h = p ? (ah >> ss_y) : ah;
    frame += align256(w * h * bps) + align256((w / 4) * (h / 4));
  }
  return (size_t)n_frames * frame + 2 * stage_bytes + (size_t)d.mi_cols * d.mi_rows * 4 +
         (size_t)d.sb64_cols * d.sb64_rows * 4 + 64;
}

rv9::Status Engine::reserve(uint32_t width, uint32_t height, uint32_t ss_x, uint32_t ss_y, uint32_t bit_depth,
                            int n_frames, size_t stage_bytes, std::string* err) {
  rv9_frame_desc d = geometry_desc(width, height, ss_x, ss_y, bit_depth);
  // Distinct frames: hold each one while taking the next.
  std::vector<DevFrame*> held;
  for (int i = 0; i < n_frames; ++i) {
    DevFrame* f = alloc_frame(d, stream_);
    if (!f) {
      for (DevFrame* h : held) --h->refs;
      *err = "out of device memory reserving frames";
      return rv9::ST_DEVICE;
    }
    ++f->refs;
    held.push_back(f);
  }
  for (DevFrame* h : held) --h->refs;
  for (int s = 0; s < 2; ++s) {
    if (stage_bytes > stage_cap_[s]) {
      CK(cudaStreamSynchronize(stream_));
      cudaFree(d_stage_[s]);
      d_stage_[s] = nullptr;
      stage_cap_[s] = 0;
      CK(cudaMalloc(&d_stage_[s], stage_bytes));
      stage_cap_[s] = stage_bytes;
    }
    if (stage_bytes > h_stage_cap_[s]) {
      CK(cudaStreamSynchronize(stream_));
      cudaFreeHost(h_stage_[s]);
      h_stage_[s] = nullptr;
      h_stage_cap_[s] = 0;
      CK(cudaMallocHost(&h_stage_[s], stage_bytes));
      h_stage_cap_[s] = stage_bytes;
    }
  }
  size_t mi_len = (size_t)d.mi_cols * d.mi_rows;
  if (mi_len > lf_mi_cap_) {
    CK(cudaStreamSynchronize(stream_));
    cudaFree(d_lf_mi_);
    CK(cudaMalloc(&d_lf_mi_, mi_len * 4));
    lf_mi_cap_ = mi_len;
  }
  size_t n_sb = (size_t)d.sb64_cols * d.sb64_rows;
  if (n_sb > sb_cap_) {
    CK(cudaStreamSynchronize(stream_));
    cudaFree(d_sb_done_);
    CK(cudaMalloc(&d_sb_done_, n_sb * 4));
    CK(cudaMemsetAsync(d_sb_done_, 0, n_sb * 4, stream_));
    sb_cap_ = n_sb;
  }
  CK(cudaStreamSynchronize(stream_));
  return rv9::ST_OK;
}

size_t fixed_scratch_need(uint32_t mi_cols, uint32_t mi_rows, uint32_t sb64_cols, uint32_t sb64_rows) {
  return 256 + align256((size_t)sb64_cols * sb64_rows * 4) + (size_t)mi_cols * mi_rows * 4;
}

// Replays alloc_frame's choices over the sequence with reference counts only:
// true when every frame the run takes is already in the pool.
bool Engine::pool_covers(const Sequence& seq) {
  DevFrame* sim_slots[8] = {nullptr};
  for (DevFrame* f : pool_) f->sim_refs = 0;
  for (const FrameWork& fw : seq.frames) {
    if (fw.show_existing) continue;
    const rv9_frame_desc& d = fw.desc;
    uint32_t aw = d.sb64_cols * 64, ah = d.sb64_rows * 64;
    DevFrame* cur = nullptr;
    for (DevFrame* f : pool_) {
      if (f->sim_refs == 0 && f->aw == aw && f->ah == ah && f->ss_x == d.ss_x && f->ss_y == d.ss_y &&
          f->bit_depth == d.bit_depth) {
        cur = f;
        break;
      }
    }
    if (!cur) return false;
    for (int i = 0; i < 8; ++i)
      if ((fw.refresh_mask >> i) & 1) {
        if (sim_slots[i]) --sim_slots[i]->sim_refs;
        sim_slots[i] = cur;
        ++cur->sim_refs;
      }
  }
  return true;
}

rv9::Status Engine::sequence_run_fixed(const Sequence& seq, float* ms, std::string* err) {
  for (const FrameWork& fw : seq.frames) {
    if (fw.show_existing) continue;
    const rv9_frame_desc& d = fw.desc;
    if (fixed_scratch_need(d.mi_cols, d.mi_rows, d.sb64_cols, d.sb64_rows) > kFixedScratchBytes) {
      *err = "frame too large for the fixed scratch array (1 MiB: 256 + 4 per superblock + 4 per 8x8 block)";
      return rv9::ST_INVALID_INPUT;
    }
  }
  int prev = -1;
  CK(cudaGetDevice(&prev));
  if (prev != device_) CK(cudaSetDevice(device_));
  void* scratch = nullptr;
  cudaError_t rc = fixed_scratch_address(device_, &scratch);
  rv9::Status st = rv9::ST_OK;
  if (rc != cudaSuccess) {
    *err = std::string("cudaGetSymbolAddress of the fixed scratch: ") + cudaGetErrorString(rc);
    st = rv9::ST_DEVICE;
  } else if (!pool_covers(seq)) {
    // Checked before anything changes: the pool is simulated with every
    // frame free, as it is once the slots are emptied below.
    *err = "the frame pool lacks frames this sequence needs (allocating nothing, it reuses the frames an "
           "earlier rv9_sequence_run of the sequence left in the pool)";
    st = rv9::ST_INVALID_INPUT;
  }
  if (st == rv9::ST_OK) {
    // Slots are emptied first, as in sequence_run; the run's tickets and
    // error word start at zero.
    reset_slots();
    fixed_ = (uint8_t*)scratch;
    rc = cudaMemsetAsync(fixed_, 0, 256, stream_);
    if (rc == cudaSuccess) rc = cudaEventRecord(ev0_, stream_);
    for (size_t i = 0; rc == cudaSuccess && st == rv9::ST_OK && i < seq.frames.size(); ++i) {
      DevFrame* shown = nullptr;
      st = run_frame(seq.frames[i], seq.d_data, false, &shown, err);
    }
    fixed_ = nullptr;
    if (rc == cudaSuccess && st == rv9::ST_OK) rc = cudaEventRecord(ev1_, stream_);
    if (rc != cudaSuccess) {
      *err = cudaGetErrorString(rc);
      st = rv9::ST_DEVICE;
    }
    if (st == rv9::ST_OK) st = sync(err);
    if (st == rv9::ST_OK && (rc = cudaEventElapsedTime(ms, ev0_, ev1_)) != cudaSuccess) {
      *err = cudaGetErrorString(rc);
      st = rv9::ST_DEVICE;
    }
    if (st == rv9::ST_OK) device_ms += *ms;
  }
  if (prev != device_) cudaSetDevice(prev);
  return st;
}

rv9::Status Engine::sequence_clone(const Sequence& src, Sequence* seq, std::string* err) {
  seq->frames = src.frames;
  seq->bytes = src.bytes;
  seq->luma_samples = src.luma_samples;
  CK(cudaMalloc(&seq->d_data, std::max<size_t>(src.bytes, 256)));
  CK(cudaMemcpy(seq->d_data, src.d_data, src.bytes, cudaMemcpyDeviceToDevice));
  return rv9::ST_OK;
}

void Engine::sequence_free(Sequence* seq) {
  if (seq->graph) {
    cudaStreamSynchronize(stream_);
    cudaGraphExecDestroy(seq->graph);
    seq->graph = nullptr;
  }
  if (seq->d_data) {
    cudaStreamSynchronize(stream_);
    cudaFree(seq->d_data);
  }
  seq->d_data = nullptr;
  seq->frames.clear();
}

}  // namespace rv9g

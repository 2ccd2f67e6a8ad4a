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

#define CK(call)                                           \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) {                               \
      *err = std::string(#call) + ": " + cudaGetErrorString(e_); \
      return rv9::ST_DEVICE;                               \
    }                                                      \
  } while (0)

Engine::~Engine() {
  if (stream_) cudaStreamSynchronize(stream_);
  for (DevFrame* f : pool_) {
    if (f->ready) cudaEventDestroy(f->ready);
    cudaFree(f->base);
    delete f;
  }
  cudaFree(d_scratch_);
  cudaFreeHost(h_scratch_);
  cudaFree(d_lf_mi_);
  cudaFree(d_sb_done_);
  cudaFree(d_counters_);
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  if (stream_) cudaStreamDestroy(stream_);
}

bool Engine::init(int device, std::string* err) {
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
  if ((e = cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreate(&ev0_)) != cudaSuccess || (e = cudaEventCreate(&ev1_)) != cudaSuccess ||
      (e = cudaMalloc(&d_counters_, 64)) != cudaSuccess) {
    *err = cudaGetErrorString(e);
    return false;
  }
  int16_t f[4][16][8];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 16; ++b)
      for (int c = 0; c < 8; ++c) f[a][b][c] = (int16_t)vp9t_subpel_filters[a][b][c];
  if ((e = upload_filters(&f[0][0][0])) != cudaSuccess) {
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

DevFrame* Engine::alloc_frame(const rv9_frame_desc& d) {
  uint32_t aw = d.sb64_cols * 64, ah = d.sb64_rows * 64;
  for (DevFrame* f : pool_) {
    if (f->refs == 0 && !f->busy && f->aw == aw && f->ah == ah && f->ss_x == d.ss_x && f->ss_y == d.ss_y &&
        f->bit_depth == d.bit_depth)
      return f;
  }
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
    off += ((size_t)w * h * bps + 255) & ~(size_t)255;
  }
  for (int p = 0; p < 3; ++p) {
    f->cell_stride[p] = f->stride[p] / 4;
    cell_off[p] = off;
    off += ((size_t)f->cell_stride[p] * (f->pheight[p] / 4) + 255) & ~(size_t)255;
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
  cudaMemsetAsync(f->base, 0, off, stream_);
  cudaEventCreateWithFlags(&f->ready, cudaEventDisableTiming);
  pool_.push_back(f);
  return f;
}

void Engine::release_ref(DevFrame* f) {
  if (f) --f->refs;
}

bool Engine::ensure_scratch(size_t bytes, std::string* err) {
  if (bytes <= scratch_cap_) return true;
  size_t cap = std::max(bytes, scratch_cap_ * 3 / 2);
  cudaStreamSynchronize(stream_);
  cudaFree(d_scratch_);
  cudaFreeHost(h_scratch_);
  d_scratch_ = nullptr;
  h_scratch_ = nullptr;
  scratch_cap_ = 0;
  if (cudaMalloc(&d_scratch_, cap) != cudaSuccess || cudaMallocHost(&h_scratch_, cap) != cudaSuccess) {
    *err = "out of memory for frame records";
    return false;
  }
  scratch_cap_ = cap;
  return true;
}

static int uv_tx_size(const rv9_frame_desc& d, const rv9_block& b) {
  if (b.mi_size < BLOCK_8X8) return TX_4X4;
  int sx = d.legacy_uv ? 1 : d.ss_x, sy = d.legacy_uv ? 1 : d.ss_y;
  int uv = SS_SIZE_LOOKUP[b.mi_size][sx][sy];
  return std::min<int>(b.tx_size, MAX_TXSIZE_LOOKUP[uv]);
}

// The work lists: the prediction regions and residuals of inter blocks, and
// the intra transform blocks in bitstream order (replay's loop structure).
void Engine::build_work(const rv9::ParsedFrame& pf) {
  const rv9_frame_desc& d = pf.desc;
  units_.clear();
  res_.clear();
  intra_.clear();
  const size_t bps = d.bit_depth > 8 ? 2 : 1;
  uint64_t ref_bytes = 0;
  for (uint32_t bi = 0; bi < pf.blocks.size(); ++bi) {
    const rv9_block& b = pf.blocks[bi];
    const bool is_inter = b.flags & RV9_BLK_INTER;
    const bool avail_l = b.flags & RV9_BLK_AVAIL_L, avail_u = b.flags & RV9_BLK_AVAIL_U;
    const int bsize = std::max<int>(b.mi_size, BLOCK_8X8);
    const int nrefs = b.ref_frame[1] > INTRA_FRAME ? 2 : 1;
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
              units_.push_back(InterUnit{bi, (uint16_t)(base_x + 4 * x), (uint16_t)(base_y + 4 * y), (uint8_t)plane, 1,
                                         1, (uint8_t)(y * n4w + x)});
        } else {
          units_.push_back(
              InterUnit{bi, (uint16_t)base_x, (uint16_t)base_y, (uint8_t)plane, (uint8_t)n4w, (uint8_t)n4h, 0});
        }
        ref_bytes += (uint64_t)n4w * n4h * 16 * bps * nrefs;
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
            if (is_inter) {
              if (t != NO_TOK) res_.push_back(ResItem{t, bi});
            } else {
              int mode = plane ? b.uv_mode : (b.mi_size >= BLOCK_8X8 ? b.y_mode : b.sub_modes[block_idx]);
              uint8_t fl = (uint8_t)((avail_l || x > 0 ? 1 : 0) | (avail_u || y > 0 ? 2 : 0) | (x + step < n4w ? 4 : 0));
              intra_.push_back(IntraItem{bi, t, (uint16_t)start_x, (uint16_t)start_y, (uint8_t)plane, (uint8_t)tx_sz,
                                         (uint8_t)mode, fl});
            }
          }
          ++block_idx;
        }
    }
  }
  uint64_t out_bytes = (uint64_t)d.mi_cols * 8 * d.mi_rows * 8 * bps;
  out_bytes += 2 * (((uint64_t)d.mi_cols * 8) >> d.ss_x) * (((uint64_t)d.mi_rows * 8) >> d.ss_y) * bps;
  uint64_t rec_bytes = pf.blocks.size() * sizeof(rv9_block) + pf.toks.size() * sizeof(rv9_tok) + pf.coefs.size() * 4;
  alg_bytes += out_bytes + ref_bytes + rec_bytes;
}

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

rv9::Status Engine::recon(rv9::ParsedFrame& pf, DevFrame** shown, std::string* err) {
  *shown = nullptr;
  if (pf.show_existing) {
    *shown = slots_[pf.show_slot];
    if (!*shown) {
      *err = "show_existing_frame of an empty slot";
      return rv9::ST_BITSTREAM;
    }
    return rv9::ST_OK;
  }
  const rv9_frame_desc& d = pf.desc;
  DevFrame* cur = alloc_frame(d);
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
  build_work(pf);
  // Stage records and work lists in one pinned buffer, one copy.
  size_t o_blocks = 0;
  size_t o_toks = align256(o_blocks + pf.blocks.size() * sizeof(rv9_block));
  size_t o_coefs = align256(o_toks + pf.toks.size() * sizeof(rv9_tok));
  size_t o_units = align256(o_coefs + pf.coefs.size() * 4);
  size_t o_res = align256(o_units + units_.size() * sizeof(InterUnit));
  size_t o_intra = align256(o_res + res_.size() * sizeof(ResItem));
  size_t total = align256(o_intra + intra_.size() * sizeof(IntraItem));
  if (!ensure_scratch(total, err)) return rv9::ST_DEVICE;
  memcpy(h_scratch_ + o_blocks, pf.blocks.data(), pf.blocks.size() * sizeof(rv9_block));
  memcpy(h_scratch_ + o_toks, pf.toks.data(), pf.toks.size() * sizeof(rv9_tok));
  memcpy(h_scratch_ + o_coefs, pf.coefs.data(), pf.coefs.size() * 4);
  memcpy(h_scratch_ + o_units, units_.data(), units_.size() * sizeof(InterUnit));
  memcpy(h_scratch_ + o_res, res_.data(), res_.size() * sizeof(ResItem));
  memcpy(h_scratch_ + o_intra, intra_.data(), intra_.size() * sizeof(IntraItem));
  CK(cudaMemcpyAsync(d_scratch_, h_scratch_, total, cudaMemcpyHostToDevice, stream_));
  // Loop filter scratch.
  size_t mi_len = (size_t)d.mi_cols * d.mi_rows;
  if (mi_len > lf_mi_cap_) {
    cudaFree(d_lf_mi_);
    CK(cudaMalloc(&d_lf_mi_, mi_len * 4));
    lf_mi_cap_ = mi_len;
  }
  size_t n_sb = (size_t)d.sb64_cols * d.sb64_rows;
  if (n_sb > sb_cap_) {
    cudaFree(d_sb_done_);
    CK(cudaMalloc(&d_sb_done_, n_sb * 4));
    CK(cudaMemsetAsync(d_sb_done_, 0, n_sb * 4, stream_));
    sb_cap_ = n_sb;
  }
  ++epoch_;
  if (epoch_ == 0) {
    CK(cudaMemsetAsync(d_sb_done_, 0, sb_cap_ * 4, stream_));
    epoch_ = 1;
  }
  // The frame's kernel arguments.
  KFrame k;
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
      DevFrame* r = slots_[pf.ref_slot[i]];
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
  for (int seg = 0; seg < 8; ++seg) {
    int q = d.base_q_idx;
    if (d.seg.enabled && d.seg.feature_enabled[seg][SEG_LVL_ALT_Q]) {
      int data = d.seg.feature_data[seg][SEG_LVL_ALT_Q];
      if (!d.seg.abs_or_delta_update) data += d.base_q_idx;
      q = std::min(std::max(data, 0), 255);
    }
    auto cq = [](int v) { return std::min(std::max(v, 0), 255); };
    k.dc_q[seg][0] = vp9t_dc_qlookup[bd_idx][cq(q + d.delta_q_y_dc)];
    k.ac_q[seg][0] = vp9t_ac_qlookup[bd_idx][cq(q)];
    k.dc_q[seg][1] = vp9t_dc_qlookup[bd_idx][cq(q + d.delta_q_uv_dc)];
    k.ac_q[seg][1] = vp9t_ac_qlookup[bd_idx][cq(q + d.delta_q_uv_ac)];
  }
  k.blocks = (const rv9_block*)(d_scratch_ + o_blocks);
  k.toks = (const rv9_tok*)(d_scratch_ + o_toks);
  k.coefs = (const uint32_t*)(d_scratch_ + o_coefs);
  k.units = (const InterUnit*)(d_scratch_ + o_units);
  k.n_units = (int32_t)units_.size();
  k.res = (const ResItem*)(d_scratch_ + o_res);
  k.n_res = (int32_t)res_.size();
  k.intra = (const IntraItem*)(d_scratch_ + o_intra);
  k.n_intra = (int32_t)intra_.size();
  // Loop filter levels and limits (8.8.1; reference loopfilter.rs:15-47,
  // 135-170).
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
  k.lf_mi = d_lf_mi_;
  k.sb_done = d_sb_done_;
  k.epoch = epoch_;
  k.counters = d_counters_;
  k.error = d_counters_ + 2;
  CK(cudaMemsetAsync(d_counters_, 0, 8, stream_));
  CK(cudaEventRecord(ev0_, stream_));
  int L = 0;
  CK(launch_frame(k, (int)pf.blocks.size(), stream_, n_sm_, &L));
  CK(cudaEventRecord(ev1_, stream_));
  launches += L;
  ++frames;
  // The staging buffer is reused by the next frame: wait for the copy (the
  // kernels keep running).
  CK(cudaEventSynchronize(ev0_));
  // Device time of the previous frames' kernels is accumulated lazily.
  float ms = 0;
  CK(cudaEventSynchronize(ev1_));
  CK(cudaEventElapsedTime(&ms, ev0_, ev1_));
  device_ms += ms;
  int32_t dev_err = 0;
  CK(cudaMemcpy(&dev_err, d_counters_ + 2, 4, cudaMemcpyDeviceToHost));
  if (dev_err) {
    *err = dev_err == 1 ? "intra wavefront wait timed out" : "loop filter wait timed out";
    // Leave the cell maps consistent for the next frame.
    cudaMemsetAsync(cur->base, 0, cur->bytes, stream_);
    cudaMemsetAsync(d_counters_, 0, 64, stream_);
    return rv9::ST_DEVICE;
  }
  // Reference update (8.10 step 1).
  for (int i = 0; i < 8; ++i)
    if ((pf.refresh_mask >> i) & 1) {
      release_ref(slots_[i]);
      slots_[i] = cur;
      ++cur->refs;
    }
  if (pf.show_frame) *shown = cur;
  return rv9::ST_OK;
}

rv9::Status Engine::download_async(DevFrame* f, uint8_t* dst, std::string* err) {
  size_t bps = f->bps();
  size_t off = 0;
  for (int p = 0; p < 3; ++p) {
    size_t w = p ? (f->width + f->ss_x) >> f->ss_x : f->width;
    size_t h = p ? (f->height + f->ss_y) >> f->ss_y : f->height;
    CK(cudaMemcpy2DAsync(dst + off, w * bps, f->planes[p], (size_t)f->stride[p] * bps, w * bps, h,
                         cudaMemcpyDeviceToHost, stream_));
    off += w * h * bps;
  }
  return rv9::ST_OK;
}

rv9::Status Engine::download(DevFrame* f, uint8_t* dst, std::string* err) {
  rv9::Status st = download_async(f, dst, err);
  if (st != rv9::ST_OK) return st;
  return sync(err);
}

rv9::Status Engine::sync(std::string* err) {
  CK(cudaStreamSynchronize(stream_));
  return rv9::ST_OK;
}

}  // namespace rv9g

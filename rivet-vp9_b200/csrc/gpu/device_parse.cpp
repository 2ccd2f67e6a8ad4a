// The device parser's batches: host planning, uploads, launches and the
// read-back of each frame's outcome.
#include "device_parse.h"

#include <string.h>

#include <algorithm>

#include "parse_plan.h"

namespace rv9g {

namespace {

constexpr size_t kAlign = 256;
inline uint64_t align_up(uint64_t x) { return (x + kAlign - 1) & ~(uint64_t)(kAlign - 1); }

#define DP_CK(x)                                              \
  do {                                                        \
    cudaError_t e_ = (x);                                     \
    if (e_ != cudaSuccess) {                                  \
      *err = std::string("device parser: ") + cudaGetErrorString(e_); \
      return rv9::ST_DEVICE;                                  \
    }                                                         \
  } while (0)

}  // namespace

DeviceParser::~DeviceParser() {
  void* dev[] = {d_data_, d_fin_, d_chains_, d_spans_, d_outs_, d_mi_, d_above_, d_prev_, d_blocks_, d_toks_,
                 d_coefs_, d_stage_[0], d_stage_[1], d_scratch_, d_build_, d_results_, d_last_prev_};
  for (void* p : dev)
    if (p) cudaFree(p);
  for (cudaEvent_t e : stage_free_)
    if (e) cudaEventDestroy(e);
  if (collected_) cudaEventDestroy(collected_);
  if (h_pinned_) cudaFreeHost(h_pinned_);
}

rv9::Status DeviceParser::init(int device, std::string* err) {
  device_ = device;
  DP_CK(parse_tables(device, &T_));
  for (cudaEvent_t& e : stage_free_)
    if (!e) DP_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  if (!collected_) DP_CK(cudaEventCreateWithFlags(&collected_, cudaEventDisableTiming | cudaEventBlockingSync));
  return rv9::ST_OK;
}

void DeviceParser::clear() {
  fin_.clear();
  chains_.clear();
  spans_.clear();
  data_.clear();
  fi_.clear();
  build_.clear();
  outs_.clear();
  frames_.clear();
  prev_host_.clear();
  n_mi_ = n_above_ = n_prev_ = n_blocks_ = n_toks_ = n_coefs_ = stage_used_ = scratch_used_ = 0;
  last_frame_ = -1;
}

bool DeviceParser::add(const rv9::Parser::ExternalTiles& x, const rv9_frame_desc& desc) {
  const uint32_t fi = (uint32_t)frames_.size();
  const size_t s0 = spans_.size(), c0 = chains_.size();
  const uint64_t data_off = data_.size();
  if (tp::plan_frame(*x.h, x.tiles, x.tiles_len, data_off, fi, &spans_, &chains_)) {
    spans_.resize(s0);
    chains_.resize(c0);
    return false;
  }
  const uint32_t mi_len = x.h->mi_rows * x.h->mi_cols;
  FrameInfo info;
  memset(&info, 0, sizeof info);
  info.first_chain = (uint32_t)c0;
  info.n_chains = (uint32_t)(chains_.size() - c0);
  info.prev_from = -1;
  info.mi_at = n_mi_;
  n_mi_ += mi_len;
  const uint64_t above_at = n_above_;
  n_above_ += align_up(tp::above_bytes(x.h->sb64_cols));
  // The previous frame is the batch's last one when the batch has frames (a
  // frame parsed on the host ends a batch, and frames begun while a batch
  // is open see the state from before it); else the state's: held by this
  // parser from an earlier batch, or by the host parser, or none.
  bool use_prev = x.use_prev;
  if (use_prev) {
    info.prev_at = n_prev_;
    n_prev_ += mi_len;
    if (last_frame_ >= 0) {
      info.prev_from = last_frame_;
      info.wave = fi_[last_frame_].wave + 1;
    } else if (x.prev_external) {
      if (!have_last_ || last_mi_len_ != mi_len) {
        n_prev_ -= mi_len;
        n_mi_ -= mi_len;
        n_above_ = above_at;
        spans_.resize(s0);
        chains_.resize(c0);
        return false;
      }
      info.prev_from = -2;  // the last device-parsed frame of an earlier batch
    } else if (x.prev_host) {
      info.prev_host = true;
      info.prev_host_at = prev_host_.size();
      const uint8_t* p = (const uint8_t*)x.prev_host;
      prev_host_.insert(prev_host_.end(), p, p + (size_t)mi_len * sizeof(tp::PrevMv));
    } else {
      use_prev = false;  // the host parser's rule: no vectors of this size held
      n_prev_ -= mi_len;
      info.prev_at = 0;
    }
  }
  data_.insert(data_.end(), x.tiles, x.tiles + x.tiles_len);
  BuildFrame bf;
  memset(&bf, 0, sizeof bf);
  bf.first_chain = info.first_chain;
  bf.n_chains = info.n_chains;
  bf.mi_cols = x.h->mi_cols;
  bf.mi_rows = x.h->mi_rows;
  bf.sb64_cols = x.h->sb64_cols;
  bf.sb64_rows = x.h->sb64_rows;
  bf.ss_x = desc.ss_x;
  bf.ss_y = desc.ss_y;
  bf.bit_depth = desc.bit_depth;
  bf.legacy_uv = desc.legacy_uv;
  bf.lf_on = desc.lf_level != 0;
  uint64_t cap_coefs = 0;
  for (size_t c = c0; c < chains_.size(); ++c) {
    tp::Chain& ch = chains_[c];
    ch.mi_at = info.mi_at;
    ch.above_at = above_at;
    ch.prev_at = info.prev_at;
    ch.blocks_at = n_blocks_;
    ch.toks_at = n_toks_;
    ch.coefs_at = n_coefs_;
    n_blocks_ += ch.blocks_cap;
    n_toks_ += ch.toks_cap;
    n_coefs_ += ch.coefs_cap;
    bf.cap_blocks += ch.blocks_cap;
    bf.cap_items += ch.toks_cap;
    cap_coefs += ch.coefs_cap;
  }
  bf.o_blocks = 0;
  bf.o_toks = align_up((uint64_t)bf.cap_blocks * sizeof(rv9_block));
  bf.o_coefs = bf.o_toks + align_up((uint64_t)bf.cap_items * sizeof(rv9_tok));
  bf.o_units = bf.o_coefs + align_up(cap_coefs * 4);
  bf.o_res = bf.o_units + align_up((uint64_t)bf.cap_items * sizeof(InterUnit));
  bf.o_intra = bf.o_res + align_up((uint64_t)bf.cap_items * sizeof(ResItem));
  bf.o_jobs = bf.o_intra + align_up((uint64_t)bf.cap_items * sizeof(IntraItem));
  info.bytes = bf.o_jobs + align_up(((uint64_t)bf.cap_items + 1) * 4);
  info.base = stage_used_;
  bf.base = info.base;
  stage_used_ += info.bytes;
  bf.scratch_at = scratch_used_;
  scratch_used_ += (uint64_t)bf.cap_blocks * 8;
  tp::FrameIn f;
  tp::fill_frame_in(x, &f);
  f.use_prev = use_prev;
  fin_.push_back(f);
  fi_.push_back(info);
  build_.push_back(bf);
  frames_.push_back(desc);
  last_frame_ = (int)fi;
  return true;
}

namespace {

// A frame's worst-case sizes in the batch arrays (what add() reserves for
// it), with the most tile columns the frame's width allows (each rounds its
// width up to whole superblocks).
struct FrameCaps {
  uint64_t mi, above, blocks, toks, coefs, stage, chains, spans, data;
};

FrameCaps frame_caps(uint32_t width, uint32_t height, uint32_t ss_x, uint32_t ss_y) {
  FrameCaps c;
  const uint32_t mi_cols = (width + 7) >> 3, mi_rows = (height + 7) >> 3;
  const uint32_t sb_cols = (mi_cols + 7) >> 3;
  uint32_t log2 = 0;
  while ((sb_cols >> (log2 + 1)) >= 4) ++log2;  // tile columns at least 4 superblocks wide
  const uint32_t cols = 1u << log2;
  uint32_t blocks, toks, coefs;
  tp::chain_caps(mi_cols + 8 * cols, mi_rows, ss_x, ss_y, &blocks, &toks, &coefs);
  c.mi = (uint64_t)mi_cols * mi_rows;
  c.above = align_up(tp::above_bytes(sb_cols));
  c.blocks = blocks;
  c.toks = toks;
  c.coefs = coefs;
  c.stage = align_up((uint64_t)blocks * sizeof(rv9_block)) + align_up((uint64_t)toks * sizeof(rv9_tok)) +
            align_up((uint64_t)coefs * 4) + align_up((uint64_t)toks * sizeof(InterUnit)) +
            align_up((uint64_t)toks * sizeof(ResItem)) + align_up((uint64_t)toks * sizeof(IntraItem)) +
            align_up(((uint64_t)toks + 1) * 4);
  c.chains = cols;
  c.spans = 4ull * cols;  // up to four tile rows
  c.data = (uint64_t)width * height / 2 + (64 << 10);
  return c;
}

}  // namespace

uint64_t DeviceParser::footprint(uint32_t width, uint32_t height, uint32_t ss_x, uint32_t ss_y, uint32_t frames,
                                 int stage_buffers) {
  const FrameCaps c = frame_caps(width, height, ss_x, ss_y);
  const uint64_t records = c.blocks * sizeof(rv9_block) + c.toks * sizeof(rv9_tok) + c.coefs * 4;
  const uint64_t per_frame = (uint64_t)stage_buffers * c.stage + records + c.mi * (sizeof(tp::Mi) + sizeof(tp::PrevMv)) + c.above +
                             c.blocks * 32 + c.data;
  return per_frame * frames + c.mi * sizeof(tp::PrevMv);
}

rv9::Status DeviceParser::reserve(uint32_t width, uint32_t height, uint32_t ss_x, uint32_t ss_y, uint32_t frames,
                                  std::string* err) {
  const FrameCaps c = frame_caps(width, height, ss_x, ss_y);
  const uint64_t n = frames;
  rv9::Status st;
#define DP_RESERVE(p, cap, need) \
  if ((st = grow(&p, &cap, (size_t)(need), err)) != rv9::ST_OK) return st
  DP_RESERVE(d_data_, data_cap_, n * c.data + 16);
  DP_RESERVE(d_fin_, fin_cap_, n);
  DP_RESERVE(d_chains_, chains_cap_, n * c.chains);
  DP_RESERVE(d_spans_, spans_cap_, n * c.spans);
  DP_RESERVE(d_outs_, outs_cap_, n * c.chains);
  DP_RESERVE(d_mi_, mi_cap_, n * c.mi);
  DP_RESERVE(d_above_, above_cap_, n * c.above);
  DP_RESERVE(d_prev_, prev_cap_, n * c.mi);
  DP_RESERVE(d_blocks_, blocks_cap_, n * c.blocks);
  DP_RESERVE(d_toks_, toks_cap_, n * c.toks);
  DP_RESERVE(d_coefs_, coefs_cap_, n * c.coefs);
  for (int b = 0; b < (single_stage_ ? 1 : 2); ++b) {
    if (stage_pending_[b] && n * c.stage > stage_cap_[b]) {
      DP_CK(cudaEventSynchronize(stage_free_[b]));
      stage_pending_[b] = false;
    }
    DP_RESERVE(d_stage_[b], stage_cap_[b], n * c.stage);
  }
  DP_RESERVE(d_scratch_, scratch_cap_, n * c.blocks * 8);
  DP_RESERVE(d_build_, build_cap_, n);
  DP_RESERVE(d_results_, results_cap_, n);
  DP_RESERVE(d_last_prev_, last_prev_cap_, c.mi);
#undef DP_RESERVE
  const size_t pinned = align_up(n * sizeof(tp::FrameIn)) + align_up(n * c.chains * sizeof(tp::Chain)) +
                        align_up(n * c.spans * sizeof(tp::Span)) + align_up(n * sizeof(BuildFrame)) +
                        align_up(c.mi * sizeof(tp::PrevMv)) + n * c.data;
  if (pinned > pinned_cap_) {
    if (h_pinned_) cudaFreeHost(h_pinned_);
    h_pinned_ = nullptr;
    pinned_cap_ = 0;
    DP_CK(cudaMallocHost(&h_pinned_, pinned));
    pinned_cap_ = pinned;
  }
  return rv9::ST_OK;
}

template <class T>
rv9::Status DeviceParser::grow(T** p, size_t* cap, size_t need, std::string* err) {
  if (need <= *cap) return rv9::ST_OK;
  const size_t n = std::max(need, *cap + *cap / 2);
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  DP_CK(cudaMalloc((void**)p, n * sizeof(T)));
  *cap = n;
  return rv9::ST_OK;
}

rv9::Status DeviceParser::launch(cudaStream_t s, std::string* err) {
  const size_t nf = frames_.size(), nc = chains_.size();
  if (nf == 0) return rv9::ST_OK;
  rv9::Status st;
#define DP_GROW(p, cap, need) \
  if ((st = grow(&p, &cap, (size_t)(need), err)) != rv9::ST_OK) return st
  DP_GROW(d_data_, data_cap_, data_.size() + 16);
  DP_GROW(d_fin_, fin_cap_, nf);
  DP_GROW(d_chains_, chains_cap_, nc);
  DP_GROW(d_spans_, spans_cap_, spans_.size());
  DP_GROW(d_outs_, outs_cap_, nc);
  DP_GROW(d_mi_, mi_cap_, n_mi_);
  DP_GROW(d_above_, above_cap_, n_above_);
  DP_GROW(d_prev_, prev_cap_, std::max<uint64_t>(n_prev_, 1));
  DP_GROW(d_blocks_, blocks_cap_, n_blocks_);
  DP_GROW(d_toks_, toks_cap_, n_toks_);
  DP_GROW(d_coefs_, coefs_cap_, n_coefs_);
  if (stage_pending_[cur_] && stage_used_ > stage_cap_[cur_]) {
    // The buffer is replaced: the reconstruction still reading it ends first.
    DP_CK(cudaEventSynchronize(stage_free_[cur_]));
    stage_pending_[cur_] = false;
  }
  DP_GROW(d_stage_[cur_], stage_cap_[cur_], stage_used_);
  DP_GROW(d_scratch_, scratch_cap_, scratch_used_);
  DP_GROW(d_build_, build_cap_, nf);
  DP_GROW(d_results_, results_cap_, nf);
#undef DP_GROW
  // Inputs: one pinned buffer, then one copy per array.
  const size_t o_fin = 0, o_ch = align_up(o_fin + nf * sizeof(tp::FrameIn));
  const size_t o_sp = align_up(o_ch + nc * sizeof(tp::Chain));
  const size_t o_bf = align_up(o_sp + spans_.size() * sizeof(tp::Span));
  const size_t o_pv = align_up(o_bf + nf * sizeof(BuildFrame));
  const size_t o_dt = align_up(o_pv + prev_host_.size());
  const size_t total = o_dt + data_.size();
  if (total > pinned_cap_) {
    if (h_pinned_) cudaFreeHost(h_pinned_);
    h_pinned_ = nullptr;
    pinned_cap_ = 0;
    const size_t cap = std::max(total, pinned_cap_ * 3 / 2);
    DP_CK(cudaMallocHost(&h_pinned_, cap));
    pinned_cap_ = cap;
  }
  memcpy(h_pinned_ + o_fin, fin_.data(), nf * sizeof(tp::FrameIn));
  memcpy(h_pinned_ + o_ch, chains_.data(), nc * sizeof(tp::Chain));
  memcpy(h_pinned_ + o_sp, spans_.data(), spans_.size() * sizeof(tp::Span));
  memcpy(h_pinned_ + o_bf, build_.data(), nf * sizeof(BuildFrame));
  if (!prev_host_.empty()) memcpy(h_pinned_ + o_pv, prev_host_.data(), prev_host_.size());
  memcpy(h_pinned_ + o_dt, data_.data(), data_.size());
  DP_CK(cudaMemcpyAsync(d_fin_, h_pinned_ + o_fin, nf * sizeof(tp::FrameIn), cudaMemcpyHostToDevice, s));
  DP_CK(cudaMemcpyAsync(d_chains_, h_pinned_ + o_ch, nc * sizeof(tp::Chain), cudaMemcpyHostToDevice, s));
  DP_CK(cudaMemcpyAsync(d_spans_, h_pinned_ + o_sp, spans_.size() * sizeof(tp::Span), cudaMemcpyHostToDevice, s));
  DP_CK(cudaMemcpyAsync(d_build_, h_pinned_ + o_bf, nf * sizeof(BuildFrame), cudaMemcpyHostToDevice, s));
  DP_CK(cudaMemcpyAsync(d_data_, h_pinned_ + o_dt, data_.size(), cudaMemcpyHostToDevice, s));
  DP_CK(cudaMemsetAsync(d_above_, 0, n_above_, s));
  // Previous motion vectors: from the host, or from the last device-parsed
  // frame of an earlier batch.
  for (size_t i = 0; i < nf; ++i) {
    const FrameInfo& fi = fi_[i];
    const size_t bytes = (size_t)frames_[i].mi_rows * frames_[i].mi_cols * sizeof(tp::PrevMv);
    if (fi.prev_host)
      DP_CK(cudaMemcpyAsync(d_prev_ + fi.prev_at, h_pinned_ + o_pv + fi.prev_host_at, bytes, cudaMemcpyHostToDevice, s));
    else if (fi.prev_from == -2)
      DP_CK(cudaMemcpyAsync(d_prev_ + fi.prev_at, d_last_prev_, bytes, cudaMemcpyDeviceToDevice, s));
  }
  // The tile columns: all frames at once, or in waves where a frame takes
  // the previous vectors from a frame of this batch.
  int max_wave = 0;
  for (const FrameInfo& fi : fi_) max_wave = std::max(max_wave, fi.wave);
  if (max_wave == 0) {
    DP_CK(launch_parse_chains(T_, d_fin_, d_chains_, 0, (uint32_t)nc, d_spans_, d_data_, d_mi_, d_above_, d_prev_,
                              d_blocks_, d_toks_, d_coefs_, d_outs_, s));
  } else {
    for (int w = 0; w <= max_wave; ++w) {
      if (w > 0) {  // the wave before, waited for on the host (see below)
        DP_CK(cudaEventRecord(collected_, s));
        DP_CK(cudaEventSynchronize(collected_));
      }
      for (size_t i = 0; i < nf; ++i) {
        const FrameInfo& fi = fi_[i];
        if (fi.wave != w) continue;
        if (fi.prev_from >= 0)
          DP_CK(launch_mi_to_prev(d_mi_ + fi_[fi.prev_from].mi_at, d_prev_ + fi.prev_at,
                                  frames_[i].mi_rows * frames_[i].mi_cols, s));
        DP_CK(launch_parse_chains(T_, d_fin_, d_chains_, fi.first_chain, fi.n_chains, d_spans_, d_data_, d_mi_,
                                  d_above_, d_prev_, d_blocks_, d_toks_, d_coefs_, d_outs_, s));
      }
    }
  }
  // The parse runs for up to hundreds of milliseconds. Nothing queued on
  // `s` waits for it inside the device's queue: the host waits (asleep) for
  // it before queuing the build. A CUDA stream whose work sits behind a
  // long kernel's dependant in a hardware queue that another stream shares
  // (the device has a fixed number of them) holds that stream up too.
  DP_CK(cudaEventRecord(collected_, s));
  DP_CK(cudaEventSynchronize(collected_));
  if (stage_pending_[cur_]) {
    DP_CK(cudaStreamWaitEvent(s, stage_free_[cur_], 0));
    stage_pending_[cur_] = false;
  }
  DP_CK(launch_build_frames(d_build_, (uint32_t)nf, d_chains_, d_outs_, d_blocks_, d_toks_, d_coefs_,
                            d_stage_[cur_], d_scratch_, d_results_, s));
  return rv9::ST_OK;
}

rv9::Status DeviceParser::collect(cudaStream_t s, std::string* err) {
  const size_t nf = frames_.size();
  outs_.assign(nf, BuildOut());
  if (nf == 0) return rv9::ST_OK;
  DP_CK(cudaMemcpyAsync(outs_.data(), d_results_, nf * sizeof(BuildOut), cudaMemcpyDeviceToHost, s));
  DP_CK(cudaEventRecord(collected_, s));
  DP_CK(cudaEventSynchronize(collected_));
  // The motion vectors a later batch (or the host parser) may read: those of
  // the last frame before the first that failed.
  int last_ok = -1;
  for (size_t i = 0; i < nf; ++i) {
    bools_ += outs_[i].bools;
    if (outs_[i].err) break;
    last_ok = (int)i;
  }
  if (last_ok >= 0) {
    const uint32_t mi_len = frames_[last_ok].mi_rows * frames_[last_ok].mi_cols;
    rv9::Status st = grow(&d_last_prev_, &last_prev_cap_, mi_len, err);
    if (st != rv9::ST_OK) return st;
    DP_CK(launch_mi_to_prev(d_mi_ + fi_[last_ok].mi_at, d_last_prev_, mi_len, s));
    have_last_ = true;
    last_mi_len_ = mi_len;
  }
  return rv9::ST_OK;
}

rv9::Status DeviceParser::wait_on(cudaStream_t s, std::string* err) {
  DP_CK(cudaEventRecord(collected_, s));
  DP_CK(cudaEventSynchronize(collected_));
  return rv9::ST_OK;
}

rv9::Status DeviceParser::frame_status(size_t i, std::string* msg) const {
  const BuildOut& o = outs_[i];
  if (!o.err) return rv9::ST_OK;
  *msg = tp::error_message(o.err);
  return o.err == tp::TP_OVERFLOW ? rv9::ST_DEVICE : rv9::ST_BITSTREAM;
}

void DeviceParser::frame_work(size_t i, FrameWork* fw) const {
  const BuildOut& o = outs_[i];
  const BuildFrame& b = build_[i];
  fw->n_blocks = o.n_blocks;
  fw->n_toks = o.n_toks;
  fw->n_coefs = o.n_coefs;
  fw->n_units = o.n_units;
  fw->n_units_small = o.n_units_small;
  fw->n_res = o.n_res;
  fw->n_intra = o.n_intra;
  fw->n_intra_jobs = o.n_intra_jobs;
  for (int z = 0; z < 4; ++z) fw->n_res_by_size[z] = o.n_res_by_size[z];
  fw->o_blocks = b.o_blocks;
  fw->o_toks = b.o_toks;
  fw->o_coefs = b.o_coefs;
  fw->o_units = b.o_units;
  fw->o_res = b.o_res;
  fw->o_intra = b.o_intra;
  fw->o_intra_jobs = b.o_jobs;
  fw->bytes = fi_[i].bytes;
  for (int k = 0; k < K_COUNT; ++k) fw->kbytes[k] = o.kbytes[k];
  fw->total_bytes = o.total_bytes;
}

rv9::Status DeviceParser::last_prev(std::vector<tp::PrevMv>* out, cudaStream_t s, std::string* err) {
  if (!have_last_) {
    *err = "device parser: no motion vectors held";
    return rv9::ST_INVALID_INPUT;
  }
  out->resize(last_mi_len_);
  DP_CK(cudaMemcpyAsync(out->data(), d_last_prev_, (size_t)last_mi_len_ * sizeof(tp::PrevMv),
                        cudaMemcpyDeviceToHost, s));
  DP_CK(cudaStreamSynchronize(s));
  return rv9::ST_OK;
}

rv9::Status DeviceParser::recon_queued(cudaStream_t s, std::string* err) {
  DP_CK(cudaEventRecord(stage_free_[cur_], s));
  stage_pending_[cur_] = true;
  if (!single_stage_) cur_ ^= 1;
  return rv9::ST_OK;
}

uint8_t* DeviceParser::release_stage() {
  uint8_t* p = d_stage_[cur_];
  d_stage_[cur_] = nullptr;
  stage_cap_[cur_] = 0;
  stage_pending_[cur_] = false;
  return p;
}

}  // namespace rv9g

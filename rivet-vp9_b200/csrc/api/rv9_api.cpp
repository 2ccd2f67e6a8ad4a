// The C ABI of rv9.h: the reference decoder API (src/decoder/mod.rs:150-216)
// over the host parser and the CUDA reconstruction engine.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/rv9.h"
#include "../gpu/device_parse.h"
#include "../gpu/engine.h"
#include "api_internal.h"
#include "../host/parser.h"

struct rv9_decoder {
  rv9::Parser parser;
  rv9g::Engine engine;
  std::string err;
  rv9::ParsedFrame pf;
  double parse_ms = 0;
  uint32_t parse_depth = 0;  // frames parsed at once; 0: one per two host threads
  uint32_t threads = 0;      // set_threads value; 0: one per core
  // Device parsing (rv9_decoder_set_device_parse).
  bool device_parse = false;
  bool dp_shared = false;  // RV9_DEVICE_PARSE_SHARED
  double dp_share = 0.25;  // the device's part of a shared batch, as last balanced
  uint32_t dp_window = 64;
  std::unique_ptr<rv9g::DeviceParser> dp;
  cudaStream_t dp_stream = nullptr;
  cudaEvent_t dp_ev[2] = {nullptr, nullptr};
  uint64_t dp_frames = 0;
  double dp_ms = 0;
  ~rv9_decoder() {
    dp.reset();
    for (cudaEvent_t e : dp_ev)
      if (e) cudaEventDestroy(e);
    if (dp_stream) cudaStreamDestroy(dp_stream);
  }
};

// Frames parsed at once by the multi-packet calls.
static int parse_depth(const rv9_decoder* d) {
  if (d->parse_depth) return (int)d->parse_depth;
  int hw = (int)std::thread::hardware_concurrency();
  return std::max(1, std::min(8, hw / 2));
}

static thread_local std::string g_global_err;

namespace rv9api {
void set_global_error(const std::string& msg) { g_global_err = msg; }
bool host_isa_ok() {
  __builtin_cpu_init();
  if (__builtin_cpu_supports("x86-64-v3")) return true;
  g_global_err = "the host parser is built for x86-64-v3 (AVX2, BMI2, LZCNT), which this CPU lacks";
  return false;
}
}  // namespace rv9api

static void fill_meta(const rv9g::DevFrame* f, rv9_frame* out) {
  out->width = f->width;
  out->height = f->height;
  out->bit_depth = f->bit_depth;
  out->chroma = f->ss_x ? (f->ss_y ? RV9_YUV420 : RV9_YUV422) : (f->ss_y ? RV9_YUV440 : RV9_YUV444);
  out->color_space = f->color_space;
  out->full_range = f->color_range;
  out->render_width = f->render_w;
  out->render_height = f->render_h;
  size_t bps = f->bps(), off = 0;
  for (int p = 0; p < 3; ++p) {
    uint32_t w = p ? (f->width + f->ss_x) >> f->ss_x : f->width;
    uint32_t h = p ? (f->height + f->ss_y) >> f->ss_y : f->height;
    out->planes[p].offset = off;
    out->planes[p].width = w;
    out->planes[p].height = h;
    off += (size_t)w * h * bps;
  }
  out->size = off;
}

extern "C" {

rv9_decoder* rv9_decoder_new(int device) {
  if (!rv9api::host_isa_ok()) return nullptr;
  rv9_decoder* d = new rv9_decoder;
  std::string err;
  if (!d->engine.init(device, &err)) {
    g_global_err = err;
    delete d;
    return nullptr;
  }
  return d;
}

void rv9_decoder_free(rv9_decoder* d) { delete d; }

rv9_status rv9_decoder_set_device_parse(rv9_decoder* d, int on, uint32_t window_frames) {
  if (!d) return RV9_INVALID_INPUT;
  d->dp_window = window_frames ? window_frames : 64;
  d->device_parse = on != 0;
  d->dp_shared = on == RV9_DEVICE_PARSE_SHARED;
  if (!on || d->dp) return RV9_OK;
  cudaError_t e = cudaSetDevice(d->engine.device());
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&d->dp_stream, cudaStreamNonBlocking);
  for (int i = 0; e == cudaSuccess && i < 2; ++i) e = cudaEventCreate(&d->dp_ev[i]);
  if (e != cudaSuccess) {
    d->err = std::string("device parser: ") + cudaGetErrorString(e);
    d->device_parse = false;
    return RV9_DEVICE;
  }
  std::unique_ptr<rv9g::DeviceParser> p(new rv9g::DeviceParser);
  rv9::Status st = p->init(d->engine.device(), &d->err);
  if (st != rv9::ST_OK) {
    d->device_parse = false;
    return (rv9_status)st;
  }
  d->dp = std::move(p);
  return RV9_OK;
}

void rv9_decoder_device_parse_stats(const rv9_decoder* d, uint64_t* frames, uint64_t* bools, double* device_ms) {
  if (frames) *frames = d ? d->dp_frames : 0;
  if (bools) *bools = d && d->dp ? d->dp->bools() : 0;
  if (device_ms) *device_ms = d ? d->dp_ms : 0;
}
void rv9_decoder_set_threads(rv9_decoder* d, uint32_t t) {
  d->threads = t;
  d->parser.set_threads((int)t);
}
void rv9_decoder_set_parse_depth(rv9_decoder* d, uint32_t frames) { d->parse_depth = frames; }
void rv9_decoder_set_max_pixels(rv9_decoder* d, uint64_t p) { d->parser.set_max_pixels(p); }
uint32_t rv9_decoder_threads(const rv9_decoder* d) {
  if (!d) return 0;
  if (d->threads) return d->threads;
  return std::max(1u, std::thread::hardware_concurrency());
}
void rv9_decoder_set_wait_limit(rv9_decoder* d, uint32_t polls) {
  if (d) d->engine.set_wait_limit(polls);
}
void rv9_decoder_set_test_fault(rv9_decoder* d, uint32_t mask) {
  if (d) d->engine.set_test_skip(mask);
}
uint64_t rv9_decoder_frames_decoded(const rv9_decoder* d) { return d->parser.frames_decoded(); }
const char* rv9_last_error(const rv9_decoder* d) { return d->err.c_str(); }
const char* rv9_last_global_error(void) { return g_global_err.c_str(); }

// One frame of a packet: parse, reconstruct; the shown frame (if any).
static rv9_status decode_one(rv9_decoder* d, const uint8_t* data, size_t len, rv9g::DevFrame** shown) {
  auto t0 = std::chrono::steady_clock::now();
  rv9::Status st = d->parser.parse_frame(data, len, &d->pf, &d->err);
  d->parse_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (st != rv9::ST_OK) return (rv9_status)st;
  st = d->engine.recon(d->pf, shown, &d->err);
  return (rv9_status)st;
}

rv9_status rv9_decode_all(rv9_decoder* d, const uint8_t* pkt, size_t len, rv9_frame* out, size_t cap,
                          size_t* n_out) {
  *n_out = 0;
  if (!d || (!pkt && len)) return RV9_INVALID_INPUT;
  std::vector<std::pair<size_t, size_t>> frames;
  rv9::superframe_split(pkt, len, &frames);
  for (auto& fr : frames) {
    rv9g::DevFrame* shown = nullptr;
    rv9_status st = decode_one(d, pkt + fr.first, fr.second, &shown);
    if (st != RV9_OK) return st;
    if (shown) {
      if (*n_out < cap) {
        rv9_frame* o = &out[*n_out];
        fill_meta(shown, o);
        o->data = (uint8_t*)malloc(o->size ? o->size : 1);
        rv9::Status s2 = d->engine.download_async(shown, o->data, &d->err);
        if (s2 == rv9::ST_OK) s2 = d->engine.sync(&d->err);
        if (s2 != rv9::ST_OK) return (rv9_status)s2;
      }
      ++*n_out;
    }
  }
  return RV9_OK;
}

rv9_status rv9_decode(rv9_decoder* d, const uint8_t* pkt, size_t len, rv9_frame* out, int* shown) {
  *shown = 0;
  std::vector<rv9_frame> frames(8);
  size_t n = 0;
  rv9_status st = rv9_decode_all(d, pkt, len, frames.data(), frames.size(), &n);
  if (st != RV9_OK) return st;
  size_t kept = n < frames.size() ? n : frames.size();
  for (size_t i = 0; i + 1 < kept; ++i) rv9_frame_release(&frames[i]);
  if (kept > 0) {
    *out = frames[kept - 1];
    *shown = 1;
  }
  return RV9_OK;
}

void rv9_frame_release(rv9_frame* f) {
  if (!f) return;
  free(f->data);
  f->data = nullptr;
  f->size = 0;
}

// rv9_decode_packets with device parsing: frames in decode order; those
// the device parser may take gather into a batch (up to the window), the
// others parse on the host once the batch before them is reconstructed. A
// batch parses and builds its work lists on the parser's stream while the
// frames of the batch before it reconstruct on the engine's.
static rv9_status decode_packets_device(rv9_decoder* d, const uint8_t* const* pkts, const size_t* lens, size_t n,
                                        uint8_t* out, size_t cap, size_t* n_frames, size_t* bytes) {
  rv9g::DeviceParser& P = *d->dp;
  P.clear();
  std::vector<rv9::Parser::Job*> pending;
  // After an error in a launched batch: the jobs not finished are dropped,
  // and the batch's stage buffer is handed back behind the reconstructions
  // already queued from it.
  auto release_pending = [&](size_t from) {
    for (size_t i = from; i < pending.size(); ++i) d->parser.release(pending[i]);
    pending.clear();
    std::string ignored;
    P.recon_queued(d->engine.stream(), &ignored);
    P.clear();
  };
  auto show = [&](rv9g::DevFrame* shown) -> rv9_status {
    if (!shown) return RV9_OK;
    size_t nb = rv9g::Engine::packed_bytes(shown);
    if (*bytes + nb > cap) {
      d->err = "output buffer too small";
      return RV9_INVALID_INPUT;
    }
    rv9::Status s2 = d->engine.download_async(shown, out + *bytes, &d->err);
    if (s2 != rv9::ST_OK) return (rv9_status)s2;
    *bytes += nb;
    ++*n_frames;
    return RV9_OK;
  };
  // A shared batch: pending[0, h) parse on the host, frame-parallel on its
  // threads, while pending[h, n) parse on the device (a thread of its own
  // waits for them); then both parts reconstruct in order. Only for frames
  // that depend on nothing earlier frames decide at finish, so that every
  // one may parse before those before it finish.
  auto flush_shared = [&]() -> rv9_status {
    const size_t n = pending.size();
    size_t n_dev = (size_t)(d->dp_share * (double)n + 0.5);
    n_dev = std::max<size_t>(1, std::min(n - 1, n_dev));
    const size_t h = n - n_dev;
    P.clear();
    for (size_t i = h; i < n; ++i) {
      rv9::Parser::ExternalTiles x;
      if (!d->parser.external_tiles(pending[i], &x) || !P.add(x, *x.desc)) {
        // Cannot happen for a frame the batch took; kept whole on the host.
        P.clear();
        return RV9_DEVICE;
      }
    }
    const auto t0 = std::chrono::steady_clock::now();
    rv9::Status dst = rv9::ST_OK;
    std::string derr;
    double dev_s = 0;
    const int device = d->engine.device();
    std::thread dev([&]() {
      cudaSetDevice(device);
      cudaEventRecord(d->dp_ev[0], d->dp_stream);
      dst = P.launch(d->dp_stream, &derr);
      if (dst == rv9::ST_OK) dst = P.collect(d->dp_stream, &derr);
      cudaEventRecord(d->dp_ev[1], d->dp_stream);
      dev_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    });
    const size_t depth = (size_t)parse_depth(d);
    size_t started = 0;
    while (started < std::min(depth, h)) d->parser.run_async(pending[started++]);
    rv9_status st = RV9_OK;
    size_t i = 0;
    for (; i < h && st == RV9_OK; ++i) {
      d->parser.wait(pending[i]);
      rv9::Status s2 = d->parser.finish(pending[i], &d->pf, &d->err);
      d->parser.release(pending[i]);
      pending[i] = nullptr;
      rv9g::DevFrame* shown = nullptr;
      if (s2 == rv9::ST_OK) s2 = d->engine.recon(d->pf, &shown, &d->err);
      st = s2 == rv9::ST_OK ? show(shown) : (rv9_status)s2;
      if (started < h) d->parser.run_async(pending[started++]);
    }
    const double host_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    dev.join();
    if (st == RV9_OK && dst != rv9::ST_OK) {
      d->err = derr;
      st = (rv9_status)dst;
    }
    if (st != RV9_OK) {
      release_pending(i);  // the jobs not finished (release joins any still parsing)
      return st;
    }
    float ms = 0;
    if (cudaEventSynchronize(d->dp_ev[1]) == cudaSuccess && cudaEventElapsedTime(&ms, d->dp_ev[0], d->dp_ev[1]) == cudaSuccess)
      d->dp_ms += ms;
    // The next split: the device's part takes about as long whatever its
    // size (its tile columns run side by side), the host's grows with its
    // frames, so the host takes as many as it parses in the device's time.
    if (host_s > 0 && dev_s > 0) {
      const double per_frame = host_s / (double)h;
      const double want = 1.0 - std::min(1.0, dev_s / (per_frame * (double)n));
      d->dp_share = std::max(0.05, std::min(0.95, 0.5 * (d->dp_share + want)));
    }
    for (size_t j = h; j < n; ++j) {
      std::string msg;
      const rv9::Status ts = P.frame_status(j - h, &msg);
      rv9::ParsedFrame meta;
      rv9::Status s2 = d->parser.finish_external(pending[j], ts, msg, &meta, &d->err);
      d->parser.release(pending[j]);
      pending[j] = nullptr;
      if (s2 != rv9::ST_OK) {
        release_pending(j + 1);
        return (rv9_status)s2;
      }
      rv9g::FrameWork fw;
      fw.desc = meta.desc;
      fw.show_existing = false;
      fw.show_frame = meta.show_frame;
      fw.refresh_mask = meta.refresh_mask;
      for (int k = 0; k < 3; ++k) fw.ref_slot[k] = meta.ref_slot[k];
      P.frame_work(j - h, &fw);
      rv9g::DevFrame* shown = nullptr;
      s2 = d->engine.recon_resident(fw, P.frame_base(j - h), &shown, &d->err);
      if (s2 != rv9::ST_OK) {
        release_pending(j + 1);
        return (rv9_status)s2;
      }
      ++d->dp_frames;
      rv9_status s3 = show(shown);
      if (s3 != RV9_OK) {
        release_pending(j + 1);
        return s3;
      }
    }
    pending.clear();
    rv9::Status s4 = P.recon_queued(d->engine.stream(), &d->err);
    P.clear();
    return (rv9_status)s4;
  };
  auto flush = [&]() -> rv9_status {
    if (pending.empty()) return RV9_OK;
    if (d->dp_shared && pending.size() >= 2) {
      bool all = true;
      for (rv9::Parser::Job* j : pending) all = all && d->parser.independent(j);
      if (all) return flush_shared();
    }
    rv9::Status st;
    cudaEventRecord(d->dp_ev[0], d->dp_stream);
    if ((st = P.launch(d->dp_stream, &d->err)) != rv9::ST_OK || (st = P.collect(d->dp_stream, &d->err)) != rv9::ST_OK) {
      release_pending(0);
      return (rv9_status)st;
    }
    cudaEventRecord(d->dp_ev[1], d->dp_stream);
    float ms = 0;
    if (cudaEventSynchronize(d->dp_ev[1]) == cudaSuccess && cudaEventElapsedTime(&ms, d->dp_ev[0], d->dp_ev[1]) == cudaSuccess)
      d->dp_ms += ms;
    for (size_t i = 0; i < pending.size(); ++i) {
      std::string msg;
      const rv9::Status ts = P.frame_status(i, &msg);
      rv9::ParsedFrame meta;
      st = d->parser.finish_external(pending[i], ts, msg, &meta, &d->err);
      d->parser.release(pending[i]);
      pending[i] = nullptr;
      if (st != rv9::ST_OK) {
        release_pending(i + 1);
        return (rv9_status)st;
      }
      rv9g::FrameWork fw;
      fw.desc = meta.desc;
      fw.show_existing = false;
      fw.show_frame = meta.show_frame;
      fw.refresh_mask = meta.refresh_mask;
      for (int k = 0; k < 3; ++k) fw.ref_slot[k] = meta.ref_slot[k];
      P.frame_work(i, &fw);
      rv9g::DevFrame* shown = nullptr;
      st = d->engine.recon_resident(fw, P.frame_base(i), &shown, &d->err);
      if (st != rv9::ST_OK) {
        release_pending(i + 1);
        return (rv9_status)st;
      }
      ++d->dp_frames;
      rv9_status s3 = show(shown);
      if (s3 != RV9_OK) {
        release_pending(i + 1);
        return s3;
      }
    }
    pending.clear();
    st = P.recon_queued(d->engine.stream(), &d->err);
    P.clear();
    return (rv9_status)st;
  };
  std::vector<std::pair<size_t, size_t>> frames;
  for (size_t i = 0; i < n; ++i) {
    rv9::superframe_split(pkts[i], lens[i], &frames);
    for (auto& fr : frames) {
      const uint8_t* data = pkts[i] + fr.first;
      auto t0 = std::chrono::steady_clock::now();
      rv9::Parser::Job* job = d->parser.begin(data, fr.second, nullptr);
      rv9::Parser::ExternalTiles x;
      const bool dev = d->parser.external_tiles(job, &x) && P.add(x, *x.desc);
      d->parse_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      if (dev) {
        pending.push_back(job);
        // A batch ends at the window or at 4 GiB of device records.
        if (pending.size() >= d->dp_window || P.stage_bytes() >= (4ull << 30)) {
          rv9_status st = flush();
          if (st != RV9_OK) return st;
        }
        continue;
      }
      // A frame for the host parser: what came before it first.
      rv9_status st = flush();
      if (st != RV9_OK) {
        d->parser.release(job);
        return st;
      }
      t0 = std::chrono::steady_clock::now();
      d->parser.bind_prev(job);  // frames begun before it have finished now
      if (d->parser.wants_external_prev(job) && P.have_last()) {
        std::vector<rv9g::tp::PrevMv> prev;
        rv9::Status s2 = P.last_prev(&prev, d->dp_stream, &d->err);
        if (s2 != rv9::ST_OK) {
          d->parser.release(job);
          return (rv9_status)s2;
        }
        d->parser.provide_prev_mvs(job, prev.data(), prev.size());
      }
      d->parser.attach_work(job);
      d->parser.run(job);
      rv9::Status s2 = d->parser.finish(job, &d->pf, &d->err);
      d->parser.release(job);
      d->parse_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      if (s2 != rv9::ST_OK) return (rv9_status)s2;
      rv9g::DevFrame* shown = nullptr;
      s2 = d->engine.recon(d->pf, &shown, &d->err);
      if (s2 != rv9::ST_OK) return (rv9_status)s2;
      if ((st = show(shown)) != RV9_OK) return st;
    }
  }
  rv9_status st = flush();
  if (st != RV9_OK) return st;
  return (rv9_status)d->engine.sync(&d->err);
}

rv9_status rv9_decode_packets(rv9_decoder* d, const uint8_t* const* pkts, const size_t* lens, size_t n,
                              uint8_t* out, size_t cap, size_t* n_frames, size_t* bytes) {
  *n_frames = 0;
  *bytes = 0;
  if (!d || (n && (!pkts || !lens))) return RV9_INVALID_INPUT;
  if (d->device_parse && d->dp) return decode_packets_device(d, pkts, lens, n, out, cap, n_frames, bytes);
  // Frames parse `depth` at a time where the stream allows (FramePipeline);
  // each is reconstructed in order as its records come out.
  const int depth = parse_depth(d);
  rv9::FramePipeline pipe(&d->parser, depth);
  std::vector<std::pair<size_t, size_t>> frames;
  rv9::ParsedFrame& pf = d->pf;
  auto consume = [&]() -> rv9_status {
    auto t0 = std::chrono::steady_clock::now();
    rv9::Status st = pipe.pop(&pf, &d->err);
    d->parse_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (st != rv9::ST_OK) return (rv9_status)st;
    rv9g::DevFrame* shown = nullptr;
    st = d->engine.recon(pf, &shown, &d->err);
    if (st != rv9::ST_OK) return (rv9_status)st;
    if (shown) {
      size_t nb = rv9g::Engine::packed_bytes(shown);
      if (*bytes + nb > cap) {
        d->err = "output buffer too small";
        return RV9_INVALID_INPUT;
      }
      rv9::Status s2 = d->engine.download_async(shown, out + *bytes, &d->err);
      if (s2 != rv9::ST_OK) return (rv9_status)s2;
      *bytes += nb;
      ++*n_frames;
    }
    return RV9_OK;
  };
  for (size_t i = 0; i < n; ++i) {
    rv9::superframe_split(pkts[i], lens[i], &frames);
    for (auto& fr : frames) {
      auto t0 = std::chrono::steady_clock::now();
      pipe.push(pkts[i] + fr.first, fr.second);
      d->parse_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      while (pipe.in_flight() >= (size_t)depth) {
        rv9_status st = consume();
        if (st != RV9_OK) return st;
      }
    }
  }
  while (pipe.in_flight() > 0) {
    rv9_status st = consume();
    if (st != RV9_OK) return st;
  }
  return (rv9_status)d->engine.sync(&d->err);
}

struct rv9_sequence {
  rv9g::Sequence seq;
};

// rv9_sequence_load with device parsing, when every frame allows it (a
// fresh parser; *done false and nothing kept otherwise): one batch, whose
// stage buffer becomes the sequence's device data.
static rv9::Status sequence_load_device(rv9_decoder* d, const uint8_t* const* pkts, const size_t* lens, size_t n,
                                        rv9g::Sequence* seq, bool* done) {
  *done = false;
  rv9::Parser parser;
  parser.set_threads(0);
  rv9g::DeviceParser& P = *d->dp;
  P.clear();
  std::vector<rv9::Parser::Job*> jobs;
  auto drop = [&](size_t from) {
    for (size_t i = from; i < jobs.size(); ++i) parser.release(jobs[i]);
    jobs.clear();
    P.clear();
  };
  std::vector<std::pair<size_t, size_t>> split;
  for (size_t i = 0; i < n; ++i) {
    rv9::superframe_split(pkts[i], lens[i], &split);
    for (auto& fr : split) {
      rv9::Parser::Job* job = parser.begin(pkts[i] + fr.first, fr.second, nullptr);
      jobs.push_back(job);
      rv9::Parser::ExternalTiles x;
      if (!parser.external_tiles(job, &x) || !P.add(x, *x.desc)) {
        drop(0);
        return rv9::ST_OK;
      }
    }
  }
  *done = true;
  rv9::Status st;
  cudaEventRecord(d->dp_ev[0], d->dp_stream);
  if ((st = P.launch(d->dp_stream, &d->err)) != rv9::ST_OK || (st = P.collect(d->dp_stream, &d->err)) != rv9::ST_OK) {
    drop(0);
    return st;
  }
  cudaEventRecord(d->dp_ev[1], d->dp_stream);
  float ms = 0;
  if (cudaEventSynchronize(d->dp_ev[1]) == cudaSuccess && cudaEventElapsedTime(&ms, d->dp_ev[0], d->dp_ev[1]) == cudaSuccess)
    d->dp_ms += ms;
  seq->frames.resize(jobs.size());
  seq->luma_samples = 0;
  for (size_t i = 0; i < jobs.size(); ++i) {
    std::string msg;
    const rv9::Status ts = P.frame_status(i, &msg);
    rv9::ParsedFrame meta;
    st = parser.finish_external(jobs[i], ts, msg, &meta, &d->err);
    parser.release(jobs[i]);
    jobs[i] = nullptr;
    if (st != rv9::ST_OK) {
      drop(i + 1);
      return st;
    }
    rv9g::FrameWork& fw = seq->frames[i];
    fw.desc = meta.desc;
    fw.show_existing = false;
    fw.show_frame = meta.show_frame;
    fw.refresh_mask = meta.refresh_mask;
    for (int k = 0; k < 3; ++k) fw.ref_slot[k] = meta.ref_slot[k];
    P.frame_work(i, &fw);
    const uint64_t off = P.frame_offset(i);
    fw.o_blocks += off;
    fw.o_toks += off;
    fw.o_coefs += off;
    fw.o_units += off;
    fw.o_res += off;
    fw.o_intra += off;
    fw.o_intra_jobs += off;
    if (meta.show_frame) seq->luma_samples += (uint64_t)meta.desc.width * meta.desc.height;
    ++d->dp_frames;
  }
  jobs.clear();
  seq->bytes = P.stage_bytes();
  seq->d_data = P.release_stage();
  P.clear();
  return rv9::ST_OK;
}

rv9_status rv9_sequence_load(rv9_decoder* d, const uint8_t* const* pkts, const size_t* lens, size_t n,
                             rv9_sequence** out) {
  *out = nullptr;
  if (d && d->device_parse && d->dp) {
    rv9_sequence* s = new rv9_sequence;
    bool done = false;
    rv9::Status st = sequence_load_device(d, pkts, lens, n, &s->seq, &done);
    if (st != rv9::ST_OK) {
      d->engine.sequence_free(&s->seq);
      delete s;
      return (rv9_status)st;
    }
    if (done) {
      *out = s;
      return RV9_OK;
    }
    delete s;
  }
  rv9::Parser parser;  // a fresh stream
  parser.set_threads(0);
  std::vector<rv9::ParsedFrame> frames;
  std::vector<std::pair<size_t, size_t>> split;
  const int depth = parse_depth(d);
  rv9::FramePipeline pipe(&parser, depth);
  auto take = [&]() -> rv9::Status {
    frames.emplace_back();
    return pipe.pop(&frames.back(), &d->err);
  };
  for (size_t i = 0; i < n; ++i) {
    rv9::superframe_split(pkts[i], lens[i], &split);
    for (auto& fr : split) {
      pipe.push(pkts[i] + fr.first, fr.second);
      while (pipe.in_flight() >= (size_t)depth) {
        rv9::Status st = take();
        if (st != rv9::ST_OK) return (rv9_status)st;
      }
    }
  }
  while (pipe.in_flight() > 0) {
    rv9::Status st = take();
    if (st != rv9::ST_OK) return (rv9_status)st;
  }
  rv9_sequence* s = new rv9_sequence;
  rv9::Status st = d->engine.sequence_load(frames, &s->seq, &d->err);
  if (st != rv9::ST_OK) {
    delete s;
    return (rv9_status)st;
  }
  *out = s;
  return RV9_OK;
}

rv9_status rv9_sequence_clone(rv9_decoder* d, const rv9_sequence* src, rv9_sequence** out) {
  if (!d || !src || !out) return RV9_INVALID_INPUT;
  *out = nullptr;
  rv9_sequence* s = new rv9_sequence;
  rv9::Status st = d->engine.sequence_clone(src->seq, &s->seq, &d->err);
  if (st != rv9::ST_OK) {
    d->engine.sequence_free(&s->seq);
    delete s;
    return (rv9_status)st;
  }
  *out = s;
  return RV9_OK;
}

rv9_status rv9_sequence_run(rv9_decoder* d, rv9_sequence* s, int flags, double* device_ms) {
  float ms = 0;
  rv9::Status st = (flags & RV9_RUN_GRAPH) ? d->engine.sequence_replay(s->seq, &ms, &d->err)
                                           : d->engine.sequence_run(s->seq, (flags & RV9_RUN_PER_KERNEL) != 0, &ms,
                                                                    &d->err);
  *device_ms = ms;
  return (rv9_status)st;
}

rv9_status rv9_sequence_run_noalloc(rv9_decoder* d, rv9_sequence* s, double* device_ms) {
  if (!d || !s || !device_ms) return RV9_INVALID_INPUT;
  float ms = 0;
  rv9::Status st = d->engine.sequence_run_fixed(s->seq, &ms, &d->err);
  *device_ms = ms;
  return (rv9_status)st;
}

rv9_status rv9_sequences_run(rv9_decoder* const* decs, rv9_sequence* const* seqs, size_t n, int flags,
                             double* device_ms) {
  if (!device_ms || (n && (!decs || !seqs))) return RV9_INVALID_INPUT;
  *device_ms = 0;
  std::vector<rv9g::Engine*> engines(n);
  std::vector<const rv9g::Sequence*> ss(n);
  for (size_t i = 0; i < n; ++i) {
    if (!decs[i] || !seqs[i]) return RV9_INVALID_INPUT;
    engines[i] = &decs[i]->engine;
    ss[i] = &seqs[i]->seq;
  }
  float ms = 0;
  std::string err;
  rv9::Status st = rv9g::Engine::run_concurrent(engines.data(), ss.data(), n, (flags & RV9_RUN_PER_KERNEL) != 0, &ms,
                                                &err, (flags & RV9_RUN_GRAPH) != 0);
  if (st != rv9::ST_OK && n) decs[0]->err = err;
  *device_ms = ms;
  return (rv9_status)st;
}

rv9_status rv9_sequences_run_batched(rv9_decoder* const* decs, rv9_sequence* const* seqs, size_t n, int groups,
                                     double* device_ms) {
  if (!device_ms || (n && (!decs || !seqs)) || groups < 1) return RV9_INVALID_INPUT;
  *device_ms = 0;
  std::vector<rv9g::Engine*> engines(n);
  std::vector<const rv9g::Sequence*> ss(n);
  for (size_t i = 0; i < n; ++i) {
    if (!decs[i] || !seqs[i]) return RV9_INVALID_INPUT;
    engines[i] = &decs[i]->engine;
    ss[i] = &seqs[i]->seq;
  }
  float ms = 0;
  std::string err;
  rv9::Status st = rv9g::Engine::run_batched(engines.data(), ss.data(), n, groups, &ms, &err);
  if (st != rv9::ST_OK && n) decs[0]->err = err;
  *device_ms = ms;
  return (rv9_status)st;
}

rv9_status rv9_sequences_autotune_batched(rv9_decoder* const* decs, rv9_sequence* const* seqs, size_t n,
                                          int32_t* groups, rv9_tune_result* out) {
  if (!out || !groups || (n && (!decs || !seqs))) return RV9_INVALID_INPUT;
  std::vector<rv9g::Engine*> engines(n);
  std::vector<const rv9g::Sequence*> ss(n);
  for (size_t i = 0; i < n; ++i) {
    if (!decs[i] || !seqs[i]) return RV9_INVALID_INPUT;
    engines[i] = &decs[i]->engine;
    ss[i] = &seqs[i]->seq;
  }
  rv9g::TuneParams best;
  float best_ms = 0, default_ms = 0;
  int g = 1;
  std::string err;
  rv9::Status st =
      rv9g::Engine::autotune_batched(engines.data(), ss.data(), n, &g, &best, &best_ms, &default_ms, &err);
  if (st != rv9::ST_OK && n) decs[0]->err = err;
  *groups = g;
  out->intra_ctas_per_sm_x4 = best.intra_ctas_per_sm_x4;
  out->inter_threads = best.inter_threads;
  out->best_ms = best_ms;
  out->default_ms = default_ms;
  out->inter_fork = best.inter_fork ? 1 : 0;
  return (rv9_status)st;
}

uint32_t rv9_sequence_frames(const rv9_sequence* s) { return (uint32_t)s->seq.frames.size(); }
uint64_t rv9_sequence_luma_samples(const rv9_sequence* s) { return s->seq.luma_samples; }
uint64_t rv9_sequence_algorithmic_bytes(const rv9_sequence* s) {
  uint64_t b = 0;
  for (const auto& f : s->seq.frames) b += f.total_bytes;
  return b;
}
uint64_t rv9_sequence_record_bytes(const rv9_sequence* s) { return s->seq.bytes; }

void rv9_sequence_free(rv9_decoder* d, rv9_sequence* s) {
  if (!s) return;
  d->engine.sequence_free(&s->seq);
  delete s;
}

rv9_status rv9_decoder_autotune(rv9_decoder* d, rv9_sequence* s, rv9_tune_result* out) {
  if (!d || !s || !out) return RV9_INVALID_INPUT;
  rv9g::TuneParams best;
  float best_ms = 0, default_ms = 0;
  rv9::Status st = d->engine.autotune(s->seq, &best, &best_ms, &default_ms, &d->err);
  out->intra_ctas_per_sm_x4 = best.intra_ctas_per_sm_x4;
  out->inter_threads = best.inter_threads;
  out->best_ms = best_ms;
  out->default_ms = default_ms;
  out->inter_fork = best.inter_fork ? 1 : 0;
  return (rv9_status)st;
}

rv9_status rv9_sequences_autotune(rv9_decoder* const* decs, rv9_sequence* const* seqs, size_t n,
                                  rv9_tune_result* out) {
  if (!out || (n && (!decs || !seqs))) return RV9_INVALID_INPUT;
  std::vector<rv9g::Engine*> engines(n);
  std::vector<const rv9g::Sequence*> ss(n);
  for (size_t i = 0; i < n; ++i) {
    if (!decs[i] || !seqs[i]) return RV9_INVALID_INPUT;
    engines[i] = &decs[i]->engine;
    ss[i] = &seqs[i]->seq;
  }
  rv9g::TuneParams best;
  float best_ms = 0, default_ms = 0;
  std::string err;
  rv9::Status st = rv9g::Engine::autotune_concurrent(engines.data(), ss.data(), n, &best, &best_ms, &default_ms, &err);
  if (st != rv9::ST_OK && n) decs[0]->err = err;
  out->intra_ctas_per_sm_x4 = best.intra_ctas_per_sm_x4;
  out->inter_threads = best.inter_threads;
  out->best_ms = best_ms;
  out->default_ms = default_ms;
  out->inter_fork = best.inter_fork ? 1 : 0;
  return (rv9_status)st;
}

rv9_status rv9_decoder_download_slot(rv9_decoder* d, int slot, uint8_t* out, size_t cap, size_t* bytes) {
  *bytes = 0;
  if (slot < 0 || slot > 7 || !d->engine.slot(slot)) return RV9_INVALID_INPUT;
  rv9g::DevFrame* f = d->engine.slot(slot);
  size_t nb = rv9g::Engine::packed_bytes(f);
  if (nb > cap) return RV9_INVALID_INPUT;
  rv9::Status st = d->engine.download_async(f, out, &d->err);
  if (st == rv9::ST_OK) st = d->engine.sync(&d->err);
  *bytes = nb;
  return (rv9_status)st;
}

size_t rv9_kernel_stats(rv9_decoder* d, rv9_kernel_stat* out, size_t cap, int reset) {
  size_t n = 0;
  for (int k = 0; k < rv9g::K_COUNT; ++k) {
    if (n < cap) {
      snprintf(out[n].name, sizeof out[n].name, "%s", rv9g::kKernelNames[k]);
      out[n].launches = d->engine.kstats[k].launches;
      out[n].ms = d->engine.kstats[k].ms;
      out[n].algorithmic_bytes = d->engine.kstats[k].bytes;
    }
    ++n;
    if (reset) d->engine.kstats[k] = rv9g::KernelStat();
  }
  return n;
}

void rv9_decoder_set_event_mask(rv9_decoder* d, uint32_t mask) { d->engine.event_mask = mask; }

void rv9_decoder_set_frame_sink(rv9_decoder* d, uint8_t* buf, size_t cap) {
  if (d) d->engine.set_sink(buf, buf ? cap : 0);
}

rv9_status rv9_decoder_set_frame_digests(rv9_decoder* d, size_t cap_frames) {
  if (!d) return RV9_INVALID_INPUT;
  return (rv9_status)d->engine.set_digests(cap_frames, &d->err);
}

size_t rv9_decoder_frame_digests(rv9_decoder* d, uint8_t* out, size_t cap) {
  if (!d || (!out && cap)) return 0;
  return d->engine.digests(out, cap);
}

void rv9_decoder_frame_sink_state(const rv9_decoder* d, uint64_t* frames, size_t* bytes, uint64_t* dropped) {
  if (frames) *frames = d ? d->engine.sink_frames() : 0;
  if (bytes) *bytes = d ? d->engine.sink_used() : 0;
  if (dropped) *dropped = d ? d->engine.sink_dropped() : 0;
}

void rv9_decoder_stats(rv9_decoder* d, rv9_stats* out, int reset) {
  out->device_ms = d->engine.device_ms;
  out->parse_ms = d->parse_ms;
  out->frames = d->engine.frames;
  out->algorithmic_bytes = d->engine.alg_bytes;
  out->kernel_launches = d->engine.launches;
  if (reset) {
    d->engine.device_ms = 0;
    d->parse_ms = 0;
    d->engine.frames = 0;
    d->engine.alg_bytes = 0;
    d->engine.launches = 0;
  }
}

}  // extern "C"

// Test shim: the frame-parallel parser (FramePipeline) against frame-by-frame
// parsing (Parser::parse_frame) on the same packets. Compares each frame's
// status, flags, frame description and records, byte for byte.
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../rivet-vp9_b200/csrc/host/parser.h"

namespace {

bool same_frame(const rv9::ParsedFrame& a, const rv9::ParsedFrame& b) {
  if (a.show_existing != b.show_existing || a.show_frame != b.show_frame || a.refresh_mask != b.refresh_mask)
    return false;
  if (a.show_existing) return a.show_slot == b.show_slot;
  if (memcmp(a.ref_slot, b.ref_slot, sizeof a.ref_slot) || memcmp(&a.desc, &b.desc, sizeof a.desc)) return false;
  if (a.blocks.size() != b.blocks.size() || a.toks.size() != b.toks.size() || a.coefs.size() != b.coefs.size())
    return false;
  return !memcmp(a.blocks.data(), b.blocks.data(), a.blocks.size() * sizeof(rv9_block)) &&
         !memcmp(a.toks.data(), b.toks.data(), a.toks.size() * sizeof(rv9_tok)) &&
         !memcmp(a.coefs.data(), b.coefs.data(), a.coefs.size() * 4);
}

}  // namespace

extern "C" {

// Parses the packets (superframes split) both ways, with `depth` frames in
// flight and `tile_threads` per frame. After an error, both parsers go on with
// the next packets, the pipeline in a new pipeline (as a caller would), and
// must keep agreeing. Returns the number of frames compared, or -1 with a
// message in `msg`.
int pipeline_check(const uint8_t* const* pkts, const size_t* lens, size_t n, int depth, int tile_threads,
                   char* msg, size_t msg_cap) {
  std::vector<std::pair<const uint8_t*, size_t>> frames;
  std::vector<std::pair<size_t, size_t>> split;
  for (size_t i = 0; i < n; ++i) {
    rv9::superframe_split(pkts[i], lens[i], &split);
    for (auto& f : split) frames.emplace_back(pkts[i] + f.first, f.second);
  }
  rv9::Parser seq, par;
  seq.set_threads(tile_threads);
  par.set_threads(tile_threads);
  // Frame by frame.
  std::vector<rv9::Status> want_st(frames.size());
  std::vector<rv9::ParsedFrame> want(frames.size());
  std::vector<std::string> want_err(frames.size());
  for (size_t i = 0; i < frames.size(); ++i)
    want_st[i] = seq.parse_frame(frames[i].first, frames[i].second, &want[i], &want_err[i]);
  // Pipelined; a new pipeline after each error.
  size_t next = 0, compared = 0;
  while (next < frames.size()) {
    rv9::FramePipeline pipe(&par, depth);
    size_t pushed = next, popped = next;
    bool stop = false;
    while (popped < frames.size() && !stop) {
      while (pushed < frames.size() && pipe.in_flight() < (size_t)depth) {
        pipe.push(frames[pushed].first, frames[pushed].second);
        ++pushed;
      }
      rv9::ParsedFrame got;
      std::string err;
      rv9::Status st = pipe.pop(&got, &err);
      size_t i = popped++;
      if (st != want_st[i]) {
        snprintf(msg, msg_cap, "frame %zu: status %d, frame by frame %d (%s)", i, (int)st, (int)want_st[i],
                 err.c_str());
        return -1;
      }
      if (st == rv9::ST_OK && !same_frame(got, want[i])) {
        snprintf(msg, msg_cap, "frame %zu: records differ", i);
        return -1;
      }
      ++compared;
      if (st != rv9::ST_OK) stop = true;  // the pipeline dropped what follows
    }
    next = popped;
  }
  if (par.frames_decoded() != seq.frames_decoded()) {
    snprintf(msg, msg_cap, "frames_decoded %llu vs %llu", (unsigned long long)par.frames_decoded(),
             (unsigned long long)seq.frames_decoded());
    return -1;
  }
  return (int)compared;
}

}  // extern "C"

extern "C" {

// The shared device-parse batch's host side (rv9_decode_packets with
// RV9_DEVICE_PARSE_SHARED), on the CPU: frames the device parser could take
// (Parser::external_tiles) gather into batches of up to `window`, begun in
// order before any of them finishes; a batch whose frames are all
// independent (Parser::independent) runs them `depth` at a time on threads
// of their own (run_async, wait) and finishes them in order, any other batch
// runs and finishes them one by one (bind_prev first, as the host parser does
// after a device batch); a frame the device parser could not take finishes
// the batch first, then parses alone. Against frame-by-frame parsing.
// Returns the number of frames in independent batches, or -1 with a message.
int shared_batch_check(const uint8_t* const* pkts, const size_t* lens, size_t n, int window, int depth, char* msg,
                       size_t msg_cap) {
  std::vector<std::pair<const uint8_t*, size_t>> frames;
  std::vector<std::pair<size_t, size_t>> split;
  for (size_t i = 0; i < n; ++i) {
    rv9::superframe_split(pkts[i], lens[i], &split);
    for (auto& f : split) frames.emplace_back(pkts[i] + f.first, f.second);
  }
  rv9::Parser seq, par;
  std::vector<rv9::Status> want_st(frames.size());
  std::vector<rv9::ParsedFrame> want(frames.size());
  std::vector<std::string> want_err(frames.size());
  for (size_t i = 0; i < frames.size(); ++i)
    want_st[i] = seq.parse_frame(frames[i].first, frames[i].second, &want[i], &want_err[i]);
  int shared = 0;
  size_t done = 0;
  bool failed = false;
  auto compare = [&](rv9::Status st, const rv9::ParsedFrame& got, const std::string& err) -> bool {
    const size_t i = done++;
    if (st != want_st[i]) {
      snprintf(msg, msg_cap, "frame %zu: status %d, frame by frame %d (%s)", i, (int)st, (int)want_st[i],
               err.c_str());
      return false;
    }
    if (st == rv9::ST_OK && !same_frame(got, want[i])) {
      snprintf(msg, msg_cap, "frame %zu: records differ", i);
      return false;
    }
    if (st != rv9::ST_OK) failed = true;
    return true;
  };
  std::vector<rv9::Parser::Job*> batch;
  auto flush = [&]() -> bool {
    bool all = batch.size() >= 2;
    for (rv9::Parser::Job* j : batch) all = all && par.independent(j);
    bool ok = true;
    if (all) {
      size_t started = 0;
      while (started < std::min<size_t>((size_t)depth, batch.size())) par.run_async(batch[started++]);
      for (size_t i = 0; i < batch.size(); ++i) {
        par.wait(batch[i]);
        rv9::ParsedFrame got;
        std::string err;
        rv9::Status st = par.finish(batch[i], &got, &err);
        par.release(batch[i]);
        batch[i] = nullptr;
        if (started < batch.size()) par.run_async(batch[started++]);
        if (ok && !failed) ok = compare(st, got, err);
        ++shared;
      }
    } else {
      for (size_t i = 0; i < batch.size(); ++i) {
        par.bind_prev(batch[i]);
        par.attach_work(batch[i]);
        par.run(batch[i]);
        rv9::ParsedFrame got;
        std::string err;
        rv9::Status st = par.finish(batch[i], &got, &err);
        par.release(batch[i]);
        if (ok && !failed) ok = compare(st, got, err);
      }
    }
    batch.clear();
    return ok;
  };
  for (size_t i = 0; i < frames.size() && !failed; ++i) {
    rv9::Parser::Job* job = par.begin(frames[i].first, frames[i].second, nullptr);
    rv9::Parser::ExternalTiles x;
    if (par.external_tiles(job, &x)) {
      batch.push_back(job);
      if (batch.size() >= (size_t)window && !flush()) return -1;
      continue;
    }
    if (!flush()) {
      par.release(job);
      return -1;
    }
    par.bind_prev(job);
    par.attach_work(job);
    par.run(job);
    rv9::ParsedFrame got;
    std::string err;
    rv9::Status st = par.finish(job, &got, &err);
    par.release(job);
    if (!failed && !compare(st, got, err)) return -1;
  }
  if (!failed && !flush()) return -1;
  for (rv9::Parser::Job* j : batch) par.release(j);
  return shared;
}

}  // extern "C"

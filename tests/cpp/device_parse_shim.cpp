// Test shim: the device tile parser (rivet-vp9_b200/csrc/gpu/tile_parse.cuh),
// compiled for the CPU, against the host parser on the same packets. Frames
// the device parser may take (Parser::external_tiles) go through it, the
// others through the host parser (given the device-held motion vectors when
// they read them), exactly as the decoder's device-parse mode splits them;
// every frame's status, message and records must equal frame-by-frame host
// parsing, byte for byte.
#include <stdio.h>
#include <string.h>

#include <memory>
#include <string>
#include <vector>

#include "../../rivet-vp9_b200/csrc/gpu/parse_plan.h"

namespace {

using namespace rv9g::tp;

bool same_records(const rv9::ParsedFrame& a, const rv9::ParsedFrame& b, char* why, size_t cap) {
  if (a.show_existing != b.show_existing || a.show_frame != b.show_frame || a.refresh_mask != b.refresh_mask) {
    snprintf(why, cap, "flags differ");
    return false;
  }
  if (a.show_existing) return a.show_slot == b.show_slot;
  if (memcmp(a.ref_slot, b.ref_slot, sizeof a.ref_slot) || memcmp(&a.desc, &b.desc, sizeof a.desc)) {
    snprintf(why, cap, "frame description differs");
    return false;
  }
  if (a.blocks.size() != b.blocks.size() || a.toks.size() != b.toks.size() || a.coefs.size() != b.coefs.size()) {
    snprintf(why, cap, "record counts differ: blocks %zu/%zu toks %zu/%zu coefs %zu/%zu", a.blocks.size(),
             b.blocks.size(), a.toks.size(), b.toks.size(), a.coefs.size(), b.coefs.size());
    return false;
  }
  for (size_t i = 0; i < a.blocks.size(); ++i)
    if (memcmp(&a.blocks[i], &b.blocks[i], sizeof(rv9_block))) {
      snprintf(why, cap, "block %zu differs (mi %u,%u)", i, a.blocks[i].mi_row, a.blocks[i].mi_col);
      return false;
    }
  for (size_t i = 0; i < a.toks.size(); ++i)
    if (memcmp(&a.toks[i], &b.toks[i], sizeof(rv9_tok))) {
      snprintf(why, cap, "transform block %zu differs", i);
      return false;
    }
  if (memcmp(a.coefs.data(), b.coefs.data(), a.coefs.size() * 4)) {
    snprintf(why, cap, "coefficients differ");
    return false;
  }
  return true;
}

// How often each source of previous motion vectors served a frame, since
// the library was loaded: [0] a batch's previous frame, [1] the host
// parser's state, [2] the last device frame of an earlier batch, [3] a host
// frame given device-held vectors.
uint64_t g_prev_counts[4] = {0, 0, 0, 0};

struct DeviceSide {
  Tables tables;
  std::vector<Mi> last_mi;  // the last device-parsed frame's mode info
  uint32_t last_cols = 0, last_rows = 0;
  uint64_t bools = 0;
};

// The device parser's path for one frame, on the CPU: returns the tiles'
// status and fills `out` with the gathered records. prev_mode: where the
// previous frame's vectors come from: 0 none, 1 the host parser
// (x.prev_host), 2 the last device-parsed frame.
rv9::Status device_frame(DeviceSide& D, const rv9::Parser::ExternalTiles& x, int prev_mode, rv9::ParsedFrame* out,
                         std::string* msg, bool* planned) {
  FrameIn fin;
  fill_frame_in(x, &fin);
  fin.use_prev = prev_mode != 0;
  std::vector<Span> spans;
  std::vector<Chain> chains;
  const char* e = plan_frame(*x.h, x.tiles, x.tiles_len, 0, 0, &spans, &chains);
  *planned = e == nullptr;
  if (e) return rv9::ST_OK;
  const size_t mi_len = (size_t)fin.mi_rows * fin.mi_cols;
  std::vector<Mi> mi(mi_len);
  std::vector<uint8_t> above(above_bytes(fin.sb64_cols), 0);
  std::vector<PrevMv> prev;
  if (fin.use_prev) {
    prev.resize(mi_len);
    if (prev_mode == 1) {
      memcpy(prev.data(), x.prev_host, mi_len * sizeof(PrevMv));
    } else {
      for (size_t i = 0; i < mi_len; ++i) {
        prev[i].ref_frame[0] = D.last_mi[i].ref_frame[0];
        prev[i].ref_frame[1] = D.last_mi[i].ref_frame[1];
        prev[i].mv[0] = D.last_mi[i].mv[0][3];
        prev[i].mv[1] = D.last_mi[i].mv[1][3];
      }
    }
  }
  uint64_t nb = 0, nt = 0, nc = 0;
  for (Chain& ch : chains) {
    ch.blocks_at = nb;
    ch.toks_at = nt;
    ch.coefs_at = nc;
    nb += ch.blocks_cap;
    nt += ch.toks_cap;
    nc += ch.coefs_cap;
  }
  std::vector<rv9_block> blocks(nb);
  std::vector<rv9_tok> toks(nt);
  std::vector<uint32_t> coefs(nc);
  std::vector<ChainOut> outs(chains.size());
  uint8_t tc[1024];
  for (size_t i = 0; i < chains.size(); ++i)
    parse_chain(&D.tables, &fin, chains[i], spans.data(), x.tiles, mi.data(), above.data(), prev.data(),
                blocks.data(), toks.data(), coefs.data(), tc, reinterpret_cast<const uint32_t*>(fin.coef_pk),
                &outs[i]);
  int first = -1;
  for (size_t i = 0; i < chains.size(); ++i) {
    D.bools += outs[i].bools;
    if (outs[i].err && (first < 0 || outs[i].err_tile < outs[first].err_tile)) first = (int)i;
  }
  if (first >= 0) {
    *msg = error_message(outs[first].err);
    return rv9::ST_BITSTREAM;
  }
  out->blocks.clear();
  out->toks.clear();
  out->coefs.clear();
  for (size_t i = 0; i < chains.size(); ++i) {
    const uint32_t tok_base = (uint32_t)out->toks.size(), coef_base = (uint32_t)out->coefs.size();
    for (uint32_t k = 0; k < outs[i].n_blocks; ++k) {
      rv9_block b = blocks[chains[i].blocks_at + k];
      b.tok_start += tok_base;
      out->blocks.push_back(b);
    }
    for (uint32_t k = 0; k < outs[i].n_toks; ++k) {
      rv9_tok t = toks[chains[i].toks_at + k];
      t.coef_start += coef_base;
      out->toks.push_back(t);
    }
    out->coefs.insert(out->coefs.end(), coefs.begin() + chains[i].coefs_at,
                      coefs.begin() + chains[i].coefs_at + outs[i].n_coefs);
  }
  D.last_mi.swap(mi);
  D.last_cols = fin.mi_cols;
  D.last_rows = fin.mi_rows;
  return rv9::ST_OK;
}

}  // namespace

extern "C" {

// Parses the packets (superframes split) frame by frame with the host parser,
// and as the decoder's device-parse mode does with a batch window of `window`
// frames: frames the device parser may take are begun and gathered until the
// window fills or a frame for the host parser comes; then the batch's frames
// are parsed (here by the CPU build of the device parser, in order, each
// taking the previous frame's vectors from the batch's previous frame, else
// from the host parser's state, else from the last device-parsed frame) and
// finished in order; a host frame then rebinds the previous vectors
// (bind_prev) and takes device-held ones when it reads them. Every frame's
// status, message and records must equal frame-by-frame parsing. After an
// error the rest of the batch is dropped, as the decoder drops it, and both
// go on with the frame after the failed one. Returns the number of frames the
// device parser took (>= 0), or -1 with a message. bools_out: boolean decodes
// of the device-parsed tiles.
int device_parse_check(const uint8_t* const* pkts, const size_t* lens, size_t n, int window, char* msg,
                       size_t msg_cap, uint64_t* bools_out) {
  std::vector<std::pair<const uint8_t*, size_t>> frames;
  std::vector<std::pair<size_t, size_t>> split;
  for (size_t i = 0; i < n; ++i) {
    rv9::superframe_split(pkts[i], lens[i], &split);
    for (auto& f : split) frames.emplace_back(pkts[i] + f.first, f.second);
  }
  std::unique_ptr<DeviceSide> D(new DeviceSide);
  fill_tables(&D->tables);
  rv9::Parser ref, par;
  ref.set_threads(1);
  par.set_threads(1);
  std::vector<rv9::Status> want_st(frames.size());
  std::vector<rv9::ParsedFrame> want(frames.size());
  std::vector<std::string> want_err(frames.size());
  for (size_t i = 0; i < frames.size(); ++i)
    want_st[i] = ref.parse_frame(frames[i].first, frames[i].second, &want[i], &want_err[i]);
  int taken = 0;
  struct Pending {
    rv9::Parser::Job* job;
    size_t idx;
    rv9::Parser::ExternalTiles x;
    bool prev_from_batch;
  };
  std::vector<Pending> pending;
  auto check = [&](size_t i, rv9::Status st, const std::string& err, const rv9::ParsedFrame& got, bool dev) {
    if (st != want_st[i] || (st != rv9::ST_OK && err != want_err[i])) {
      snprintf(msg, msg_cap, "frame %zu%s: status %d (%s), host %d (%s)", i, dev ? " (device)" : "", (int)st,
               err.c_str(), (int)want_st[i], want_err[i].c_str());
      return false;
    }
    char why[160] = "";
    if (st == rv9::ST_OK && !same_records(got, want[i], why, sizeof why)) {
      snprintf(msg, msg_cap, "frame %zu%s: %s", i, dev ? " (device)" : "", why);
      return false;
    }
    return true;
  };
  // Returns the index of the frame the next frame to begin follows: the
  // failed frame's successor after an error, else `next`. -1: mismatch.
  auto flush = [&](size_t next, long* resume) -> bool {
    *resume = (long)next;
    for (size_t k = 0; k < pending.size(); ++k) {
      Pending& pe = pending[k];
      rv9::ParsedFrame got;
      std::string tmsg, err;
      bool planned = false;
      const rv9::Parser::ExternalTiles& x = pe.x;
      // The source DeviceParser::add picks.
      int prev_mode = 0;
      if (x.use_prev) {
        if (pe.prev_from_batch) {
          prev_mode = 2;
          ++g_prev_counts[0];
        } else if (x.prev_external) {
          prev_mode = 2;
          ++g_prev_counts[2];
        } else if (x.prev_host) {
          prev_mode = 1;
          ++g_prev_counts[1];
        }
      }
      rv9::Status tst = device_frame(*D, x, prev_mode, &got, &tmsg, &planned);
      rv9::ParsedFrame meta;
      rv9::Status st = par.finish_external(pe.job, tst, tmsg, &meta, &err);
      par.release(pe.job);
      if (st == rv9::ST_OK) {
        meta.blocks.swap(got.blocks);
        meta.toks.swap(got.toks);
        meta.coefs.swap(got.coefs);
      }
      ++taken;
      if (!check(pe.idx, st, err, meta, true)) return false;
      if (st != rv9::ST_OK) {
        for (size_t j = k + 1; j < pending.size(); ++j) par.release(pending[j].job);
        *resume = (long)pe.idx + 1;
        pending.clear();
        return true;
      }
    }
    pending.clear();
    return true;
  };
  size_t i = 0;
  while (i < frames.size()) {
    rv9::Parser::Job* job = par.begin(frames[i].first, frames[i].second, nullptr);
    rv9::Parser::ExternalTiles x;
    bool dev = par.external_tiles(job, &x);
    if (dev) {
      // The device parser refuses a frame whose tiles do not split.
      std::vector<Span> sp;
      std::vector<Chain> ch;
      if (plan_frame(*x.h, x.tiles, x.tiles_len, 0, 0, &sp, &ch)) dev = false;
      if (dev && x.use_prev && pending.empty() && x.prev_external && D->last_mi.empty()) dev = false;
    }
    if (dev) {
      pending.push_back(Pending{job, i, x, !pending.empty()});
      ++i;
      if ((int)pending.size() >= window) {
        long resume;
        if (!flush(i, &resume)) return -1;
        i = (size_t)resume;
      }
      continue;
    }
    long resume;
    if (!flush(i, &resume)) {
      par.release(job);
      return -1;
    }
    if ((size_t)resume != i) {
      // An error in the batch: this frame was begun after it; drop it.
      par.release(job);
      i = (size_t)resume;
      continue;
    }
    par.bind_prev(job);
    if (par.wants_external_prev(job) && !D->last_mi.empty()) {
      std::vector<rv9g::tp::PrevMv> prev(D->last_mi.size());
      for (size_t k = 0; k < prev.size(); ++k) {
        prev[k].ref_frame[0] = D->last_mi[k].ref_frame[0];
        prev[k].ref_frame[1] = D->last_mi[k].ref_frame[1];
        prev[k].mv[0] = D->last_mi[k].mv[0][3];
        prev[k].mv[1] = D->last_mi[k].mv[1][3];
      }
      par.provide_prev_mvs(job, prev.data(), prev.size());
      ++g_prev_counts[3];
    }
    rv9::ParsedFrame got;
    std::string err;
    par.attach_work(job);
    par.run(job);
    rv9::Status st = par.finish(job, &got, &err);
    par.release(job);
    if (!check(i, st, err, got, false)) return -1;
    ++i;
  }
  long resume;
  if (!flush(frames.size(), &resume)) return -1;
  if (bools_out) *bools_out = D->bools;
  return taken;
}

void device_parse_prev_counts(uint64_t* out) {
  for (int k = 0; k < 4; ++k) out[k] = g_prev_counts[k];
}

}  // extern "C"

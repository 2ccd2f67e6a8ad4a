// Serving engine of rv9_server.h: many live streams on one GPU.
//
// Each stream owns a host parser and a reconstruction engine (reference
// slots, pooled frames, its own CUDA stream). Host workers take one request
// at a time from streams that are ready and parse it. Then, in the plain
// form, the worker launches its frames' reconstruction on the stream's CUDA
// stream and queues the copies of the shown frames into pinned buffers; a
// host function queued after them on the same CUDA stream completes the
// request. One stream is only ever worked on by one worker at a time, so its
// requests complete in order, while requests of different streams overlap
// on the device.
//
// In the batched form (rv9_engine_create_batched) the worker only stages the
// parsed frames (work lists built and copied to the device) and hands them
// to its stream's group. A launcher thread per group forms steps as frames
// arrive: the next staged frame of every stream of the group that has one,
// reconstructed together with one launch per stage (Engine::launch_step),
// then the shown frames' copies and the completions, all on the group's CUDA
// stream. A launcher keeps at most kStepsAhead steps queued on the device,
// so that while the GPU is busy, frames arriving meanwhile join the next
// step. Requests of a stream still complete in order (one CUDA stream per
// group), and requests arriving while others are on the GPU join the next
// step: continuous batching on the device.
//
// With device parsing (rv9_engine_set_device_parse, plain form), a worker
// that takes a stream with several queued requests takes a window of them
// and parses their frames on the GPU as one batch (one thread per tile
// column of every frame, rv9g::DeviceParser), then reconstructs them on the
// stream's CUDA stream as above. While a batch parses, the worker sleeps
// and the other workers parse other streams' requests on the host, so the
// device parser adds to the host's parsing rate rather than replacing it.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/rv9_server.h"
#include "../api/api_internal.h"
#include "../gpu/device_parse.h"
#include "../gpu/engine.h"
#include "../host/parser.h"

namespace {

using Clock = std::chrono::steady_clock;

constexpr int kReservedFrames = 10;  // eight slots, the frame being built, one spare
constexpr int kOutBuffers = 4;       // pinned output buffers per stream
constexpr int kMaxShown = 2;         // shown frames one request may carry
constexpr int kStepsAhead = 2;       // batched form: steps queued on the device per group
constexpr int kTableRing = kStepsAhead + 2;  // batch-table buffers per group
constexpr uint32_t kDefaultBatches = 32;     // device-parse batches in flight (the device's hardware queues)

struct OutBuf {
  uint8_t* data = nullptr;
  size_t cap = 0;
};

struct Request {
  uint64_t tag = 0;
  std::vector<uint8_t> packet;
  double submit_ms = 0;
};

struct Stream;

// A finished (or failed) request on its way to rv9_poll.
struct Done {
  std::shared_ptr<Stream> stream;
  int64_t stream_id = 0;
  uint64_t tag = 0;
  rv9_status status = RV9_OK;
  std::string err;
  double submit_ms = 0, latency_ms = 0;
  int out = -1;  // index of the stream's output buffer, or -1
  uint32_t n_frames = 0;
  size_t out_used = 0;  // bytes of the output buffer its frames fill
  rv9_frame frames[kMaxShown];
  // A second shown frame that the output buffer (one frame of the stream's
  // largest size) cannot hold: a packet normally shows one frame.
  std::vector<uint8_t> extra;
};

enum StreamState { PENDING, ADMITTING, ACTIVE, CLOSED };

struct Stream {
  int64_t id = 0;
  rv9_stream_spec spec{};
  uint64_t reservation = 0;
  StreamState state = PENDING;
  bool busy = false;         // a worker holds it
  bool closing = false;      // close requested
  bool needs_reset = false;  // a device error: reset the engine's scratch first
  int inflight = 0;          // requests launched, not yet completed
  std::deque<Request> queue;
  // Batched form: the stream's group, its staged frames awaiting a step
  // (in order; an entry without a frame only completes its request), and
  // whether the group's launcher is using the stream's engine now.
  int group = 0;
  struct Staged {
    bool has_frame = false;
    rv9g::FrameWork fw;
    const uint8_t* d_base = nullptr;
    Done* done = nullptr;  // set on a request's last entry: completes it
  };
  std::deque<Staged> ready;
  bool launching = false;
  Done* open_done = nullptr;  // launcher: the request whose frames it is launching
  rv9::Parser parser;
  std::unique_ptr<rv9g::Engine> engine;
  std::vector<OutBuf> outs;
  std::vector<int> free_outs;
  // Device parsing: requests per batch (0: off for this stream) and the
  // stream's device parser, its buffers allocated at admission. Batches
  // parse on the engine's CUDA stream, ahead of their reconstruction, and
  // the engine runs without its side stream: one CUDA stream per stream
  // keeps the device's hardware queues (32 at most) from being shared
  // between streams, where one stream's parse, hundreds of milliseconds
  // long, would hold up the other's reconstruction.
  uint32_t dp_window = 0;
  std::unique_ptr<rv9g::DeviceParser> dp;
  ~Stream() {
    for (OutBuf& b : outs) cudaFreeHost(b.data);
  }
};

size_t stage_bytes_of(const rv9_stream_spec& s) {
  return std::max<size_t>((size_t)s.max_width * s.max_height * 3, 1 << 20);
}

uint64_t reservation_of(const rv9_stream_spec& s) {
  return rv9g::Engine::footprint(s.max_width, s.max_height, s.ss_x, s.ss_y, s.bit_depth, kReservedFrames,
                                 stage_bytes_of(s));
}

// A stream's reservation when its requests may parse on the device in
// batches of `window` frames: the device parser's buffers are added.
uint64_t reservation_of(const rv9_stream_spec& s, uint32_t window) {
  uint64_t r = reservation_of(s);
  if (window) r += rv9g::DeviceParser::footprint(s.max_width, s.max_height, s.ss_x, s.ss_y, window, 1);
  return r;
}

size_t packed_cap(const rv9_stream_spec& s) {
  size_t bps = s.bit_depth > 8 ? 2 : 1;
  size_t cw = (s.max_width + s.ss_x) >> s.ss_x, ch = (s.max_height + s.ss_y) >> s.ss_y;
  return ((size_t)s.max_width * s.max_height + 2 * cw * ch) * bps;
}

}  // namespace

namespace {

// A group of the batched form: its CUDA stream, launcher thread and the
// pinned / device batch tables of its steps in flight (a ring).
struct Group {
  cudaStream_t stream = nullptr;
  std::thread launcher;
  struct Tables {
    uint8_t* h = nullptr;
    uint8_t* d = nullptr;
    size_t cap = 0;
    cudaEvent_t done = nullptr;  // the step that last used them
  } ring[kTableRing];
  int next = 0;
  cudaEvent_t step_done[kStepsAhead] = {};
  int step = 0;
  uint64_t steps = 0, frames = 0;  // statistics
};

// The rv9_frame of a shown frame whose packed planes go to `data`.
void fill_frame(const rv9g::DevFrame* shown, uint8_t* data, size_t nb, rv9_frame* f) {
  memset(f, 0, sizeof *f);
  f->width = shown->width;
  f->height = shown->height;
  f->bit_depth = shown->bit_depth;
  f->chroma = shown->ss_x ? (shown->ss_y ? RV9_YUV420 : RV9_YUV422) : (shown->ss_y ? RV9_YUV440 : RV9_YUV444);
  f->color_space = shown->color_space;
  f->full_range = shown->color_range;
  f->render_width = shown->render_w;
  f->render_height = shown->render_h;
  f->data = data;
  f->size = nb;
  size_t poff = 0, bps = shown->bps();
  for (int p = 0; p < 3; ++p) {
    uint32_t w = p ? (shown->width + shown->ss_x) >> shown->ss_x : shown->width;
    uint32_t h = p ? (shown->height + shown->ss_y) >> shown->ss_y : shown->height;
    f->planes[p].offset = poff;
    f->planes[p].width = w;
    f->planes[p].height = h;
    poff += (size_t)w * h * bps;
  }
}

}  // namespace

struct rv9_engine {
  int device = 0;
  uint64_t budget = 0, reserved = 0;
  // Batched form: launch groups (empty in the plain form).
  std::vector<std::unique_ptr<Group>> groups;
  std::condition_variable ready_cv;
  int next_group = 0;
  Clock::time_point t0 = Clock::now();
  std::mutex mu;
  std::condition_variable work_cv, done_cv, idle_cv;
  std::map<int64_t, std::shared_ptr<Stream>> streams;
  std::deque<int64_t> pending;  // admission order
  std::deque<Done*> done;
  std::set<Done*> polled;  // handed out by rv9_poll, not yet released
  int64_t next_id = 1;
  bool stop = false;
  bool stop_launchers = false;
  std::vector<std::thread> workers;
  size_t cursor = 0;
  uint64_t n_submitted = 0, n_completed = 0, n_frames = 0;
  // Device parsing (plain form): requests per batch (0: off), batches on the
  // device at once, and statistics.
  uint32_t dp_window = 0, dp_max = 0;
  int dp_active = 0;
  uint64_t dp_batches = 0, dp_frames = 0, dp_wait_us = 0, dp_batch_us = 0;
  int n_host_workers = 0;
  uint32_t n_extra_workers = 0;  // workers added for device-parse batches

  double now_ms() const { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }

  // Admits pending streams in order while the budget allows (caller holds mu).
  void admit_locked() {
    while (!pending.empty()) {
      auto it = streams.find(pending.front());
      if (it == streams.end()) {
        pending.pop_front();
        continue;
      }
      Stream& s = *it->second;
      if (reserved + s.reservation > budget) break;
      reserved += s.reservation;
      s.state = ADMITTING;
      pending.pop_front();
    }
  }

  // Fails every queued request of `sp` with `st` (caller holds mu).
  void fail_queue_locked(const std::shared_ptr<Stream>& sp, rv9_status st, const std::string& err) {
    Stream& s = *sp;
    while (!s.queue.empty()) {
      Done* d = new Done;
      d->stream = sp;
      d->stream_id = s.id;
      d->tag = s.queue.front().tag;
      d->submit_ms = s.queue.front().submit_ms;
      d->status = st;
      d->err = err;
      d->latency_ms = now_ms() - d->submit_ms;
      s.queue.pop_front();
      ++n_completed;
      done.push_back(d);
    }
    done_cv.notify_all();
  }

  enum Action { NONE, ADMIT, DECODE, CLOSE };

  // The next stream a worker may take, and what to do with it (caller holds
  // mu): admit it, decode its next request (it has one and a free output
  // buffer), or close it (closing and drained). Round-robin over streams.
  Action pick_locked(std::shared_ptr<Stream>* out) {
    if (streams.empty()) return NONE;
    std::vector<std::shared_ptr<Stream>> order;
    order.reserve(streams.size());
    for (auto& kv : streams) order.push_back(kv.second);
    size_t n = order.size();
    for (size_t k = 0; k < n; ++k) {
      auto& s = order[(cursor + k) % n];
      if (s->busy) continue;
      Action a = NONE;
      // In the batched form a stream's next request is parsed once its
      // staged frames have gone to the device (the engine's two staging
      // buffers bound what may wait) and its launcher is done with it.
      const bool staged_free = s->ready.empty() && !s->launching;
      if (s->state == ADMITTING)
        a = ADMIT;
      else if (s->state == ACTIVE && !s->queue.empty() && !s->free_outs.empty() && staged_free)
        a = DECODE;
      else if (s->state == ACTIVE && s->closing && s->queue.empty() && s->inflight == 0 && staged_free)
        a = CLOSE;
      if (a != NONE) {
        cursor = (cursor + k + 1) % n;
        s->busy = true;
        *out = s;
        return a;
      }
    }
    return NONE;
  }

  // Returns a completion's output buffer to its stream and frees it (caller
  // holds mu). The stream reference comes back to be dropped after the lock
  // is released: the last one frees pinned memory, which must not happen
  // under the lock that completion callbacks take.
  std::shared_ptr<Stream> release_locked(Done* d) {
    if (d->out >= 0) d->stream->free_outs.push_back(d->out);
    std::shared_ptr<Stream> keep = std::move(d->stream);
    delete d;
    work_cv.notify_all();
    return keep;
  }

  void finish(Done* d) {
    std::lock_guard<std::mutex> lock(mu);
    d->latency_ms = now_ms() - d->submit_ms;
    if (d->stream->engine && d->stream->engine->error_word() != 0) {
      // The engine's scratch is reset before the stream's next request.
      d->stream->needs_reset = true;
      if (d->status == RV9_OK) {
        d->status = RV9_DEVICE;
        d->err = "a device-side wait timed out";
      }
    }
    d->stream->inflight -= 1;
    ++n_completed;
    if (d->status == RV9_OK) n_frames += d->n_frames;
    done.push_back(d);
    done_cv.notify_all();
    work_cv.notify_all();
    idle_cv.notify_all();
  }

  struct Callback {
    rv9_engine* eng;
    Done* d;
  };
  static void CUDART_CB host_fn(void* p) {
    Callback* c = static_cast<Callback*>(p);
    c->eng->finish(c->d);
    delete c;
  }

  // Device-parse batches: the worker waits (asleep) for the batch's copies,
  // then completes its requests in order. A host function per request (as
  // the plain form queues) was measured to block its own queuing call for
  // seconds once 32 streams' batches were in flight, each request behind a
  // parse hundreds of milliseconds long; one per batch still blocked for
  // about a second.
  void complete_when_done(Stream& s, std::vector<Done*>* ds) {
    if (ds->empty()) return;
    std::string e;
    const rv9::Status st = s.dp->wait_on(s.engine->stream(), &e);
    for (Done* d : *ds) {
      if (st != rv9::ST_OK && d->status == RV9_OK) {
        d->status = (rv9_status)st;
        d->err = e;
      }
      finish(d);
    }
    ds->clear();
  }

  // Queues the completion behind the stream's device work.
  void complete_after_device(Stream& s, Done* d) {
    Callback* cb = new Callback{this, d};
    if (cudaLaunchHostFunc(s.engine->stream(), host_fn, cb) == cudaSuccess) return;
    delete cb;
    if (d->status == RV9_OK) {
      d->status = RV9_DEVICE;
      d->err = "could not queue the completion";
    }
    finish(d);
  }

  void admit(const std::shared_ptr<Stream>& sp) {
    Stream& s = *sp;
    std::string err;
    std::unique_ptr<rv9g::Engine> engine(new rv9g::Engine);
    // A stream that parses on the device keeps all its work on one CUDA
    // stream (see Stream::dp).
    bool ok = engine->init(device, &err, s.dp_window == 0);
    if (ok)
      ok = engine->reserve(s.spec.max_width, s.spec.max_height, s.spec.ss_x, s.spec.ss_y, s.spec.bit_depth,
                           kReservedFrames, stage_bytes_of(s.spec), &err) == rv9::ST_OK;
    std::vector<OutBuf> outs;
    size_t cap = packed_cap(s.spec);
    // A device-parse batch takes a free output buffer per request; twice
    // the window lets the next batch fill while the last one's buffers are
    // still with the caller.
    const int n_outs = std::max(kOutBuffers, 2 * (int)s.dp_window);
    for (int i = 0; ok && i < n_outs; ++i) {
      OutBuf b;
      if (cudaMallocHost(&b.data, cap) != cudaSuccess) {
        ok = false;
        err = "out of pinned host memory for output buffers";
        break;
      }
      b.cap = cap;
      outs.push_back(b);
    }
    std::unique_ptr<rv9g::DeviceParser> dp;
    if (ok && s.dp_window) {
      dp.reset(new rv9g::DeviceParser);
      // A batch's reconstruction ends before the stream's next batch is
      // launched (complete_when_done): one stage buffer is enough.
      dp->set_single_stage();
      ok = dp->init(device, &err) == rv9::ST_OK &&
           dp->reserve(s.spec.max_width, s.spec.max_height, s.spec.ss_x, s.spec.ss_y, s.dp_window, &err) ==
               rv9::ST_OK;
    }
    std::lock_guard<std::mutex> lock(mu);
    s.outs = std::move(outs);
    if (ok) {
      s.engine = std::move(engine);
      s.dp = std::move(dp);
      for (int i = 0; i < (int)s.outs.size(); ++i) s.free_outs.push_back(i);
      if (!groups.empty()) s.group = next_group++ % (int)groups.size();
      s.state = ACTIVE;
    } else {
      // Fail the stream's requests and drop it; its reservation returns.
      s.state = CLOSED;
      s.closing = true;
      reserved -= s.reservation;
      fail_queue_locked(sp, RV9_DEVICE, err.empty() ? "admission failed" : err);
      streams.erase(s.id);
      admit_locked();
      idle_cv.notify_all();
    }
    s.busy = false;
    work_cv.notify_all();
  }

  void close_drained(const std::shared_ptr<Stream>& sp) {
    Stream& s = *sp;
    std::unique_ptr<rv9g::Engine> engine;
    {
      std::lock_guard<std::mutex> lock(mu);
      reserved -= s.reservation;
      s.state = CLOSED;
      engine.swap(s.engine);
      streams.erase(s.id);
      admit_locked();
      s.busy = false;
      work_cv.notify_all();
    }
    engine.reset();  // outside the lock: frees device memory
    s.dp.reset();
    std::lock_guard<std::mutex> lock(mu);
    idle_cv.notify_all();
  }

  void decode_request(const std::shared_ptr<Stream>& sp) {
    Stream& s = *sp;
    if (s.needs_reset) {
      std::string err;
      // Nothing of the stream is in flight on its group's stream after this.
      if (!groups.empty()) cudaStreamSynchronize(groups[(size_t)s.group]->stream);
      s.engine->sync(&err);  // reports the error once more and resets the scratch
      s.needs_reset = false;
    }
    if (!groups.empty()) {
      stage_request(sp);
      return;
    }
    Request req;
    int out;
    {
      std::unique_lock<std::mutex> lock(mu);
      // Several requests queued: a device-parse batch of them, while fewer
      // than dp_max batches are on the device. A lone request (low load) is
      // parsed on the host: a batch takes as long as its longest tile
      // column, hundreds of milliseconds at 2160p.
      if (s.dp_window && dp_active < (int)dp_max && s.queue.size() >= 2 && s.free_outs.size() >= 2) {
        const size_t k = std::min<size_t>({s.queue.size(), s.free_outs.size(), s.dp_window});
        ++dp_active;
        lock.unlock();
        decode_batch_device(sp, k);
        return;
      }
      req = std::move(s.queue.front());
      s.queue.pop_front();
      out = s.free_outs.back();
      s.free_outs.pop_back();
      s.inflight += 1;
    }
    Done* d = new Done;
    d->stream = sp;
    d->stream_id = s.id;
    d->tag = req.tag;
    d->submit_ms = req.submit_ms;
    d->out = out;
    std::string err;
    std::vector<std::pair<size_t, size_t>> frames;
    rv9::superframe_split(req.packet.data(), req.packet.size(), &frames);
    if (req.packet.empty()) {
      d->status = RV9_BITSTREAM;
      d->err = "empty packet";
    }
    rv9::ParsedFrame pf;
    for (auto& fr : frames) {
      rv9::Status st = host_parse(s, s.parser.begin(req.packet.data() + fr.first, fr.second, nullptr), &pf, &err);
      rv9g::DevFrame* shown = nullptr;
      if (st == rv9::ST_OK) st = s.engine->recon(pf, &shown, &err);
      if (st != rv9::ST_OK) {
        d->status = (rv9_status)st;
        d->err = err;
        break;
      }
      if (!shown) continue;
      place_frame(s, d, shown, s.engine->stream());
      if (d->status != RV9_OK) break;
    }
    complete_after_device(s, d);
    std::lock_guard<std::mutex> lock(mu);
    s.busy = false;
    work_cv.notify_all();
  }

  // One frame parsed on the host (a job from s.parser.begin; released here).
  // When the frame before it was parsed on the device, the motion vectors
  // the frame may read are on the device too: they are read back first.
  rv9::Status host_parse(Stream& s, rv9::Parser::Job* job, rv9::ParsedFrame* pf, std::string* err) {
    if (s.dp) {
      s.parser.bind_prev(job);
      if (s.parser.wants_external_prev(job) && s.dp->have_last()) {
        std::vector<rv9g::tp::PrevMv> prev;
        rv9::Status st = s.dp->last_prev(&prev, s.engine->stream(), err);
        if (st != rv9::ST_OK) {
          s.parser.release(job);
          return st;
        }
        s.parser.provide_prev_mvs(job, prev.data(), prev.size());
      }
    }
    s.parser.attach_work(job);
    s.parser.run(job);
    rv9::Status st = s.parser.finish(job, pf, err);
    s.parser.release(job);
    return st;
  }

  // Plain form with device parsing: the stream's next k requests. Their
  // frames go, in decode order, to one device batch where the device parser
  // takes them (rv9::Parser::external_tiles); a frame it does not take is
  // parsed on the host once the batch before it is reconstructed. Each
  // request completes behind the copies of its shown frames. A frame that
  // fails fails its request and drops the batch's later frames, whose
  // requests fail with it; the requests after the batch decode as usual.
  void decode_batch_device(const std::shared_ptr<Stream>& sp, size_t k) {
    Stream& s = *sp;
    std::vector<Request> reqs(k);
    std::vector<Done*> dones(k);
    {
      std::lock_guard<std::mutex> lock(mu);
      for (size_t r = 0; r < k; ++r) {
        reqs[r] = std::move(s.queue.front());
        s.queue.pop_front();
        Done* d = new Done;
        d->stream = sp;
        d->stream_id = s.id;
        d->tag = reqs[r].tag;
        d->submit_ms = reqs[r].submit_ms;
        d->out = s.free_outs.back();
        s.free_outs.pop_back();
        dones[r] = d;
      }
      s.inflight += (int)k;
    }
    const cudaStream_t es = s.engine->stream();
    const auto t_batch = Clock::now();
    uint64_t wait_us = 0;
    std::string err;
    std::vector<int> open(k, 0);         // the request's frames waiting in the batch
    std::vector<char> begun(k, 0);       // every frame of the request begun
    size_t next_done = 0;
    uint64_t n_dev = 0;
    auto fail = [&](size_t r, rv9::Status st, const std::string& msg) {
      if (dones[r]->status != RV9_OK) return;
      dones[r]->status = (rv9_status)st;
      dones[r]->err = msg;
    };
    // Requests in order, each once its frames are all queued; they complete
    // together when the batch's copies are done.
    std::vector<Done*> ready;
    auto complete_ready = [&]() {
      while (next_done < k && begun[next_done] && open[next_done] == 0) ready.push_back(dones[next_done++]);
    };
    struct Pend {
      rv9::Parser::Job* job;
      size_t owner;
    };
    std::vector<Pend> pending;
    // Drops the batch's frames from i on (their requests fail) and hands the
    // stage buffer back behind the reconstructions already queued from it.
    auto drop_from = [&](size_t i, rv9::Status st, const std::string& msg) {
      for (size_t j = i; j < pending.size(); ++j) {
        s.parser.release(pending[j].job);
        fail(pending[j].owner, st, msg);
        open[pending[j].owner] -= 1;
      }
      pending.clear();
      std::string ignored;
      s.dp->recon_queued(es, &ignored);
      s.dp->clear();
    };
    auto flush = [&]() {
      if (pending.empty()) return;
      rv9g::DeviceParser& P = *s.dp;
      std::string e2;
      const auto tw = Clock::now();
      rv9::Status st = P.launch(es, &e2);
      if (st == rv9::ST_OK) st = P.collect(es, &e2);
      wait_us += (uint64_t)std::chrono::duration_cast<std::chrono::microseconds>(Clock::now() - tw).count();
      if (st != rv9::ST_OK) {
        drop_from(0, st, e2);
        complete_ready();
        return;
      }
      for (size_t i = 0; i < pending.size(); ++i) {
        const size_t r = pending[i].owner;
        std::string msg;
        const rv9::Status ts = P.frame_status(i, &msg);
        rv9::ParsedFrame meta;
        st = s.parser.finish_external(pending[i].job, ts, msg, &meta, &e2);
        s.parser.release(pending[i].job);
        pending[i].job = nullptr;
        open[r] -= 1;
        if (st == rv9::ST_OK) {
          rv9g::FrameWork fw;
          fw.desc = meta.desc;
          fw.show_existing = false;
          fw.show_frame = meta.show_frame;
          fw.refresh_mask = meta.refresh_mask;
          for (int q = 0; q < 3; ++q) fw.ref_slot[q] = meta.ref_slot[q];
          P.frame_work(i, &fw);
          rv9g::DevFrame* shown = nullptr;
          st = s.engine->recon_resident(fw, P.frame_base(i), &shown, &e2);
          if (st == rv9::ST_OK) {
            ++n_dev;
            if (shown && dones[r]->status == RV9_OK) place_frame(s, dones[r], shown, es);
          }
        }
        if (st != rv9::ST_OK) {
          fail(r, st, e2);
          drop_from(i + 1, st, "an earlier frame of the stream failed: " + e2);
          complete_ready();
          return;
        }
        complete_ready();
      }
      pending.clear();
      // Should the stage buffer's release fail to queue, the batch's
      // reconstructions end before the buffer is written again.
      if (P.recon_queued(es, &e2) != rv9::ST_OK) cudaStreamSynchronize(es);
      P.clear();
    };
    std::vector<std::pair<size_t, size_t>> frames;
    rv9::ParsedFrame pf;
    for (size_t r = 0; r < k; ++r) {
      const Request& q = reqs[r];
      Done* d = dones[r];
      if (q.packet.empty()) fail(r, rv9::ST_BITSTREAM, "empty packet");
      rv9::superframe_split(q.packet.data(), q.packet.size(), &frames);
      for (auto& fr : frames) {
        if (d->status != RV9_OK) break;
        rv9::Parser::Job* job = s.parser.begin(q.packet.data() + fr.first, fr.second, nullptr);
        rv9::Parser::ExternalTiles x;
        if (s.parser.external_tiles(job, &x) && s.dp->add(x, *x.desc)) {
          pending.push_back({job, r});
          open[r] += 1;
          if (pending.size() >= s.dp_window || s.dp->stage_bytes() >= (4ull << 30)) flush();
          continue;
        }
        // A frame for the host parser: the batch before it first.
        flush();
        if (d->status != RV9_OK) {
          s.parser.release(job);
          break;
        }
        rv9::Status st = host_parse(s, job, &pf, &err);
        rv9g::DevFrame* shown = nullptr;
        if (st == rv9::ST_OK) st = s.engine->recon(pf, &shown, &err);
        if (st != rv9::ST_OK) {
          fail(r, st, err);
          break;
        }
        if (shown) place_frame(s, d, shown, es);
      }
      begun[r] = 1;
      complete_ready();
    }
    flush();
    complete_ready();
    complete_when_done(s, &ready);
    std::lock_guard<std::mutex> lock(mu);
    --dp_active;
    dp_batches += 1;
    dp_frames += n_dev;
    dp_wait_us += wait_us;
    dp_batch_us += (uint64_t)std::chrono::duration_cast<std::chrono::microseconds>(Clock::now() - t_batch).count();
    s.busy = false;
    work_cv.notify_all();
  }

  // Batched form, worker side: parses the stream's next request and stages
  // its frames for the group's launcher; the request's last entry carries
  // its completion (alone, when parsing failed before any frame).
  void stage_request(const std::shared_ptr<Stream>& sp) {
    Stream& s = *sp;
    Request req;
    int out;
    {
      std::lock_guard<std::mutex> lock(mu);
      req = std::move(s.queue.front());
      s.queue.pop_front();
      out = s.free_outs.back();
      s.free_outs.pop_back();
      s.inflight += 1;
    }
    Done* d = new Done;
    d->stream = sp;
    d->stream_id = s.id;
    d->tag = req.tag;
    d->submit_ms = req.submit_ms;
    d->out = out;
    std::vector<Stream::Staged> staged;
    std::string err;
    std::vector<std::pair<size_t, size_t>> frames;
    rv9::superframe_split(req.packet.data(), req.packet.size(), &frames);
    if (req.packet.empty()) {
      d->status = RV9_BITSTREAM;
      d->err = "empty packet";
    }
    const cudaStream_t gs = groups[(size_t)s.group]->stream;
    rv9::ParsedFrame pf;
    for (auto& fr : frames) {
      rv9::Status st = s.parser.parse_frame(req.packet.data() + fr.first, fr.second, &pf, &err);
      Stream::Staged it;
      if (st == rv9::ST_OK) st = s.engine->stage(pf, gs, &it.fw, &it.d_base, &err);
      if (st != rv9::ST_OK) {
        d->status = (rv9_status)st;
        d->err = err;
        break;
      }
      it.has_frame = true;
      staged.push_back(std::move(it));
    }
    if (staged.empty()) staged.emplace_back();
    staged.back().done = d;
    std::lock_guard<std::mutex> lock(mu);
    for (auto& it : staged) s.ready.push_back(std::move(it));
    s.busy = false;
    work_cv.notify_all();
    ready_cv.notify_all();
  }

  // Batched form, launcher side: one step at a time for group g.
  void launcher_loop(int g) {
    cudaSetDevice(device);
    Group& G = *groups[(size_t)g];
    std::vector<std::shared_ptr<Stream>> taken;
    std::vector<Stream::Staged> items;
    std::vector<rv9g::Engine*> engines;
    std::vector<const rv9g::FrameWork*> fws;
    std::vector<const uint8_t*> bases;
    std::vector<rv9g::DevFrame*> shown;
    std::vector<size_t> frame_of;  // item -> index in the step's frames, or -1
    for (;;) {
      // At most kStepsAhead steps queued: wait for the oldest to finish, so
      // that frames arriving meanwhile join the next step.
      cudaEventSynchronize(G.step_done[G.step]);
      taken.clear();
      items.clear();
      {
        std::unique_lock<std::mutex> lock(mu);
        ready_cv.wait(lock, [&] {
          if (stop_launchers) return true;
          for (auto& kv : streams)
            if (kv.second->group == g && !kv.second->ready.empty() && !kv.second->launching) return true;
          return false;
        });
        if (stop_launchers) return;
        // The next staged entry of every stream of the group that has one.
        for (auto& kv : streams) {
          Stream& st = *kv.second;
          if (st.group != g || st.ready.empty() || st.launching) continue;
          st.launching = true;
          taken.push_back(kv.second);
          items.push_back(std::move(st.ready.front()));
          st.ready.pop_front();
        }
      }
      engines.clear();
      fws.clear();
      bases.clear();
      frame_of.assign(items.size(), (size_t)-1);
      for (size_t i = 0; i < items.size(); ++i) {
        if (!items[i].has_frame) continue;
        frame_of[i] = engines.size();
        engines.push_back(taken[i]->engine.get());
        fws.push_back(&items[i].fw);
        bases.push_back(items[i].d_base);
      }
      std::string err;
      rv9::Status st = rv9::ST_OK;
      if (!engines.empty()) {
        Group::Tables& tb = G.ring[G.next];
        G.next = (G.next + 1) % kTableRing;
        cudaEventSynchronize(tb.done);  // the step that used them last has finished
        const size_t need = rv9g::Engine::step_table_bytes(engines.size());
        if (need > tb.cap) {
          cudaFree(tb.d);
          cudaFreeHost(tb.h);
          tb.d = tb.h = nullptr;
          tb.cap = 0;
          const size_t cap = std::max(need, (size_t)64 << 10);
          if (cudaMalloc(&tb.d, cap) == cudaSuccess && cudaMallocHost(&tb.h, cap) == cudaSuccess) {
            tb.cap = cap;
          } else {
            st = rv9::ST_DEVICE;
            err = "out of memory for a step's batch tables";
          }
        }
        shown.assign(engines.size(), nullptr);
        if (st == rv9::ST_OK) {
          size_t used = 0;
          int launches = 0;
          st = rv9g::Engine::launch_step(engines.data(), fws.data(), bases.data(), engines.size(), G.stream,
                                         rv9g::TuneParams(), tb.h, tb.d, &used, shown.data(), &launches, &err);
          cudaEventRecord(tb.done, G.stream);
          G.steps += 1;
          G.frames += engines.size();
        }
      }
      // Shown frames to their requests' output buffers, then completions,
      // in stream order behind the step.
      for (size_t i = 0; i < items.size(); ++i) {
        Stream& sm = *taken[i];
        Done* d = items[i].done;
        if (frame_of[i] != (size_t)-1) {
          Done* owner = d ? d : pending_done(sm);
          rv9g::DevFrame* f = st == rv9::ST_OK ? shown[frame_of[i]] : nullptr;
          if (st != rv9::ST_OK && owner->status == RV9_OK) {
            owner->status = (rv9_status)st;
            owner->err = err;
          }
          if (f && owner->status == RV9_OK) place_frame(sm, owner, f, G.stream);
        }
        if (d) {
          sm.open_done = nullptr;
          complete_on(G.stream, d);
        }
      }
      cudaEventRecord(G.step_done[G.step], G.stream);
      G.step = (G.step + 1) % kStepsAhead;
      {
        std::lock_guard<std::mutex> lock(mu);
        for (auto& sp : taken) sp->launching = false;
        work_cv.notify_all();
        ready_cv.notify_all();
      }
      taken.clear();  // (streams may be freed once released)
    }
  }

  // The Done of the stream's request whose frames are being launched (a
  // request's entries before its last carry none): the last entry's, found
  // ahead in the stream's ready queue.
  Done* pending_done(Stream& s) {
    if (s.open_done) return s.open_done;
    std::lock_guard<std::mutex> lock(mu);
    for (auto& it : s.ready)
      if (it.done) {
        s.open_done = it.done;
        break;
      }
    return s.open_done;
  }

  // A shown frame's copy into its request's output buffer (queued on `gs`),
  // or, for a second frame the buffer cannot hold, into the request's heap
  // buffer (a copy into pageable memory, which returns once done).
  void place_frame(Stream& s, Done* d, rv9g::DevFrame* shown, cudaStream_t gs) {
    const size_t nb = rv9g::Engine::packed_bytes(shown);
    if (d->n_frames >= (uint32_t)kMaxShown || nb > packed_cap(s.spec)) {
      d->status = RV9_UNSUPPORTED;
      d->err = "a request showed more frames, or larger ones, than its stream spec allows";
      return;
    }
    const OutBuf& b = s.outs[(size_t)d->out];
    const bool fits = d->out_used + nb <= b.cap;
    uint8_t* dst;
    if (fits) {
      dst = b.data + d->out_used;
    } else {
      d->extra.resize(nb);  // once: the first frame is in the output buffer
      dst = d->extra.data();
    }
    rv9_frame& f = d->frames[d->n_frames++];
    fill_frame(shown, dst, nb, &f);
    std::string err;
    if (s.engine->download_on(shown, f.data, gs, &err) != rv9::ST_OK) {
      d->status = RV9_DEVICE;
      d->err = err;
      return;
    }
    if (fits) d->out_used += nb;
  }

  // Queues the completion behind the work on `gs`.
  void complete_on(cudaStream_t gs, Done* d) {
    Callback* cb = new Callback{this, d};
    if (cudaLaunchHostFunc(gs, host_fn, cb) == cudaSuccess) return;
    delete cb;
    if (d->status == RV9_OK) {
      d->status = RV9_DEVICE;
      d->err = "could not queue the completion";
    }
    finish(d);
  }

  // Joins the launchers (stop_launchers set) and frees the groups' streams,
  // events and tables.
  void destroy_groups() {
    for (auto& G : groups) {
      if (G->launcher.joinable()) G->launcher.join();
      if (G->stream) cudaStreamSynchronize(G->stream);
      for (auto& tb : G->ring) {
        cudaFree(tb.d);
        cudaFreeHost(tb.h);
        if (tb.done) cudaEventDestroy(tb.done);
      }
      for (auto& ev : G->step_done)
        if (ev) cudaEventDestroy(ev);
      if (G->stream) cudaStreamDestroy(G->stream);
    }
    groups.clear();
  }

  void worker_loop() {
    cudaSetDevice(device);
    for (;;) {
      std::shared_ptr<Stream> s;
      Action a = NONE;
      {
        std::unique_lock<std::mutex> lock(mu);
        work_cv.wait(lock, [&] { return stop || (a = pick_locked(&s)) != NONE; });
        if (a == NONE) return;  // stop
      }
      if (a == ADMIT)
        admit(s);
      else if (a == CLOSE)
        close_drained(s);
      else
        decode_request(s);
    }
  }
};

extern "C" {

uint64_t rv9_stream_reservation(const rv9_stream_spec* spec) { return spec ? reservation_of(*spec) : 0; }

uint64_t rv9_engine_stream_reservation(rv9_engine* e, const rv9_stream_spec* spec) {
  if (!e || !spec) return 0;
  std::lock_guard<std::mutex> lock(e->mu);
  return reservation_of(*spec, e->dp_window);
}

static rv9_engine* engine_create(int device, uint64_t hbm_budget_bytes, uint32_t workers, uint32_t n_groups);

rv9_engine* rv9_engine_create(int device, uint64_t hbm_budget_bytes, uint32_t workers) {
  return engine_create(device, hbm_budget_bytes, workers, 0);
}

rv9_engine* rv9_engine_create_batched(int device, uint64_t hbm_budget_bytes, uint32_t workers, uint32_t groups) {
  return engine_create(device, hbm_budget_bytes, workers, groups ? groups : 1);
}

static rv9_engine* engine_create(int device, uint64_t hbm_budget_bytes, uint32_t workers, uint32_t n_groups) {
  if (!rv9api::host_isa_ok()) return nullptr;
  {
    // The same device check as rv9_decoder_new, with its message.
    rv9g::Engine probe;
    std::string err;
    if (!probe.init(device, &err)) {
      rv9api::set_global_error(err);
      return nullptr;
    }
    device = probe.device();
  }
  rv9_engine* e = new rv9_engine;
  e->device = device;
  e->budget = hbm_budget_bytes;
  if (n_groups) {
    cudaSetDevice(device);
    for (uint32_t g = 0; g < n_groups; ++g) {
      std::unique_ptr<Group> G(new Group);
      bool ok = cudaStreamCreateWithFlags(&G->stream, cudaStreamNonBlocking) == cudaSuccess;
      for (int i = 0; ok && i < kTableRing; ++i)
        ok = cudaEventCreateWithFlags(&G->ring[i].done, cudaEventDisableTiming) == cudaSuccess;
      for (int i = 0; ok && i < kStepsAhead; ++i)
        ok = cudaEventCreateWithFlags(&G->step_done[i], cudaEventDisableTiming) == cudaSuccess;
      e->groups.push_back(std::move(G));
      if (!ok) {
        rv9api::set_global_error("creating the launch groups' CUDA streams and events failed");
        e->destroy_groups();
        delete e;
        return nullptr;
      }
    }
    for (uint32_t g = 0; g < n_groups; ++g)
      e->groups[g]->launcher = std::thread([e, g] { e->launcher_loop((int)g); });
  }
  int n = workers ? (int)workers : (int)std::max(1u, std::thread::hardware_concurrency());
  e->n_host_workers = n;
  for (int i = 0; i < n; ++i) e->workers.emplace_back([e] { e->worker_loop(); });
  return e;
}

rv9_status rv9_stream_close(rv9_engine* e, int64_t id);

void rv9_engine_free(rv9_engine* e) {
  if (!e) return;
  std::vector<int64_t> ids;
  {
    std::lock_guard<std::mutex> lock(e->mu);
    for (auto& kv : e->streams) ids.push_back(kv.first);
  }
  for (int64_t id : ids) rv9_stream_close(e, id);
  {
    // Every stream drains and closes, then the workers stop. Completions are
    // released as they come, so that no stream waits for an output buffer.
    std::vector<std::shared_ptr<Stream>> dropped;
    std::unique_lock<std::mutex> lock(e->mu);
    for (;;) {
      for (Done* d : e->polled) dropped.push_back(e->release_locked(d));
      e->polled.clear();
      while (!e->done.empty()) {
        dropped.push_back(e->release_locked(e->done.front()));
        e->done.pop_front();
      }
      if (e->streams.empty()) break;
      lock.unlock();
      dropped.clear();
      lock.lock();
      e->idle_cv.wait_for(lock, std::chrono::milliseconds(20));
    }
    e->stop = true;
    e->work_cv.notify_all();
    lock.unlock();
    dropped.clear();
  }
  for (auto& t : e->workers) t.join();
  {
    std::lock_guard<std::mutex> lock(e->mu);
    e->stop_launchers = true;
    e->ready_cv.notify_all();
  }
  e->destroy_groups();
  for (Done* d : e->done) delete d;
  delete e;
}

rv9_status rv9_stream_open(rv9_engine* e, const rv9_stream_spec* spec, int64_t* id) {
  if (!e || !spec || !id) return RV9_INVALID_INPUT;
  *id = 0;
  if (spec->max_width == 0 || spec->max_height == 0 || spec->max_width > 16384 || spec->max_height > 16384 ||
      (spec->bit_depth != 8 && spec->bit_depth != 10 && spec->bit_depth != 12) || spec->ss_x > 1 || spec->ss_y > 1)
    return RV9_INVALID_INPUT;
  std::lock_guard<std::mutex> lock(e->mu);
  const uint64_t r = reservation_of(*spec, e->dp_window);
  if (r > e->budget) return RV9_UNSUPPORTED;
  auto s = std::make_shared<Stream>();
  s->id = e->next_id++;
  s->spec = *spec;
  s->reservation = r;
  s->dp_window = e->dp_window;
  // Tile columns on threads: one request's latency shrinks when cores are
  // free; under load the workers keep every core busy anyway.
  s->parser.set_threads(0);
  e->streams[s->id] = s;
  e->pending.push_back(s->id);
  e->admit_locked();
  *id = s->id;
  e->work_cv.notify_all();
  return RV9_OK;
}

rv9_status rv9_stream_close(rv9_engine* e, int64_t id) {
  if (!e) return RV9_INVALID_INPUT;
  std::lock_guard<std::mutex> lock(e->mu);
  auto it = e->streams.find(id);
  if (it == e->streams.end()) return RV9_INVALID_INPUT;
  std::shared_ptr<Stream> sp = it->second;
  sp->closing = true;
  if (sp->state == PENDING && sp->queue.empty()) {
    // Never admitted and nothing to do: dropped at once. A pending stream
    // with requests is admitted in turn, decodes them, then closes.
    sp->state = CLOSED;
    e->streams.erase(it);
    e->idle_cv.notify_all();
  }
  e->work_cv.notify_all();
  return RV9_OK;
}

rv9_status rv9_submit(rv9_engine* e, int64_t id, const uint8_t* packet, size_t len, uint64_t tag) {
  if (!e || (!packet && len)) return RV9_INVALID_INPUT;
  Request r;
  r.tag = tag;
  r.packet.assign(packet, packet + len);
  std::lock_guard<std::mutex> lock(e->mu);
  auto it = e->streams.find(id);
  if (it == e->streams.end() || it->second->closing) return RV9_INVALID_INPUT;
  r.submit_ms = e->now_ms();
  it->second->queue.push_back(std::move(r));
  ++e->n_submitted;
  e->work_cv.notify_all();
  return RV9_OK;
}

size_t rv9_poll(rv9_engine* e, rv9_completion* out, size_t cap, int timeout_ms) {
  if (!e || !out || cap == 0) return 0;
  std::unique_lock<std::mutex> lock(e->mu);
  if (e->done.empty() && timeout_ms > 0)
    e->done_cv.wait_for(lock, std::chrono::milliseconds(timeout_ms), [&] { return !e->done.empty(); });
  size_t n = 0;
  while (n < cap && !e->done.empty()) {
    Done* d = e->done.front();
    e->done.pop_front();
    rv9_completion& c = out[n++];
    memset(&c, 0, sizeof c);
    c.stream = d->stream_id;
    c.tag = d->tag;
    c.status = d->status;
    c.n_frames = d->status == RV9_OK ? d->n_frames : 0;
    c.submit_ms = d->submit_ms;
    c.latency_ms = d->latency_ms;
    for (uint32_t i = 0; i < c.n_frames; ++i) c.frames[i] = d->frames[i];
    c.handle = d;
    e->polled.insert(d);
  }
  return n;
}

void rv9_completion_release(rv9_engine* e, rv9_completion* c) {
  if (!e || !c || !c->handle) return;
  Done* d = static_cast<Done*>(c->handle);
  std::shared_ptr<Stream> keep;
  {
    std::lock_guard<std::mutex> lock(e->mu);
    if (!e->polled.erase(d)) return;  // not a live handle of this engine
    keep = e->release_locked(d);
  }
  c->handle = nullptr;
  // `keep` may be the last reference to a closed stream: freed here.
}

void rv9_engine_get_stats(rv9_engine* e, rv9_engine_stats* out) {
  if (!e || !out) return;
  std::lock_guard<std::mutex> lock(e->mu);
  memset(out, 0, sizeof *out);
  for (auto& kv : e->streams) {
    if (kv.second->state == PENDING)
      ++out->streams_pending;
    else if (kv.second->state != CLOSED)
      ++out->streams_open;
  }
  out->requests_submitted = e->n_submitted;
  out->requests_completed = e->n_completed;
  out->frames_decoded = e->n_frames;
  out->reserved_bytes = e->reserved;
  out->budget_bytes = e->budget;
  for (auto& G : e->groups) {
    out->batched_steps += G->steps;
    out->batched_frames += G->frames;
  }
  out->device_parse_batches = e->dp_batches;
  out->device_parsed_frames = e->dp_frames;
  out->device_parse_wait_us = e->dp_wait_us;
  out->device_parse_batch_us = e->dp_batch_us;
}

rv9_status rv9_engine_set_device_parse(rv9_engine* e, int on, uint32_t window, uint32_t max_batches) {
  if (!e) return RV9_INVALID_INPUT;
  if (!e->groups.empty()) return RV9_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(e->mu);
  if (!on) {
    e->dp_window = 0;
    e->dp_max = 0;
    return RV9_OK;
  }
  e->dp_window = window ? std::min<uint32_t>(window, 64) : 8;
  e->dp_max = max_batches ? max_batches : kDefaultBatches;
  // A worker waiting for its batch sleeps: one more worker per batch keeps
  // the host's parsing rate while batches are on the device.
  while (e->n_extra_workers < e->dp_max) {
    e->workers.emplace_back([e] { e->worker_loop(); });
    ++e->n_extra_workers;
  }
  e->work_cv.notify_all();
  return RV9_OK;
}

}  // extern "C"

// Serving across the GPUs of one node: a serving engine (rv9_engine) per
// device, each stream placed whole on one of them.
//
// A stream's frames chain through its reference slots and its parse state is
// sequential, so a stream is never split across devices; streams share
// nothing, so there is no exchange between devices either (no collective, no
// peer access). A new stream goes to the device with the fewest reserved
// bytes among those whose HBM budget can take its reservation, and to the
// least loaded device when none can (it then waits there, pending, until
// streams on that device close). Requests and completions pass through to the
// stream's engine; completions of all engines come back through one poll.
#include <string.h>

#include <chrono>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "../../../include/rv9_server.h"

namespace {

struct Placed {
  size_t dev = 0;       // index into the cluster's engines
  int64_t local = 0;    // the stream's id in that engine
  uint64_t bytes = 0;   // its reservation
};

}  // namespace

struct rv9_cluster {
  std::vector<rv9_engine*> engines;
  std::vector<int> devices;
  std::vector<uint64_t> load;  // reserved bytes of the open streams, per engine
  uint64_t budget = 0;
  std::mutex mu;
  std::map<int64_t, Placed> streams;                    // cluster id -> placement
  std::map<std::pair<size_t, int64_t>, int64_t> back;   // (engine, local id) -> cluster id
  std::map<void*, size_t> handles;                      // polled completion -> engine
  int64_t next_id = 1;
  size_t cursor = 0;  // the engine polled first, round-robin
};

extern "C" {

int rv9_place_least_loaded(const uint64_t* load, const uint64_t* budget, size_t n, uint64_t need) {
  if (!load || !budget) return -1;
  int best = -1, any = -1;
  for (size_t i = 0; i < n; ++i) {
    if (need > budget[i]) continue;  // could never be admitted there
    if (any < 0 || load[i] < load[(size_t)any]) any = (int)i;
    if (load[i] + need <= budget[i] && (best < 0 || load[i] < load[(size_t)best])) best = (int)i;
  }
  // The least loaded device with room now; else the least loaded one that
  // could ever take the stream (it waits there, pending); else none.
  return best >= 0 ? best : any;
}

rv9_cluster* rv9_cluster_create(const int* devices, size_t n, uint64_t hbm_budget_per_device,
                                uint32_t workers_per_device) {
  if (!devices || n == 0) return nullptr;
  rv9_cluster* c = new rv9_cluster;
  c->budget = hbm_budget_per_device;
  for (size_t i = 0; i < n; ++i) {
    rv9_engine* e = rv9_engine_create(devices[i], hbm_budget_per_device, workers_per_device);
    if (!e) {
      for (rv9_engine* x : c->engines) rv9_engine_free(x);
      delete c;
      return nullptr;  // rv9_last_global_error says why
    }
    c->engines.push_back(e);
    c->devices.push_back(devices[i]);
    c->load.push_back(0);
  }
  return c;
}

rv9_status rv9_cluster_set_device_parse(rv9_cluster* c, int on, uint32_t window, uint32_t max_batches) {
  if (!c) return RV9_INVALID_INPUT;
  std::lock_guard<std::mutex> lock(c->mu);
  for (rv9_engine* e : c->engines) {
    rv9_status st = rv9_engine_set_device_parse(e, on, window, max_batches);
    if (st != RV9_OK) return st;
  }
  return RV9_OK;
}

void rv9_cluster_free(rv9_cluster* c) {
  if (!c) return;
  for (rv9_engine* e : c->engines) rv9_engine_free(e);
  delete c;
}

rv9_status rv9_cluster_stream_open(rv9_cluster* c, const rv9_stream_spec* spec, int64_t* id, int* device) {
  if (!c || !spec || !id) return RV9_INVALID_INPUT;
  *id = 0;
  std::lock_guard<std::mutex> lock(c->mu);
  // The engines share their settings: the first one's reservation holds.
  const uint64_t need = rv9_engine_stream_reservation(c->engines[0], spec);
  std::vector<uint64_t> budgets(c->engines.size(), c->budget);
  const int d = rv9_place_least_loaded(c->load.data(), budgets.data(), c->engines.size(), need);
  if (d < 0) return RV9_UNSUPPORTED;
  int64_t local = 0;
  rv9_status st = rv9_stream_open(c->engines[(size_t)d], spec, &local);
  if (st != RV9_OK) return st;
  const int64_t cid = c->next_id++;
  c->streams[cid] = Placed{(size_t)d, local, need};
  c->back[{(size_t)d, local}] = cid;
  c->load[(size_t)d] += need;
  *id = cid;
  if (device) *device = c->devices[(size_t)d];
  return RV9_OK;
}

rv9_status rv9_cluster_stream_close(rv9_cluster* c, int64_t id) {
  if (!c) return RV9_INVALID_INPUT;
  std::lock_guard<std::mutex> lock(c->mu);
  auto it = c->streams.find(id);
  if (it == c->streams.end()) return RV9_INVALID_INPUT;
  const Placed p = it->second;
  rv9_status st = rv9_stream_close(c->engines[p.dev], p.local);
  if (st != RV9_OK) return st;
  // The device's load drops at once: the engine admits its pending streams as
  // this one drains, and new streams are placed against what stays open.
  c->load[p.dev] -= p.bytes;
  c->streams.erase(it);
  return RV9_OK;
}

rv9_status rv9_cluster_submit(rv9_cluster* c, int64_t id, const uint8_t* packet, size_t len, uint64_t tag) {
  if (!c) return RV9_INVALID_INPUT;
  Placed p;
  {
    std::lock_guard<std::mutex> lock(c->mu);
    auto it = c->streams.find(id);
    if (it == c->streams.end()) return RV9_INVALID_INPUT;
    p = it->second;
  }
  return rv9_submit(c->engines[p.dev], p.local, packet, len, tag);
}

size_t rv9_cluster_poll(rv9_cluster* c, rv9_completion* out, size_t cap, int timeout_ms) {
  if (!c || !out || cap == 0) return 0;
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms > 0 ? timeout_ms : 0);
  const size_t n_eng = c->engines.size();
  for (;;) {
    size_t n = 0;
    size_t first;
    {
      std::lock_guard<std::mutex> lock(c->mu);
      first = c->cursor;
      c->cursor = (c->cursor + 1) % n_eng;
    }
    for (size_t k = 0; k < n_eng && n < cap; ++k) {
      const size_t e = (first + k) % n_eng;
      const size_t got = rv9_poll(c->engines[e], out + n, cap - n, 0);
      std::lock_guard<std::mutex> lock(c->mu);
      for (size_t i = n; i < n + got; ++i) {
        auto b = c->back.find({e, out[i].stream});
        out[i].stream = b != c->back.end() ? b->second : 0;
        c->handles[out[i].handle] = e;
      }
      n += got;
    }
    if (n > 0 || std::chrono::steady_clock::now() >= deadline) return n;
    std::this_thread::sleep_for(std::chrono::microseconds(200));
  }
}

void rv9_cluster_completion_release(rv9_cluster* c, rv9_completion* comp) {
  if (!c || !comp || !comp->handle) return;
  size_t e;
  {
    std::lock_guard<std::mutex> lock(c->mu);
    auto it = c->handles.find(comp->handle);
    if (it == c->handles.end()) return;
    e = it->second;
    c->handles.erase(it);
  }
  rv9_completion_release(c->engines[e], comp);
}

void rv9_cluster_get_stats(rv9_cluster* c, int device_index, rv9_engine_stats* out) {
  if (!out) return;
  memset(out, 0, sizeof *out);
  if (!c || device_index < 0 || (size_t)device_index >= c->engines.size()) return;
  rv9_engine_get_stats(c->engines[(size_t)device_index], out);
}

}  // extern "C"

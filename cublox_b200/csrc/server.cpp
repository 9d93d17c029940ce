// Served integration: a request loop over many resident maps
// (include/cublox_b200.h, cublox_server_*).
//
// Callers (one per robot, any thread) submit scans and sphere fetches; the
// call copies the request and returns.  One worker thread forms "ticks":
// every map whose oldest pending request is a scan contributes that scan,
// up to the tick's point budget, and the tick is integrated by one batched
// launch sequence (cublox_batch_update, then each map's recenter).  A tick
// is enqueued while the previous one still runs on the device, so requests
// that arrive meanwhile join the next launch instead of waiting for a queue
// to drain (continuous batching); per-map order is kept because every map
// lives on the one stream and takes at most one scan per tick.  A second
// thread waits on each tick's event and stamps its requests done.
//
// Device memory is admitted against a budget: a map's voxel buffers (12 B a
// voxel) are allocated when its first request is served; if they do not fit
// beside the maps already resident, the least recently used maps with no
// work in the current tick are evicted (stored log-odds copied to host
// memory, buffers freed) and brought back, bit for bit, when their next
// request is served.  A map larger than the whole budget fails its requests.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/cublox_b200.h"
#include "grid_internal.hpp"

using cublox_b200::detail::fail;
using Clock = std::chrono::steady_clock;

namespace {

enum ReqKind { kScan = 0, kFetch = 1 };

struct Request {
  int64_t id = 0;
  int kind = kScan;
  int map = 0;
  // scan
  std::vector<float> pts;  // x0 y0 z0 x1 ... (when no pinned block was free)
  float *pin = nullptr;    // or the same in a pinned block of the server's pool
  int pin_cls = -1;
  size_t pin_floats = 0;
  float sensor[3] = {0, 0, 0};
  int recenter = 0;
  // fetch
  std::vector<float> centers;
  float radius = 0.0f;
  int filter = CUBLOX_FILTER_ALL;
  int max_results = 0;
  std::vector<int64_t> offsets;
  std::vector<float> fpos;
  std::vector<uint8_t> fstate;
  // progress
  int state = CUBLOX_REQ_QUEUED;
  int error = CUBLOX_OK;
  std::string message;
  Clock::time_point t_submit, t_start, t_done;
};

struct MapState {
  int half[3];
  float res;
  int ctr, has_thr;
  double thr;
  float origin[3];
  float max_range;
  float lo[6];
  bool has_lo = false;
  cublox_grid *g = nullptr;  // created at first admission
  bool resident = false;
  // stored log-odds while evicted (the grid's own layout): a pinned buffer
  // allocated when the maps outgrow the budget (cublox_server_add_map) or at
  // the map's first eviction, and kept; pageable memory if pinning failed
  float *snap_pinned = nullptr;
  std::vector<float> snap_pageable;
  const float *snapshot() const {
    return snap_pinned ? snap_pinned : (snap_pageable.empty() ? nullptr : snap_pageable.data());
  }
  size_t vox_bytes = 0;  // device bytes of the map's arrays
  int64_t nalloc = 0;    // voxels each array holds (padding included)
  int64_t voxels = 0;
  uint64_t last_use = 0;
  std::deque<Request *> queue;  // pending requests, arrival order
  std::atomic<bool> fetching{false};  // a fetch of this map is in flight
};

struct FetchJob {
  Request *r;
  cudaEvent_t after;  // the map's earlier work, on the server stream
};

struct Tick {
  cudaEvent_t done = nullptr;
  std::vector<Request *> reqs;
};

}  // namespace

// Pinned host blocks for scan points, reused by size class (64 KiB << c).
// A scan submitted into one is copied to the device by DMA straight from
// it, so the worker thread copies nothing for a one-scan tick.  Blocks are
// carved from one pinned arena allocated when the server is created: a
// class with no free block takes the next piece of the arena, and a block
// returns to its class when its request ends (its tick's copy has run by
// then).  Submitting never allocates; a scan that finds no room stays in
// pageable memory and the batch stages it.
struct PinnedPool {
  static constexpr size_t kMinBytes = size_t(64) << 10;
  std::mutex mu;
  std::vector<std::vector<float *>> free_by_class;
  char *arena = nullptr;
  size_t arena_bytes = 0, carved = 0;

  // Allocates the arena with `device` current (the calling thread's own
  // current device is put back afterwards).
  int init(size_t bytes, int device) {
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      prev = -1;
    }
    const bool switched = prev >= 0 && prev != device && cudaSetDevice(device) == cudaSuccess;
    void *p = nullptr;
    const cudaError_t e = bytes ? cublox_b200::detail::hmalloc(&p, bytes) : cudaSuccess;
    if (switched) cudaSetDevice(prev);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(CUBLOX_ERR_NOMEM, "server: pinned arena allocation failed");
    }
    arena = static_cast<char *>(p);
    arena_bytes = bytes;
    return CUBLOX_OK;
  }
  float *take(size_t bytes, int *cls) {
    int c = 0;
    while ((kMinBytes << c) < bytes) ++c;
    std::lock_guard<std::mutex> lk(mu);
    if (c < static_cast<int>(free_by_class.size()) && !free_by_class[c].empty()) {
      float *p = free_by_class[c].back();
      free_by_class[c].pop_back();
      *cls = c;
      return p;
    }
    const size_t sz = kMinBytes << c;
    if (carved + sz > arena_bytes) return nullptr;
    float *p = reinterpret_cast<float *>(arena + carved);
    carved += sz;
    *cls = c;
    return p;
  }
  void give(float *p, int c) {
    std::lock_guard<std::mutex> lk(mu);
    if (static_cast<int>(free_by_class.size()) <= c) free_by_class.resize(c + 1);
    free_by_class[c].push_back(p);
  }
  void release_all() {
    cublox_b200::detail::hfree(arena);
    arena = nullptr;
    arena_bytes = carved = 0;
    free_by_class.clear();
  }
};

struct cublox_server {
  cublox_server_config cfg{};
  PinnedPool pinned;  // scan points
  cublox_b200::FetchScratch fscratch;  // shared by fetches (one at a time)
  int reserved_maps = 0;  // maps the batch's item buffers are sized for
  cublox_batch *batch = nullptr;
  cudaStream_t stream = nullptr;
  int device = 0;
  std::mutex mu;
  std::condition_variable cv_work;      // new requests, or stop
  std::condition_variable cv_done;      // a request finished
  std::condition_variable cv_inflight;  // a tick left the device
  std::unordered_map<int64_t, std::unique_ptr<Request>> reqs;
  std::vector<std::unique_ptr<MapState>> maps;  // reserved: never reallocated
  // voxel buffers of evicted maps, kept for the next map of the same size
  // (worker thread only)
  std::vector<cublox_b200::detail::VoxelBuffers> spare;
  std::atomic<int> n_maps{0};                    // maps[0, n_maps) are published
  std::deque<Tick> inflight;
  std::deque<FetchJob> fetch_jobs;
  std::condition_variable cv_fetch;  // a fetch job, or stop
  cudaStream_t fstream = nullptr;    // fetches, ordered after their map's work
  std::vector<cudaEvent_t> free_events;
  int64_t next_id = 1;
  int64_t pending = 0;  // requests not yet done
  uint64_t clock = 0;   // use counter for LRU
  cublox_server_stats stats{};
  bool stop = false;
  std::thread worker, completer, fetcher;
  int rr = 0;  // round-robin start of tick formation
};

namespace {

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

const float *pts_data(const Request *r) { return r->pin ? r->pin : r->pts.data(); }
size_t pts_floats(const Request *r) { return r->pin ? r->pin_floats : r->pts.size(); }

void finish(cublox_server *s, Request *r, int error, const std::string &msg) {
  if (r->pin) {
    s->pinned.give(r->pin, r->pin_cls);
    r->pin = nullptr;
    r->pin_floats = 0;
  }
  r->t_done = Clock::now();
  r->error = error;
  r->message = msg;
  r->state = error ? CUBLOX_REQ_FAILED : CUBLOX_REQ_DONE;
  --s->pending;
}

// Fetch scratch sized for cfg's fetch limits (the query block, 13 B a
// sample).
size_t fetch_scratch_bytes(const cublox_server_config &cfg) {
  const size_t nq = static_cast<size_t>(cfg.max_fetch_centres);
  const size_t nu = nq + 32 * 160;
  return 4 * nq * 12 + 4 * nu * 40 + 13 * static_cast<size_t>(cfg.max_fetch_samples) +
         (size_t(16) << 10);
}

size_t scratch_bytes(const cublox_server_config &cfg) {
  // batch point buffer at the tick budget, descriptors, fetch scratch
  return 12 * static_cast<size_t>(cfg.max_tick_points) + (1u << 20) + fetch_scratch_bytes(cfg);
}

size_t scratch_bytes(cublox_server *s) { return scratch_bytes(s->cfg); }

void fill_defaults(cublox_server_config *cfg) {
  if (cfg->max_tick_points <= 0) cfg->max_tick_points = 1 << 20;
  if (cfg->pinned_pool_bytes == 0) cfg->pinned_pool_bytes = size_t(256) << 20;
  if (cfg->max_fetch_centres <= 0) cfg->max_fetch_centres = 1024;
  if (cfg->max_fetch_samples <= 0) cfg->max_fetch_samples = int64_t(1) << 22;
}

constexpr int kMaxMaps = 4096;
constexpr double kSwapAgeMs = 25.0;  // a request this old may force a second swap in a tick

size_t used_bytes(cublox_server *s) {
  size_t b = scratch_bytes(s);
  const int nm = s->n_maps.load();
  for (int j = 0; j < nm; ++j)
    if (s->maps[j]->resident) b += cublox_b200::detail::device_bytes(s->maps[j]->g);
  for (const auto &v : s->spare) b += v.bytes();
  return b;
}

// Hand map m a spare set of voxel buffers of its size, if there is one: its
// stored log-odds are copied in on the server stream (no allocation, no
// sync).  Returns 1 if it did, 0 if no spare fits, <0 on error.
int take_spare(cublox_server *s, MapState &m) {
  for (size_t i = 0; i < s->spare.size(); ++i) {
    if (s->spare[i].nalloc != m.nalloc) continue;
    const int rc = cublox_b200::detail::attach_voxels(m.g, &s->spare[i], m.snapshot());
    if (rc) return rc;
    s->spare.erase(s->spare.begin() + static_cast<std::ptrdiff_t>(i));
    return 1;
  }
  return 0;
}

// Free spare buffer sets (largest first) until `need` more bytes fit the
// budget.  cudaFree waits for the device: only a map's first admission, or
// one whose size no spare has, comes here.
void free_spares(cublox_server *s, size_t need) {
  while (!s->spare.empty() && used_bytes(s) + need > s->cfg.hbm_budget_bytes) {
    size_t big = 0;
    for (size_t i = 1; i < s->spare.size(); ++i)
      if (s->spare[i].nalloc > s->spare[big].nalloc) big = i;
    auto &v = s->spare[big];
    cublox_b200::detail::dfree(v.occ);
    cublox_b200::detail::dfree(v.cnt);
    cublox_b200::detail::dfree(v.hit);
    s->spare.erase(s->spare.begin() + static_cast<std::ptrdiff_t>(big));
  }
}

// Make map `mi` resident, evicting least recently used maps not in `busy`
// (the maps already admitted for the launch being formed).  *later is set
// when the map fits the budget but not beside the busy maps: the request
// waits for a later tick.  Runs on the worker thread, without the lock.
int admit(cublox_server *s, int mi, const std::vector<char> &busy, bool *later) {
  *later = false;
  MapState &m = *s->maps[mi];
  m.last_use = ++s->clock;
  if (m.resident) return CUBLOX_OK;
  size_t need = m.vox_bytes;
  if (need + scratch_bytes(s) > s->cfg.hbm_budget_bytes)
    return fail(CUBLOX_ERR_NOMEM, "server: map needs " + std::to_string(need) +
                                      " bytes, more than the budget allows");
  // First give back the per-call scratch (fetch outputs) of idle maps that
  // hold some (release_scratch waits for the server stream).
  if (used_bytes(s) + need > s->cfg.hbm_budget_bytes)
    for (int j = 0; j < static_cast<int>(busy.size()); ++j) {
      MapState &o = *s->maps[j];
      if (j != mi && o.resident && !busy[j] && !o.fetching.load() &&
          cublox_b200::detail::device_bytes(o.g) > o.vox_bytes)
        cublox_b200::detail::release_scratch(o.g);
    }
  // A map that was resident before takes a spare set of its size, if any
  // (an eviction earlier left one), without allocating.  Otherwise maps are
  // evicted (their buffers become spare sets) until one of them fits, or
  // until freeing spare sets of other sizes makes room.
  for (;;) {
    if (m.g) {
      const int rc = take_spare(s, m);
      if (rc < 0) return rc;
      if (rc == 1) {
        need = 0;
        break;
      }
    }
    size_t spare = 0;
    for (const auto &v : s->spare) spare += v.bytes();
    if (used_bytes(s) - spare + need <= s->cfg.hbm_budget_bytes) break;
    // the victim: a resident map outside this tick, preferring maps with no
    // queued request (their next use is furthest off), then maps of this
    // map's size (their buffers can be handed over), least recently used
    // first
    int victim = -1;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      bool victim_idle = false, victim_same = false;
      for (int j = 0; j < static_cast<int>(busy.size()); ++j) {
        MapState &o = *s->maps[j];
        if (j == mi || !o.resident || busy[j] || o.fetching.load()) continue;
        const bool idle = o.queue.empty(), same = o.nalloc == m.nalloc;
        const bool better =
            victim < 0 || (idle && !victim_idle) ||
            (idle == victim_idle && same && !victim_same) ||
            (idle == victim_idle && same == victim_same && o.last_use < s->maps[victim]->last_use);
        if (better) {
          victim = j;
          victim_idle = idle;
          victim_same = same;
        }
      }
    }
    if (victim < 0) {
      *later = true;
      return fail(CUBLOX_ERR_NOMEM, "server: no map can be evicted");
    }
    MapState &v = *s->maps[victim];
    const size_t n = static_cast<size_t>(v.nalloc);
    if (!v.snap_pinned && v.snap_pageable.empty() &&
        cublox_b200::detail::hmalloc(&v.snap_pinned, n * sizeof(float)) != cudaSuccess) {
      cudaGetLastError();
      v.snap_pinned = nullptr;
      v.snap_pageable.resize(n);
    }
    // The stored log-odds go to the snapshot on the server stream, ordered
    // before any later use of the buffers; the buffers become a spare set.
    cublox_b200::detail::VoxelBuffers vb;
    int rc = cublox_b200::detail::detach_voxels(
        v.g, v.snap_pinned ? v.snap_pinned : v.snap_pageable.data(), &vb);
    if (rc) return rc;
    s->spare.push_back(vb);
    v.resident = false;
    std::lock_guard<std::mutex> lk(s->mu);
    ++s->stats.evictions;
  }
  int rc;
  if (!m.g) {
    free_spares(s, need);
    rc = cublox_grid_create(m.half, m.res, m.ctr, m.has_thr, m.thr, m.origin, s->stream, &m.g);
    if (rc) return rc;
    cublox_grid_set_max_range(m.g, m.max_range);
    if (m.has_lo)
      cublox_grid_set_log_odds(m.g, m.lo[0], m.lo[1], m.lo[2], m.lo[3], m.lo[4], m.lo[5]);
  } else if (need) {
    free_spares(s, need);
    rc = cublox_b200::detail::acquire_device(m.g, m.snapshot());
    if (rc) return rc;
  }
  m.resident = true;
  const size_t used = used_bytes(s);
  std::lock_guard<std::mutex> lk(s->mu);
  ++s->stats.admissions;
  s->stats.resident_bytes = used;
  s->stats.peak_resident_bytes = std::max(s->stats.peak_resident_bytes, used);
  return CUBLOX_OK;
}

// Tick and fetch-order events (the completer thread polls them, see
// completer_loop).
constexpr unsigned kEventFlags = cudaEventDisableTiming;
constexpr int kEventPool = 64;  // created with the server

// Caller holds the lock.
cudaEvent_t take_event(cublox_server *s) {
  if (!s->free_events.empty()) {
    cudaEvent_t e = s->free_events.back();
    s->free_events.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreateWithFlags(&e, kEventFlags);
  return e;
}

// Put a request back at the head of its map's queue.
void defer(cublox_server *s, Request *r) {
  std::lock_guard<std::mutex> lk(s->mu);
  r->state = CUBLOX_REQ_QUEUED;
  s->maps[r->map]->queue.push_front(r);
}

// Fetches run on their own thread and stream: the job waits (on the device)
// for the work queued on its map before it, and the map takes no new tick
// until the fetch is done, so later scans cannot overtake it.
void fetcher_loop(cublox_server *s) {
  cudaSetDevice(s->device);
  for (;;) {
    FetchJob job;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_fetch.wait(lk, [&] { return s->stop || !s->fetch_jobs.empty(); });
      if (s->fetch_jobs.empty()) return;
      job = s->fetch_jobs.front();
      s->fetch_jobs.pop_front();
    }
    Request *r = job.r;
    MapState &m = *s->maps[r->map];
    int rc = CUBLOX_OK;
    if (cudaStreamWaitEvent(s->fstream, job.after, 0) != cudaSuccess) {
      cudaGetLastError();
      rc = fail(CUBLOX_ERR_CUDA, "server: fetch ordering failed");
    }
    if (!rc)
      rc = cublox_b200::detail::fetch_into(m.g, s->fstream, r->centers.data(),
                                           static_cast<int>(r->centers.size() / 3), r->radius,
                                           r->filter, r->max_results, r->offsets, r->fpos,
                                           r->fstate, &s->fscratch);
    const std::string msg = rc ? cublox_last_error() : "";
    std::lock_guard<std::mutex> lk(s->mu);
    ++s->stats.fetches;
    finish(s, r, rc, msg);
    s->free_events.push_back(job.after);
    m.fetching = false;
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
}

void worker_loop(cublox_server *s) {
  cudaSetDevice(s->device);
  const int max_inflight = s->cfg.max_inflight_ticks > 0 ? s->cfg.max_inflight_ticks : 2;
  for (;;) {
    std::vector<Request *> scans, fetches;
    int nm = 0;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      for (;;) {
        if (s->stop) return;
        // heads of the per-map queues.  Under memory pressure a map that is
        // not resident costs a swap (an eviction and a restore): a tick
        // takes at most one such map, unless a map's oldest request has
        // waited kSwapAgeMs, so resident maps' backlogs are served between
        // swaps.
        nm = s->n_maps.load();
        int64_t pts = 0;
        const auto now = Clock::now();
        size_t room = s->cfg.hbm_budget_bytes - std::min(s->cfg.hbm_budget_bytes, used_bytes(s));
        bool swapped = false;
        for (int k = 0; k < nm; ++k) {
          const int mi = (s->rr + k) % nm;
          MapState &m = *s->maps[mi];
          if (m.queue.empty() || m.fetching) continue;
          Request *r = m.queue.front();
          if (!m.resident) {
            if (m.vox_bytes <= room) {
              room -= m.vox_bytes;  // fits without an eviction
            } else if (swapped && ms_between(r->t_submit, now) < kSwapAgeMs) {
              continue;
            } else {
              swapped = true;
            }
          }
          if (r->kind == kFetch) {
            fetches.push_back(r);
            m.queue.pop_front();
            m.fetching = true;
            continue;
          }
          const int64_t n = static_cast<int64_t>(pts_floats(r) / 3);
          if (!scans.empty() && (pts + n > s->cfg.max_tick_points ||
                                 (s->cfg.max_tick_maps > 0 &&
                                  static_cast<int>(scans.size()) >= s->cfg.max_tick_maps)))
            continue;
          scans.push_back(r);
          m.queue.pop_front();
          pts += n;
        }
        if (nm) s->rr = (s->rr + 1) % nm;
        if (!scans.empty() || !fetches.empty()) break;
        s->cv_work.wait(lk);
      }
      // bound the launches queued on the device
      s->cv_inflight.wait(lk, [&] {
        return s->stop || static_cast<int>(s->inflight.size()) < max_inflight;
      });
      if (s->stop) return;
      const auto now = Clock::now();
      for (Request *r : scans) r->state = CUBLOX_REQ_RUNNING, r->t_start = now;
      for (Request *r : fetches) r->state = CUBLOX_REQ_RUNNING, r->t_start = now;
    }
    // The batch's work-item buffers, sized once for every map known so far
    // (a tick never holds more), so that ticks allocate nothing.
    if (nm > s->reserved_maps) {
      int64_t vox = 0;
      for (int j = 0; j < nm; ++j) vox += s->maps[j]->voxels;
      if (cublox_batch_reserve_maps(s->batch, s->cfg.max_tick_points, nm, vox) == CUBLOX_OK)
        s->reserved_maps = nm;
    }
    // A map gives a tick one request, its oldest: a scan or a fetch.
    // scans: admit, concatenate, one batched update, recenters
    std::vector<char> busy(static_cast<size_t>(nm), 0);
    std::vector<Request *> ok;
    for (Request *r : scans) {
      bool later = false;
      const int rc = admit(s, r->map, busy, &later);
      if (later) {
        defer(s, r);
        continue;
      }
      busy[r->map] = 1;
      if (rc) {
        const std::string msg = cublox_last_error();
        std::lock_guard<std::mutex> lk(s->mu);
        finish(s, r, rc, msg);
        s->cv_done.notify_all();
        continue;
      }
      ok.push_back(r);
    }
    if (!ok.empty()) {
      std::vector<cublox_grid *> grids;
      std::vector<int64_t> offsets(1, 0);
      std::vector<float> sensors;
      size_t floats = 0;
      for (Request *r : ok) floats += pts_floats(r);
      // One scan (the usual tick) is passed in place — the batch's walk reads
      // it from its pinned block, which goes back to the pool only when the
      // tick has completed; several are concatenated into an uninitialised
      // buffer, which the batch stages in its own pinned buffer.
      std::unique_ptr<float[]> joined;
      const float *xyz = ok.size() == 1 ? pts_data(ok[0]) : nullptr;
      if (!xyz) {
        joined.reset(new float[floats > 0 ? floats : 1]);
        xyz = joined.get();
      }
      size_t at = 0;
      for (Request *r : ok) {
        grids.push_back(s->maps[r->map]->g);
        if (joined)
          std::memcpy(joined.get() + at, pts_data(r), pts_floats(r) * sizeof(float));
        at += pts_floats(r);
        offsets.push_back(static_cast<int64_t>(at / 3));
        sensors.insert(sensors.end(), r->sensor, r->sensor + 3);
      }
      int rc = cublox_batch_update(s->batch, static_cast<int>(ok.size()), grids.data(), xyz,
                                   offsets.data(), sensors.data());
      for (size_t i = 0; !rc && i < ok.size(); ++i) {
        if (!ok[i]->recenter) continue;
        int action = 0;
        rc = cublox_grid_recenter(grids[i], ok[i]->sensor, &action);
      }
      cudaEvent_t ev = nullptr;
      if (!rc) {
        std::lock_guard<std::mutex> lk(s->mu);
        ev = take_event(s);
      }
      if (!rc && cudaEventRecord(ev, s->stream) != cudaSuccess) {
        cudaGetLastError();
        rc = fail(CUBLOX_ERR_CUDA, "server: event record failed");
      }
      std::string fail_msg;
      if (rc) {
        // the failed tick may have queued a copy out of its requests' pinned
        // blocks: let it run before the blocks go back to the pool
        fail_msg = cublox_last_error();
        cudaStreamSynchronize(s->stream);
        cudaGetLastError();
      }
      std::lock_guard<std::mutex> lk(s->mu);
      ++s->stats.ticks;
      s->stats.scans += static_cast<int64_t>(ok.size());
      s->stats.points += offsets.back();
      if (rc) {
        for (Request *r : ok) finish(s, r, rc, fail_msg);
        s->cv_done.notify_all();
      } else {
        s->inflight.push_back(Tick{ev, ok});
        s->cv_work.notify_all();  // wakes the completer
      }
    }
    // fetches: admitted beside the tick's maps, handed to the fetch thread
    for (Request *r : fetches) {
      MapState &m = *s->maps[r->map];
      bool later = false;
      int rc = admit(s, r->map, busy, &later);
      if (later) {
        std::lock_guard<std::mutex> lk(s->mu);
        r->state = CUBLOX_REQ_QUEUED;
        m.queue.push_front(r);
        m.fetching = false;
        continue;
      }
      busy[r->map] = 1;
      cudaEvent_t ev = nullptr;
      if (!rc) {
        std::lock_guard<std::mutex> lk(s->mu);
        ev = take_event(s);
      }
      if (!rc && cudaEventRecord(ev, s->stream) != cudaSuccess) {
        cudaGetLastError();
        rc = fail(CUBLOX_ERR_CUDA, "server: event record failed");
      }
      std::lock_guard<std::mutex> lk(s->mu);
      if (rc) {
        if (ev) s->free_events.push_back(ev);
        finish(s, r, rc, cublox_last_error());
        m.fetching = false;
        s->cv_done.notify_all();
        continue;
      }
      s->fetch_jobs.push_back(FetchJob{r, ev});
      s->cv_fetch.notify_one();
    }
  }
}

void completer_loop(cublox_server *s) {
  cudaSetDevice(s->device);
  for (;;) {
    cudaEvent_t ev;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] { return s->stop || !s->inflight.empty(); });
      if (s->inflight.empty()) return;  // stop, nothing in flight
      ev = s->inflight.front().done;
    }
    // Poll, yielding the core between queries: a tick takes a fraction of a
    // millisecond, and a blocking wait's wake-up would add more than that to
    // every request's latency.
    cudaError_t e;
    while ((e = cudaEventQuery(ev)) == cudaErrorNotReady) std::this_thread::yield();
    std::lock_guard<std::mutex> lk(s->mu);
    Tick t = std::move(s->inflight.front());
    s->inflight.pop_front();
    for (Request *r : t.reqs)
      finish(s, r, e == cudaSuccess ? CUBLOX_OK : CUBLOX_ERR_CUDA,
             e == cudaSuccess ? "" : cudaGetErrorString(e));
    s->free_events.push_back(ev);
    s->cv_done.notify_all();
    s->cv_inflight.notify_all();
  }
}

Request *find(cublox_server *s, int64_t id) {
  auto it = s->reqs.find(id);
  return it == s->reqs.end() ? nullptr : it->second.get();
}

}  // namespace

extern "C" {

int cublox_server_create(const cublox_server_config *cfg, cublox_server **out) {
  if (!cfg || !out) return fail(CUBLOX_ERR_INVALID, "server_create: null argument");
  *out = nullptr;
  auto s = std::make_unique<cublox_server>();
  s->cfg = *cfg;
  s->maps.reserve(kMaxMaps);
  fill_defaults(&s->cfg);
  if (s->cfg.hbm_budget_bytes < scratch_bytes(s.get()))
    return fail(CUBLOX_ERR_INVALID, "server_create: budget below the tick and fetch scratch (" +
                                        std::to_string(scratch_bytes(s.get())) + " bytes)");
  cudaGetDevice(&s->device);
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->fstream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    if (s->stream) cudaStreamDestroy(s->stream);
    return fail(CUBLOX_ERR_CUDA, "server_create: stream creation failed");
  }
  int rc = cublox_batch_create(s->stream, &s->batch);
  if (rc) {
    cudaStreamDestroy(s->stream);
    cudaStreamDestroy(s->fstream);
    return rc;
  }
  cublox_batch_set_option(s->batch, CUBLOX_BATCH_OPT_GRAPHS, s->cfg.graphs ? 1 : 0);
  rc = cublox_batch_reserve(s->batch, s->cfg.max_tick_points, 64);
  if (!rc) rc = s->pinned.init(s->cfg.pinned_pool_bytes, s->device);
  if (!rc)
    rc = cublox_b200::detail::reserve_fetch(&s->fscratch, s->cfg.max_fetch_centres,
                                            s->cfg.max_fetch_samples, s->fstream);
  if (rc) {
    const std::string msg = cublox_last_error();
    cublox_b200::detail::free_fetch(&s->fscratch);
    s->pinned.release_all();
    cublox_batch_destroy(s->batch);
    cudaStreamDestroy(s->stream);
    cudaStreamDestroy(s->fstream);
    return fail(rc, msg);
  }
  for (int i = 0; i < kEventPool; ++i) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, kEventFlags) == cudaSuccess) s->free_events.push_back(e);
  }
  cudaGetLastError();
  cublox_server *raw = s.release();
  raw->worker = std::thread(worker_loop, raw);
  raw->completer = std::thread(completer_loop, raw);
  raw->fetcher = std::thread(fetcher_loop, raw);
  *out = raw;
  return CUBLOX_OK;
}

int cublox_server_destroy(cublox_server *s) {
  if (!s) return CUBLOX_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  s->cv_inflight.notify_all();
  s->cv_fetch.notify_all();
  if (s->worker.joinable()) s->worker.join();
  if (s->fetcher.joinable()) s->fetcher.join();
  cudaStreamSynchronize(s->stream);
  if (s->completer.joinable()) s->completer.join();
  for (Tick &t : s->inflight) s->free_events.push_back(t.done);
  for (cudaEvent_t e : s->free_events)
    if (e) cudaEventDestroy(e);
  for (auto &m : s->maps) {
    if (m->g) cublox_grid_destroy(m->g);
    cublox_b200::detail::hfree(m->snap_pinned);
  }
  for (auto &v : s->spare) {
    cublox_b200::detail::dfree(v.occ);
    cublox_b200::detail::dfree(v.cnt);
    cublox_b200::detail::dfree(v.hit);
  }
  cublox_batch_destroy(s->batch);
  cublox_b200::detail::free_fetch(&s->fscratch);
  s->pinned.release_all();
  cudaStreamDestroy(s->stream);
  cudaStreamDestroy(s->fstream);
  delete s;
  return CUBLOX_OK;
}

int cublox_server_add_map(cublox_server *s, const int half_map_size[3], float resolution,
                          int origin_at_center, int has_recenter_threshold,
                          double recenter_threshold, const float origin[3], float max_range,
                          const float log_odds[6], int *map_id) {
  if (!s || !half_map_size || !origin || !map_id)
    return fail(CUBLOX_ERR_INVALID, "server_add_map: null argument");
  int64_t vox = 1;
  for (int a = 0; a < 3; ++a) {
    if (half_map_size[a] < 0) return fail(CUBLOX_ERR_INVALID, "server_add_map: negative half");
    vox *= 2 * static_cast<int64_t>(half_map_size[a]) + 1;
  }
  if (!(resolution > 0.0f) || vox > 0x7fffffff)
    return fail(CUBLOX_ERR_INVALID, "server_add_map: bad resolution or size");
  auto m = std::make_unique<MapState>();
  for (int a = 0; a < 3; ++a) {
    m->half[a] = half_map_size[a];
    m->origin[a] = origin[a];
  }
  m->res = resolution;
  m->ctr = origin_at_center;
  m->has_thr = has_recenter_threshold;
  m->thr = recenter_threshold;
  m->max_range = max_range;
  if (log_odds) {
    std::memcpy(m->lo, log_odds, sizeof(m->lo));
    m->has_lo = true;
  }
  m->voxels = vox;
  m->vox_bytes = cublox_b200::detail::voxel_bytes_for(m->half);
  m->nalloc = cublox_b200::detail::nalloc_for(m->half);
  std::lock_guard<std::mutex> lk(s->mu);
  if (static_cast<int>(s->maps.size()) >= kMaxMaps)
    return fail(CUBLOX_ERR_INVALID, "server_add_map: at most 4096 maps");
  *map_id = static_cast<int>(s->maps.size());
  s->maps.push_back(std::move(m));
  s->n_maps.store(static_cast<int>(s->maps.size()));
  // Once the maps outgrow the budget, evictions will come: pin every map's
  // snapshot buffer now, so that no eviction pins memory while serving
  // (pinning a few hundred MB takes tens of milliseconds).
  size_t total = scratch_bytes(s);
  for (const auto &o : s->maps) total += o->vox_bytes;
  if (total > s->cfg.hbm_budget_bytes)
    for (auto &o : s->maps)
      if (!o->snap_pinned && o->snap_pageable.empty() &&
          cublox_b200::detail::hmalloc(&o->snap_pinned,
                                       static_cast<size_t>(o->nalloc) * sizeof(float)) !=
              cudaSuccess) {
        cudaGetLastError();  // pinned later, or pageable
        o->snap_pinned = nullptr;
      }
  return CUBLOX_OK;
}

static int submit(cublox_server *s, std::unique_ptr<Request> r, int64_t *request_id) {
  r->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(s->mu);
  if (r->map < 0 || r->map >= static_cast<int>(s->maps.size()))
    return fail(CUBLOX_ERR_INVALID, "server: unknown map id");
  r->id = s->next_id++;
  if (request_id) *request_id = r->id;
  s->maps[r->map]->queue.push_back(r.get());
  s->reqs[r->id] = std::move(r);
  ++s->pending;
  s->cv_work.notify_all();
  return CUBLOX_OK;
}

int cublox_server_submit_scan(cublox_server *s, int map_id, const float *xyz, int n,
                              const float sensor_origin[3], int recenter, int64_t *request_id) {
  if (!s || !sensor_origin || (n > 0 && !xyz))
    return fail(CUBLOX_ERR_INVALID, "server_submit_scan: null argument");
  if (n < 0) return fail(CUBLOX_ERR_INVALID, "server_submit_scan: negative point count");
  auto r = std::make_unique<Request>();
  r->kind = kScan;
  r->map = map_id;
  const size_t floats = 3 * static_cast<size_t>(n);
  int cls = -1;
  float *pin = floats ? s->pinned.take(floats * sizeof(float), &cls) : nullptr;
  if (pin) {
    std::memcpy(pin, xyz, floats * sizeof(float));
    r->pin = pin;
    r->pin_cls = cls;
    r->pin_floats = floats;
  } else {
    r->pts.assign(xyz, xyz + floats);
  }
  std::memcpy(r->sensor, sensor_origin, sizeof(r->sensor));
  r->recenter = recenter;
  return submit(s, std::move(r), request_id);
}

int cublox_server_submit_fetch(cublox_server *s, int map_id, const float *centers,
                               int n_centers, float radius, int filter, int max_results,
                               int64_t *request_id) {
  if (!s || (n_centers > 0 && !centers))
    return fail(CUBLOX_ERR_INVALID, "server_submit_fetch: null argument");
  if (n_centers < 0) return fail(CUBLOX_ERR_INVALID, "server_submit_fetch: negative count");
  auto r = std::make_unique<Request>();
  r->kind = kFetch;
  r->map = map_id;
  r->centers.assign(centers, centers + 3 * static_cast<size_t>(n_centers));
  r->radius = radius;
  r->filter = filter;
  r->max_results = max_results;
  return submit(s, std::move(r), request_id);
}

int cublox_server_wait(cublox_server *s, int64_t request_id, double timeout_s, int *state) {
  if (!s) return fail(CUBLOX_ERR_INVALID, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  Request *r = find(s, request_id);
  if (!r) return fail(CUBLOX_ERR_INVALID, "server_wait: unknown request");
  auto done = [&] { return r->state == CUBLOX_REQ_DONE || r->state == CUBLOX_REQ_FAILED; };
  if (timeout_s < 0)
    s->cv_done.wait(lk, done);
  else
    s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done);
  if (state) *state = r->state;
  if (r->state == CUBLOX_REQ_FAILED) return fail(r->error, "server request: " + r->message);
  return CUBLOX_OK;
}

int cublox_server_drain(cublox_server *s) {
  if (!s) return fail(CUBLOX_ERR_INVALID, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  s->cv_done.wait(lk, [&] { return s->pending == 0; });
  return CUBLOX_OK;
}

int cublox_server_request_times(cublox_server *s, int64_t request_id, double *queued_ms,
                                double *latency_ms) {
  if (!s) return fail(CUBLOX_ERR_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  Request *r = find(s, request_id);
  if (!r) return fail(CUBLOX_ERR_INVALID, "request_times: unknown request");
  if (r->state != CUBLOX_REQ_DONE && r->state != CUBLOX_REQ_FAILED)
    return fail(CUBLOX_ERR_INVALID, "request_times: request not finished");
  if (queued_ms) *queued_ms = ms_between(r->t_submit, r->t_start);
  if (latency_ms) *latency_ms = ms_between(r->t_submit, r->t_done);
  return CUBLOX_OK;
}

int cublox_server_fetch_result(cublox_server *s, int64_t request_id, int64_t *offsets,
                               float *out_pos, uint8_t *out_state, int64_t capacity,
                               int64_t *n_samples) {
  if (!s) return fail(CUBLOX_ERR_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  Request *r = find(s, request_id);
  if (!r || r->kind != kFetch) return fail(CUBLOX_ERR_INVALID, "fetch_result: not a fetch");
  if (r->state != CUBLOX_REQ_DONE) return fail(CUBLOX_ERR_INVALID, "fetch_result: not done");
  const int64_t n = static_cast<int64_t>(r->fstate.size());
  if (n_samples) *n_samples = n;
  if (offsets) std::copy(r->offsets.begin(), r->offsets.end(), offsets);
  if (out_pos || out_state) {
    if (capacity < n) return fail(CUBLOX_ERR_INVALID, "fetch_result: capacity too small");
    if (out_pos) std::copy(r->fpos.begin(), r->fpos.end(), out_pos);
    if (out_state) std::copy(r->fstate.begin(), r->fstate.end(), out_state);
  }
  return CUBLOX_OK;
}

int cublox_server_release(cublox_server *s, int64_t request_id) {
  if (!s) return fail(CUBLOX_ERR_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  Request *r = find(s, request_id);
  if (!r) return fail(CUBLOX_ERR_INVALID, "release: unknown request");
  if (r->state != CUBLOX_REQ_DONE && r->state != CUBLOX_REQ_FAILED)
    return fail(CUBLOX_ERR_INVALID, "release: request not finished");
  s->reqs.erase(request_id);
  return CUBLOX_OK;
}

int cublox_server_export(cublox_server *s, int map_id, float *occ_host, int origin_index[3]) {
  if (!s || !occ_host) return fail(CUBLOX_ERR_INVALID, "server_export: null argument");
  int rc = cublox_server_drain(s);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(s->mu);
  if (map_id < 0 || map_id >= static_cast<int>(s->maps.size()))
    return fail(CUBLOX_ERR_INVALID, "server_export: unknown map id");
  MapState &m = *s->maps[map_id];
  const size_t vox = static_cast<size_t>(m.voxels);
  if (!m.g) {
    std::fill(occ_host, occ_host + vox, 0.0f);
    if (origin_index) {
      cublox_grid *tmp = nullptr;  // a never-served map: its constructor origin
      rc = cublox_grid_create(m.half, m.res, m.ctr, m.has_thr, m.thr, m.origin, s->stream, &tmp);
      if (rc) return rc;
      cublox_grid_origin(tmp, origin_index, nullptr);
      cublox_grid_destroy(tmp);
    }
    return CUBLOX_OK;
  }
  if (m.resident) {
    rc = cublox_grid_export(m.g, occ_host);
    if (rc) return rc;
  } else {
    // the snapshot is complete once the server stream has run its copy
    if (cudaStreamSynchronize(s->stream) != cudaSuccess)
      return fail(CUBLOX_ERR_CUDA, "server_export: stream synchronisation failed");
    cublox_b200::detail::layout_to_reference(m.g, m.snapshot(), occ_host);
  }
  if (origin_index) cublox_grid_origin(m.g, origin_index, nullptr);
  return CUBLOX_OK;
}

int cublox_server_cancel(cublox_server *s, int64_t request_id) {
  if (!s) return fail(CUBLOX_ERR_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  Request *r = find(s, request_id);
  if (!r) return fail(CUBLOX_ERR_INVALID, "cancel: unknown request");
  std::deque<Request *> &q = s->maps[r->map]->queue;
  const auto it = std::find(q.begin(), q.end(), r);
  // Only a request still waiting in its map's queue can be withdrawn; one
  // the worker has taken is being served (or done).
  if (r->state != CUBLOX_REQ_QUEUED || it == q.end())
    return fail(CUBLOX_ERR_INVALID, "cancel: request is already being served or finished");
  q.erase(it);
  ++s->stats.cancelled;
  finish(s, r, CUBLOX_ERR_CANCELLED, "cancelled before it was served");
  s->cv_done.notify_all();
  return CUBLOX_OK;
}

int cublox_server_scratch_bytes(const cublox_server_config *cfg, uint64_t *bytes) {
  if (!cfg || !bytes) return fail(CUBLOX_ERR_INVALID, "server_scratch_bytes: null argument");
  cublox_server_config c = *cfg;
  fill_defaults(&c);
  *bytes = scratch_bytes(c);
  return CUBLOX_OK;
}

int cublox_server_get_stats(cublox_server *s, cublox_server_stats *out) {
  if (!s || !out) return fail(CUBLOX_ERR_INVALID, "server_stats: null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  int resident = 0;
  for (auto &m : s->maps) resident += m->resident ? 1 : 0;
  out->resident_maps = resident;
  return CUBLOX_OK;
}

}  // extern "C"

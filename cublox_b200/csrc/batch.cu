// Batched integration: scans of many grids in one walk launch and one fold
// launch (include/cublox_b200.h, cublox_batch_*).
//
//  walk  persistent CTAs take work items — a contiguous run of one map's
//        rays — from a device queue.  A CTA zeroes an S^3 shared-memory cube
//        centred on that map's sensor voxel, walks the run (one thread per
//        ray, the exact walk of ray_walk.cuh), and flushes the cube into the
//        map's counters.  Points are read in place from one concatenated
//        x0 y0 z0 x1 ... buffer.
//  fold  persistent CTAs take (map, line range) items; their warps fold the
//        32-voxel lines the walk flagged, a whole 128-byte line per access
//        (fold.cuh, fold_lines).
//
// The per-step launch sequence reads everything it needs (map descriptors,
// item lists and counts) from device buffers, so it can be captured once
// into a CUDA graph and replayed: each step only copies the new descriptors
// and items, then launches the graph.  Launch shapes (cube side, rays per
// item, CTA size) are chosen online: the first updates rotate through the
// candidate shapes — every one gives identical results — timing the walk,
// and the fastest is kept.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cublox_b200.h"
#include "exact_fp.cuh"
#include "fold.cuh"
#include "grid_internal.hpp"
#include "kernels.cuh"
#include "far_walk.cuh"
#include "ray_walk.cuh"

using namespace cublox_b200;
using cublox_b200::detail::cuda_fail;
using cublox_b200::detail::fail;

namespace {

struct MapDesc {
  RayParams ray;
  float *occ;
  float l_hit, l_miss, l_min, l_max, l_unknown;
  int clo[3];  // cube corner, global voxel index
  int n_walk;  // walk items of this map (fused launch: its folds wait for them)
};

struct WalkItem {
  int map, start, count, pad;
};

struct FoldItem {
  int map, start, count, pad;  // lines [start, start + count) of the map
};

// counters: [0] walk queue, [1] walk items, [2] fold queue, [3] fold items,
// [4] a fused launch's fold wait gave up (the rest of the launch then skips
// its waits and folds), [5] the fused launch's wait limit (sleep rounds)
constexpr int kCounters = 6;
constexpr int kFoldItemLines = 1 << 11;  // 32-voxel lines per fold item
static_assert(kFoldItemLines <= kListLines && kFoldItemLines % 16 == 0,
              "a fold item fits one CTA's line list");
// Fused launch: how long a fold item waits for its map's walk items
// (rounds of a ~256 ns sleep, about 2 s) before it gives up and flags
// kErrWaitTimeout in the map's error word (CUBLOX_BATCH_OPT_WAIT_LIMIT).
constexpr int kWaitIters = 1 << 23;

// Near phase of the two-phase walk (far_walk.cuh), from the ray's start.
// Returns true if the ray's loop ended in it; false once the walk is inside
// the window and outside the cube (f then holds it).
template <int S, int SZ = S>
__device__ __forceinline__ bool walk_near(const RayParams &p, uint32_t *cube, const int clo[3],
                                          RayWalk &w, FarWalk &f, uint32_t &incs) {
  for (int k = 0;; ++k) {
    if (k >= w.max_steps || at_end(w)) return true;
    if (in_window(w, p)) {
      const int c = cube_cell<S, SZ>(w.id[0], w.id[1], w.id[2], clo);
      if (c < 0) {
        to_far(p, w, k, f);
        return false;
      }
      atomicAdd(&cube[c], 1u);
      ++incs;
    } else if (left_for_good(w, p)) {
      return true;
    }
    ray_step(w, p);
  }
}

// One walk item: zero the cube, walk the item's rays (in order of their
// estimated length when the item has at most twice as many rays as the CTA
// has threads), flush the cube into the map's counters.  Ends with a CTA
// barrier.
template <int S, int SZ = S>
__device__ __forceinline__ void walk_item(const MapDesc &md, const WalkItem &item,
                                          uint32_t *cube) {
  constexpr int kCube = S * S * SZ;
  const RayParams p = md.ray;
  const int clo[3] = {md.clo[0], md.clo[1], md.clo[2]};
  for (int q = threadIdx.x; q < kCube / 4; q += blockDim.x)
    reinterpret_cast<uint4 *>(cube)[q] = make_uint4(0u, 0u, 0u, 0u);
  __shared__ RayOrder order;
  const int t = threadIdx.x, nt = blockDim.x;
  const bool ordered = item.count <= 2 * nt && item.count <= kOrderCap;
  if (ordered)
    order_rays(p, item.start, item.count, order);  // ends with a barrier
  else
    __syncthreads();
  uint32_t rays = 0, incs = 0, hits = 0;
  // Ordered: thread t walks the t-th shortest ray, then (items of more rays
  // than threads) the t-th longest, so every thread gets about the same
  // work.  Every lane runs every round (live or not) and the warp meets
  // after the near phase, so that its lanes walk their far phases together
  // rather than in groups that entered the far loop at different times.
  const int rounds = ordered ? (item.count > nt ? 2 : 1) : (item.count + nt - 1) / nt;
#pragma unroll 1
  for (int r = 0; r < rounds; ++r) {
    int j;
    bool live;
    float x = 0.0f, y = 0.0f, z = 0.0f;
    if (ordered) {
      j = r ? item.count - 1 - t : t;
      live = r ? j >= nt : j < item.count;
      if (live) {
        j = order.idx[j];
        x = order.x[j];
        y = order.y[j];
        z = order.z[j];
      }
    } else {
      j = r * nt + t;
      live = j < item.count;
      if (live) {
        const size_t k = static_cast<size_t>(item.start + j) * p.stride;
        x = p.x[k];
        y = p.y[k];
        z = p.z[k];
      }
    }
    FarWalk f;
    RayEnd re{-1, -1, false};
    bool far = false;
    if (live) {
      RayWalk w;
      if (ray_begin(p, x, y, z, w)) {
        ++rays;
        re = ray_end_of<S, SZ>(p, w, clo);
        far = !walk_near<S, SZ>(p, cube, clo, w, f, incs);
      } else {
        live = false;
      }
    }
    __syncwarp();
    if (far) walk_far(p, f, f.left, incs);
    if (live) apply_end<S>(p, cube, re, incs, hits);
  }
  __syncthreads();
  flush_cube<S, SZ>(p, cube, clo);
  if (p.stats) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      rays += __shfl_down_sync(0xffffffffu, rays, off);
      incs += __shfl_down_sync(0xffffffffu, incs, off);
      hits += __shfl_down_sync(0xffffffffu, hits, off);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(p.stats + 0, static_cast<unsigned long long>(rays));
      atomicAdd(p.stats + 1, static_cast<unsigned long long>(incs));
      atomicAdd(p.stats + 2, static_cast<unsigned long long>(hits));
    }
  }
  __syncthreads();
}

// ---- refill walk -----------------------------------------------------------
// One thread per ray leaves lanes idle: a warp runs until its longest ray
// ends, and rays of one azimuth column differ several-fold in length.  The
// refill walk splits an item in two phases.  Phase A: every thread sets up
// its ray and walks its near phase (the sensor cube); a ray that goes on
// leaves its far-phase state in a shared-memory queue.  Phase B: lanes take
// far states from the queue and walk them kRefillSteps loop iterations at a
// time; a lane whose ray is over takes the next state, so the warp's lanes
// stay busy until the item's queue is empty.  The loop iterations walked,
// and so the counts, are those of the single loop.
constexpr int kRefillRays = 512;   // rays per item (queue capacity)
constexpr int kRefillSteps = 32;   // far-loop iterations between refills
constexpr int kFarWords = 27;      // queued state: FarWalk (23) + RayEnd (3), odd stride

__device__ __forceinline__ void far_store(uint32_t *q, const FarWalk &f, const RayEnd &re) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    q[a] = __float_as_uint(f.tM[a]);
    q[3 + a] = __float_as_uint(f.tD[a]);
    q[6 + a] = static_cast<uint32_t>(f.e[a]);
    q[9 + a] = static_cast<uint32_t>(f.out[a]);
    q[12 + a] = static_cast<uint32_t>(f.slot[a]);
    q[15 + a] = static_cast<uint32_t>(f.st[a]);
    q[18 + a] = static_cast<uint32_t>(f.off[a]);
  }
  q[21] = static_cast<uint32_t>(f.left);
  q[22] = static_cast<uint32_t>(f.h);
  q[23] = static_cast<uint32_t>(re.h);
  q[24] = static_cast<uint32_t>(re.c);
  q[25] = re.hit ? 1u : 0u;
}

__device__ __forceinline__ void far_load(const uint32_t *q, FarWalk &f, RayEnd &re) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    f.tM[a] = __uint_as_float(q[a]);
    f.tD[a] = __uint_as_float(q[3 + a]);
    f.e[a] = static_cast<int>(q[6 + a]);
    f.out[a] = static_cast<int>(q[9 + a]);
    f.slot[a] = static_cast<int>(q[12 + a]);
    f.st[a] = static_cast<int>(q[15 + a]);
    f.off[a] = static_cast<int>(q[18 + a]);
  }
  f.left = static_cast<int>(q[21]);
  f.h = static_cast<int>(q[22]);
  f.line = -1;
  re.h = static_cast<int>(q[23]);
  re.c = static_cast<int>(q[24]);
  re.hit = q[25] != 0u;
}

// One walk item (at most kRefillRays rays) in the two phases above.  Ends
// with a CTA barrier.
template <int S>
__device__ __forceinline__ void walk_item_refill(const MapDesc &md, const WalkItem &item,
                                                 uint32_t *cube, uint32_t *fq, int *s_q) {
  constexpr int kCube = S * S * S;
  const RayParams p = md.ray;
  const int clo[3] = {md.clo[0], md.clo[1], md.clo[2]};
  for (int q = threadIdx.x; q < kCube / 4; q += blockDim.x)
    reinterpret_cast<uint4 *>(cube)[q] = make_uint4(0u, 0u, 0u, 0u);
  if (threadIdx.x == 0) s_q[0] = s_q[1] = 0;  // queued, taken
  __syncthreads();
  uint32_t rays = 0, incs = 0, hits = 0;
  for (int i = item.start + threadIdx.x; i < item.start + item.count; i += blockDim.x) {
    const size_t k = static_cast<size_t>(i) * p.stride;
    RayWalk w;
    if (!ray_begin(p, p.x[k], p.y[k], p.z[k], w)) continue;
    ++rays;
    const RayEnd re = ray_end_of<S>(p, w, clo);
    FarWalk f;
    if (walk_near<S>(p, cube, clo, w, f, incs)) {
      apply_end<S>(p, cube, re, incs, hits);
    } else {
      const int slot = atomicAdd(&s_q[0], 1);
      far_store(fq + slot * kFarWords, f, re);
    }
  }
  __syncthreads();
  const int queued = s_q[0];
  FarWalk f;
  RayEnd re;
  bool alive = false;
  for (;;) {
    if (!alive) {
      const int t = atomicAdd(&s_q[1], 1);
      if (t >= queued) break;
      far_load(fq + t * kFarWords, f, re);
      alive = true;
    }
    if (walk_far(p, f, kRefillSteps, incs)) {
      apply_end<S>(p, cube, re, incs, hits);
      alive = false;
    }
  }
  __syncthreads();
  flush_cube<S>(p, cube, clo);
  if (p.stats) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      rays += __shfl_down_sync(0xffffffffu, rays, off);
      incs += __shfl_down_sync(0xffffffffu, incs, off);
      hits += __shfl_down_sync(0xffffffffu, hits, off);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(p.stats + 0, static_cast<unsigned long long>(rays));
      atomicAdd(p.stats + 1, static_cast<unsigned long long>(incs));
      atomicAdd(p.stats + 2, static_cast<unsigned long long>(hits));
    }
  }
  __syncthreads();
}

// Persistent refill walk: CTAs take walk items (at most kRefillRays rays
// each) from counters[0].  Shared memory: the S^3 cube, then the far-state
// queue.
template <int S>
__global__ void __launch_bounds__(512, 1) batch_walk_refill_kernel(const MapDesc *maps,
                                                                   const WalkItem *items,
                                                                   int *counters) {
  extern __shared__ uint32_t smem[];
  __shared__ int s_item;
  __shared__ int s_q[2];
  const int n_items = counters[1];
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(&counters[0], 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n_items) break;
    const WalkItem item = items[it];
    walk_item_refill<S>(maps[item.map], item, smem, smem + S * S * S, s_q);
  }
}

__device__ __forceinline__ FoldView fold_view(const MapDesc &m) {
  return FoldView{m.occ, m.ray.cnt, m.ray.hit, m.ray.vnum, m.l_hit, m.l_miss, m.l_min, m.l_max,
                  m.l_unknown, m.ray.fp};
}

// One fold item: the flagged lines among [start, start + count), the CTA's
// warps taking groups of 32 lines in turn.  kAll: fold every line of the
// item, flagged or not (the reference's full sweep, for comparison).
template <bool kL2, bool kAll = false>
__device__ __forceinline__ uint32_t fold_item(const MapDesc &m, const FoldItem &item) {
  const FoldView v = fold_view(m);
  const int warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  return fold_lines<8, kL2, kAll>(v, m.ray.dirty, item.start + 32 * warp, item.start + item.count,
                                  32 * warps);
}

__device__ __forceinline__ void add_touched(const MapDesc &m, uint32_t t) {
  if (!m.ray.stats) return;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
  if ((threadIdx.x & 31) == 0 && t) atomicAdd(m.ray.stats + 3, static_cast<unsigned long long>(t));
}

// Persistent walk: CTAs take walk items from counters[0] until none is left.
// kMinCtas 2 caps registers so that two 1024-thread CTAs share an SM.
template <int S, int kMinCtas>
__global__ void __launch_bounds__(1024, kMinCtas) batch_walk_kernel(const MapDesc *maps,
                                                                    const WalkItem *items,
                                                                    int *counters) {
  extern __shared__ uint32_t cube[];
  __shared__ int s_item;
  const int n_items = counters[1];
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(&counters[0], 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n_items) break;
    const WalkItem item = items[it];
    walk_item<S>(maps[item.map], item, cube);
  }
}

// The same with a flat S x S x S/2 cube (64 KB at S = 32) and 512-thread
// CTAs capped at 64 registers, so that two CTAs share an SM: twice the
// resident warps of the 32^3 cube.  LiDAR beams within +-22.5 degrees stay
// within +-0.66 m of the sensor's height inside the cube's +-1.6 m, so the
// flat cube holds the same near field.
template <int S>
__global__ void __launch_bounds__(512, 2) batch_walk_flat_kernel(const MapDesc *maps,
                                                                 const WalkItem *items,
                                                                 int *counters) {
  extern __shared__ uint32_t cube[];
  __shared__ int s_item;
  const int n_items = counters[1];
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(&counters[0], 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n_items) break;
    const WalkItem item = items[it];
    walk_item<S, S / 2>(maps[item.map], item, cube);
  }
}

// Persistent walk without per-item barriers.  A CTA adopts one map at a
// time (starting at blockIdx % maps, then the next map with rays left): it
// zeroes its cube around that map's sensor, and its warps take 32-ray items
// of the map from the map's own counter until none is left; only then does
// the CTA synchronise, flush the cube and move on.  A warp waits only for
// its own longest ray, never for the rest of the CTA.  counters[1] holds the
// number of maps; next[m] is map m's item counter (zero at launch).
template <int S>
__global__ void __launch_bounds__(1024) batch_walk_wq_kernel(const MapDesc *maps,
                                                             const WalkItem * /*items*/,
                                                             int *counters, int *next) {
  extern __shared__ uint32_t cube[];
  constexpr int kCube = S * S * S;
  __shared__ int s_map;
  const int n_maps = counters[1];
  const unsigned lane = threadIdx.x & 31u;
  int m = n_maps > 0 ? static_cast<int>(blockIdx.x) % n_maps : 0;
  for (;;) {
    if (threadIdx.x == 0) {
      int found = -1;
      for (int k = 0; k < n_maps; ++k) {
        const int mm = (m + k) % n_maps;
        if (*reinterpret_cast<volatile int *>(next + mm) * 32 < maps[mm].ray.n) {
          found = mm;
          break;
        }
      }
      s_map = found;
    }
    __syncthreads();
    m = s_map;
    if (m < 0) break;
    const MapDesc &md = maps[m];
    const RayParams p = md.ray;
    const int clo[3] = {md.clo[0], md.clo[1], md.clo[2]};
    for (int q = threadIdx.x; q < kCube / 4; q += blockDim.x)
      reinterpret_cast<uint4 *>(cube)[q] = make_uint4(0u, 0u, 0u, 0u);
    __syncthreads();
    uint32_t rays = 0, incs = 0, hits = 0;
    for (;;) {
      int it = 0;
      if (lane == 0) it = atomicAdd(next + m, 1);
      it = __shfl_sync(0xffffffffu, it, 0);
      if (it * 32 >= p.n) break;
      const int i = it * 32 + static_cast<int>(lane);
      if (i >= p.n) continue;
      const size_t k = static_cast<size_t>(i) * p.stride;
      RayWalk w;
      if (!ray_begin(p, p.x[k], p.y[k], p.z[k], w)) continue;
      ++rays;
      const RayEnd re = ray_end_of<S>(p, w, clo);
      FarWalk f;
      if (!walk_near<S>(p, cube, clo, w, f, incs)) walk_far(p, f, f.left, incs);
      apply_end<S>(p, cube, re, incs, hits);
    }
    __syncthreads();
    flush_cube<S>(p, cube, clo);
    if (p.stats) {
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        rays += __shfl_down_sync(0xffffffffu, rays, off);
        incs += __shfl_down_sync(0xffffffffu, incs, off);
        hits += __shfl_down_sync(0xffffffffu, hits, off);
      }
      if (lane == 0) {
        atomicAdd(p.stats + 0, static_cast<unsigned long long>(rays));
        atomicAdd(p.stats + 1, static_cast<unsigned long long>(incs));
        atomicAdd(p.stats + 2, static_cast<unsigned long long>(hits));
      }
    }
    __syncthreads();
    m = (m + 1) % n_maps;
  }
}

// Persistent fold: CTAs take fold items from counters[2].  kAll: every
// line, not only the flagged ones.
template <bool kAll>
__global__ void __launch_bounds__(256) batch_fold_kernel(const MapDesc *maps,
                                                         const FoldItem *items,
                                                         int *counters) {
  __shared__ int s_item;
  const int n_items = counters[3];
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(&counters[2], 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= n_items) break;
    const FoldItem item = items[it];
    const MapDesc &m = maps[item.map];
    add_touched(m, fold_item<false, kAll>(m, item));
  }
}

// Persistent fold over per-item lists of the flagged lines (fold.cuh,
// build_line_list / fold_line_list): CTAs take fold items from counters[2]
// and load the next item's flags before folding the current list.
template <int kQuads, int kMinCtas>
__global__ void __launch_bounds__(kListThreads, kMinCtas) batch_fold_list_kernel(
    const MapDesc *maps, const FoldItem *items, int *counters) {
  __shared__ LineList L;
  __shared__ HitQueue hq;
  __shared__ int s_item;
  const int n_items = counters[3];
  if (threadIdx.x == 0) {
    s_item = atomicAdd(&counters[2], 1);
    hq.n = 0;
  }
  __syncthreads();
  int it = s_item;
  uint4 f = make_uint4(0u, 0u, 0u, 0u);
  if (it < n_items) {
    const FoldItem fi = items[it];
    f = load_line_flags(maps[fi.map].ray.dirty, fi.start, fi.count);
  }
  while (it < n_items) {
    const FoldItem item = items[it];
    const MapDesc &m = maps[item.map];
    const int n = build_line_list(line_flag_bits(f), L, m.ray.dirty, item.start, item.count);
    if (threadIdx.x == 0) s_item = atomicAdd(&counters[2], 1);
    __syncthreads();
    const int next = s_item;
    if (next < n_items) {
      const FoldItem fi = items[next];
      f = load_line_flags(maps[fi.map].ray.dirty, fi.start, fi.count);
    }
    const FoldView v = fold_view(m);
    add_touched(m, fold_line_list<kQuads, false>(v, L.line, n, item.start, &hq));
    __syncthreads();
    fold_hit_queue(v, hq);  // ends with a barrier: the list and s_item are rewritten next
    it = next;
  }
}

// Thread 0 of a CTA about to fold map m: waits until all of m's walk items
// have finished (*done == n_walk), at most counters[5] sleep rounds.  Once
// one wait of the launch gave up (counters[4]), the rest do not wait; a wait
// that gives up sets the map's error word.  Returns 1 if the walks finished.
__device__ __forceinline__ int wait_walks(const MapDesc &m, const int *done, int *counters) {
  volatile const int *vd = done;
  volatile int *gave_up = counters + 4;
  int ok = 0;
  const int limit = counters[5];
  for (int k = 0; k < limit && !*gave_up; ++k) {
    if (*vd >= m.n_walk) {
      ok = 1;
      break;
    }
    __nanosleep(256);
  }
  __threadfence();
  if (!ok) {
    *gave_up = 1;
    atomicOr(m.ray.err, kErrWaitTimeout);
  }
  return ok;
}

// Walk and fold in one persistent launch.  Items come from one queue, in
// the order the host wrote them: map 0's walk items, map 1's walk items,
// map 0's fold items, map 2's walk items, map 1's fold items, ... (a fold
// item is a WalkItem with map = ~map and its FoldItem fields in place).  A
// fold item of map m starts once all of m's walk items have finished, so
// CTAs fold map m while others walk map m + 2 and later: the DRAM-bound
// sweep overlaps the atomic-bound walk.  A CTA waits only on walk items
// that running CTAs have already taken (they come earlier in the queue), so
// the wait always ends; it is bounded all the same, and once one wait gives
// up the launch skips the remaining waits and folds (the map's error word
// says so).
template <int S>
__global__ void __launch_bounds__(1024) batch_fused_kernel(const MapDesc *maps,
                                                           const WalkItem *items,
                                                           const FoldItem * /*fold items*/,
                                                           int *counters, int *done) {
  extern __shared__ uint32_t cube[];
  __shared__ int s_item, s_ok;
  const int n_all = counters[1];
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(&counters[0], 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n_all) break;
    const WalkItem raw = items[it];
    if (raw.map >= 0) {
      walk_item<S>(maps[raw.map], raw, cube);  // ends with a barrier
      if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(done + raw.map, 1);
      }
    } else {
      const FoldItem item{~raw.map, raw.start, raw.count, raw.pad};
      const MapDesc &m = maps[item.map];
      if (threadIdx.x == 0) s_ok = wait_walks(m, done + item.map, counters);
      __syncthreads();
      if (s_ok) add_touched(m, fold_item<true>(m, item));
      __syncthreads();
    }
  }
}

// The fused launch with the flat cube: 512-thread CTAs, two per SM (as the
// flat walk), folding through per-item line lists.  Items come in the order
// the host wrote them, a map's fold items `lag` maps after its walk items
// (the shape's `fused` value), and wait (bounded) as in batch_fused_kernel.
template <int S>
__global__ void __launch_bounds__(512, 2) batch_fused_flat_kernel(const MapDesc *maps,
                                                                  const WalkItem *items,
                                                                  const FoldItem * /*fold items*/,
                                                                  int *counters, int *done) {
  extern __shared__ uint32_t cube[];
  __shared__ LineList L;
  __shared__ HitQueue hq;
  __shared__ int s_item, s_ok;
  if (threadIdx.x == 0) hq.n = 0;
  const int n_all = counters[1];
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(&counters[0], 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n_all) break;
    const WalkItem raw = items[it];
    if (raw.map >= 0) {
      walk_item<S, S / 2>(maps[raw.map], raw, cube);  // ends with a barrier
      if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(done + raw.map, 1);
      }
    } else {
      const FoldItem item{~raw.map, raw.start, raw.count, raw.pad};
      const MapDesc &m = maps[item.map];
      if (threadIdx.x == 0) s_ok = wait_walks(m, done + item.map, counters);
      __syncthreads();
      if (s_ok) {
        const uint4 f = load_line_flags<true>(m.ray.dirty, item.start, item.count);
        const int n = build_line_list(line_flag_bits(f), L, m.ray.dirty, item.start, item.count);
        const FoldView v = fold_view(m);
        add_touched(m, fold_line_list<2, true>(v, L.line, n, item.start, &hq));
        __syncthreads();
        fold_hit_queue(v, hq);
      }
      __syncthreads();
    }
  }
}

struct Shape {
  int cube;      // 0, 16, 32
  int rays;      // rays per walk item; 0: about two items per resident CTA
  int block;     // walk (or fused) CTA size
  int fused;     // >= 1: one launch, a map's folds queued `fused` maps after its walks
  int min_ctas;  // 2: registers capped for two CTAs per SM (cube <= 16)
  int wq;        // 1: warps take 32-ray items of a CTA's current map (no item barriers)
  int refill;    // 1: two-phase items, lanes refilled from a far-state queue
  int flat;      // 1: S x S x S/2 cube, two 512-thread CTAs per SM
};

const Shape kShapes[] = {{32, 512, 512, 0, 1, 0, 0},  {32, 1024, 1024, 0, 1, 0, 0},
                         {32, 0, 512, 0, 1, 1, 0},    {32, 0, 1024, 0, 1, 1, 0},
                         {16, 0, 512, 0, 1, 1, 0},    {16, 1024, 1024, 0, 2, 0, 0},
                         {32, 1024, 1024, 1, 1, 0, 0}, {16, 512, 512, 1, 1, 0, 0},
                         {32, kRefillRays, 512, 0, 1, 0, 1}, {16, kRefillRays, 512, 0, 1, 0, 1},
                         {32, 512, 512, 0, 2, 0, 0, 1},     {32, 256, 512, 0, 2, 0, 0, 1},
                         {32, 512, 512, 2, 2, 0, 0, 1},     {32, 512, 512, 1, 2, 0, 0, 1},
                         {32, 1024, 512, 0, 2, 0, 0, 1},    {32, 768, 512, 0, 2, 0, 0, 1}};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

// The tuner's candidates: the launch shapes that have been fastest on some
// workload, with the default voxel layout (8 x 4 x 1 bricks), then the two
// fastest walk shapes with the other layouts (4 x 8 x 1 and 4 x 4 x 2
// bricks, the reference's hash order).  Shapes 3, 4, 5, 8, 9 and 13 stay
// selectable.  A candidate with another layout moves every grid of the
// update to it first.
struct Candidate {
  int shape, layout;
};
const Candidate kCandidates[] = {{0, 320},  {1, 320},  {2, 320},  {6, 320},  {7, 320},
                                 {10, 320}, {11, 320}, {12, 320}, {14, 320}, {15, 320},
                                 {1, 230},  {10, 230}, {1, 221},  {10, 221}, {1, 0}};
constexpr int kNumCandidates = sizeof(kCandidates) / sizeof(kCandidates[0]);

int sm_count_batch() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

template <int S>
const void *shape_kernel_s(const Shape &sh) {
  if (sh.flat && sh.fused) return reinterpret_cast<const void *>(batch_fused_flat_kernel<S>);
  if (sh.flat) return reinterpret_cast<const void *>(batch_walk_flat_kernel<S>);
  if (sh.refill) return reinterpret_cast<const void *>(batch_walk_refill_kernel<S>);
  if (sh.fused) return reinterpret_cast<const void *>(batch_fused_kernel<S>);
  if (sh.wq) return reinterpret_cast<const void *>(batch_walk_wq_kernel<S>);
  if constexpr (S < 32) {
    if (sh.min_ctas >= 2) return reinterpret_cast<const void *>(batch_walk_kernel<S, 2>);
  }
  return reinterpret_cast<const void *>(batch_walk_kernel<S, 1>);
}

// The walk (or fused) kernel of a shape.
const void *shape_kernel(const Shape &sh) {
  return sh.cube >= 32 ? shape_kernel_s<32>(sh)
                       : (sh.cube >= 16 ? shape_kernel_s<16>(sh) : shape_kernel_s<0>(sh));
}

size_t shape_smem(const Shape &sh) {
  return sizeof(uint32_t) * (sh.cube * sh.cube * (sh.flat ? sh.cube / 2 : sh.cube) +
                             (sh.refill ? kRefillRays * kFarWords : 0));
}

// CTAs of a shape's persistent launch: resident CTAs per SM x SMs.  Sets
// the shared-memory attribute on first use; every shape is prepared when a
// batch is created, so a graph capture only enqueues launches.
int shape_grid(int shape) {
  static int cached[kNumShapes] = {};
  if (cached[shape] == 0) {
    const Shape &sh = kShapes[shape];
    const void *fn = shape_kernel(sh);
    const size_t smem = shape_smem(sh);
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem)) != cudaSuccess)
      cudaGetLastError();
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, sh.block, smem) !=
        cudaSuccess) {
      cudaGetLastError();
      per_sm = 1;
    }
    cached[shape] = sm_count_batch() * (per_sm < 1 ? 1 : per_sm);
  }
  return cached[shape];
}

// Rays per walk item of a shape for a step of `total` rays.
int shape_rays(int shape, int64_t total) {
  const Shape &sh = kShapes[shape];
  if (sh.rays > 0) return sh.rays;
  const int64_t items = 2 * static_cast<int64_t>(shape_grid(shape));
  const int64_t per = (total + items - 1) / items;
  return static_cast<int>(std::min<int64_t>(1 << 20, std::max<int64_t>(256, (per + 31) & ~31)));
}

cudaError_t launch_walk(const MapDesc *maps, const WalkItem *witems, const FoldItem *fitems,
                        int *counters, int *done, int shape, cudaStream_t s) {
  const Shape &sh = kShapes[shape];
  void *walk_args[] = {&maps, &witems, &counters};
  void *fused_args[] = {&maps, &witems, &fitems, &counters, &done};
  void *wq_args[] = {&maps, &witems, &counters, &done};
  return cudaLaunchKernel(shape_kernel(sh), dim3(shape_grid(shape)), dim3(sh.block),
                          sh.fused ? fused_args : (sh.wq ? wq_args : walk_args), shape_smem(sh),
                          s);
}

cudaError_t launch_fold(const MapDesc *maps, const FoldItem *fitems, int *counters,
                        int variant, cudaStream_t s) {
  const dim3 grid(sm_count_batch() * 8), block(256);
  if (variant == 0) {
    batch_fold_list_kernel<4, 4><<<sm_count_batch() * 4, kListThreads, 0, s>>>(maps, fitems, counters);
  } else if (variant == 1) {
    batch_fold_kernel<true><<<grid, block, 0, s>>>(maps, fitems, counters);
  } else {
    batch_fold_kernel<false><<<grid, block, 0, s>>>(maps, fitems, counters);
  }
  return cudaGetLastError();
}

}  // namespace

struct cublox_batch {
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::vector<cublox_grid *> grids;  // owned by the batch
  // device side
  MapDesc *d_maps = nullptr;
  int maps_cap = 0;
  WalkItem *d_witems = nullptr;
  int witems_cap = 0;
  FoldItem *d_fitems = nullptr;
  int fitems_cap = 0;
  int *d_counters = nullptr;
  int *d_done = nullptr;  // per map: walk items finished (fused launch)
  float *d_points = nullptr;
  size_t points_cap = 0;  // floats
  // pinned host staging
  MapDesc *h_maps = nullptr;
  WalkItem *h_witems = nullptr;
  FoldItem *h_fitems = nullptr;
  int *h_counters = nullptr;
  float *h_points = nullptr;
  size_t h_points_cap = 0;
  cudaEvent_t staged = nullptr;  // host staging free again
  cudaEvent_t points_read = nullptr;  // the walk is done with points it read from h_points
  // shape choice
  int shape = 0;
  int layout = detail::kDefaultLayout;  // voxel layout of the batch's grids
  int wait_limit = kWaitIters;  // fused launch: sleep rounds a fold item waits
  bool inject_missing_walk = false;  // test hook (CUBLOX_BATCH_OPT_INJECT_MISSING_WALK)
  bool autotune = true;
  int tune_step = 0;
  int tune_rounds = 2;
  std::vector<float> tune_ms;
  std::vector<WalkItem> order;  // fused launch: the queue in launch order (capacity kept)
  std::vector<int> w_end, f_end;  // per map of an update: end of its walk / fold items
  bool graphs = false;
  bool host_read = true;  // the walk reads host points in place (CUBLOX_BATCH_OPT_HOST_READ)
  int fold_variant = 0;
  cudaGraphExec_t graph = nullptr;
  int graph_shape = -1;
  // timing
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  bool timed = false;
};

namespace {

int ensure_pinned(void **p, size_t bytes) {
  if (*p) cublox_b200::detail::hfree(*p);
  *p = nullptr;
  if (cublox_b200::detail::hmalloc(p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(CUBLOX_ERR_NOMEM, "batch: pinned allocation failed");
  }
  return CUBLOX_OK;
}

int ensure_dev(void **p, size_t bytes) {
  cublox_b200::detail::dfree(*p);
  *p = nullptr;
  if (cublox_b200::detail::dmalloc(p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(CUBLOX_ERR_NOMEM, "batch: device allocation failed");
  }
  return CUBLOX_OK;
}

void drop_graph(cublox_batch *b);

int ensure_capacity(cublox_batch *b, int n_maps, int n_witems, int n_fitems) {
  if (n_maps > b->maps_cap || n_witems > b->witems_cap || n_fitems > b->fitems_cap) {
    if (b->staged) cudaEventSynchronize(b->staged);
    cudaStreamSynchronize(b->stream);
    const int mc = std::max(n_maps, 2 * b->maps_cap);
    const int wc = std::max(n_witems, 2 * b->witems_cap);
    const int fc = std::max(n_fitems, 2 * b->fitems_cap);
    int rc;
    if ((rc = ensure_dev(reinterpret_cast<void **>(&b->d_maps), sizeof(MapDesc) * mc)) ||
        (rc = ensure_dev(reinterpret_cast<void **>(&b->d_done), sizeof(int) * mc)) ||
        (rc = ensure_dev(reinterpret_cast<void **>(&b->d_witems), sizeof(WalkItem) * wc)) ||
        (rc = ensure_dev(reinterpret_cast<void **>(&b->d_fitems), sizeof(FoldItem) * fc)) ||
        (rc = ensure_pinned(reinterpret_cast<void **>(&b->h_maps), sizeof(MapDesc) * mc)) ||
        (rc = ensure_pinned(reinterpret_cast<void **>(&b->h_witems), sizeof(WalkItem) * wc)) ||
        (rc = ensure_pinned(reinterpret_cast<void **>(&b->h_fitems), sizeof(FoldItem) * fc))) {
      // some buffers are gone: the next update sizes them all again
      b->maps_cap = b->witems_cap = b->fitems_cap = 0;
      drop_graph(b);
      return rc;
    }
    b->maps_cap = mc;
    b->witems_cap = wc;
    b->fitems_cap = fc;
    if (b->graph) {  // pointers changed: recapture
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
      b->graph_shape = -1;
    }
  }
  return CUBLOX_OK;
}

// Point staging (pinned) and device buffers for `floats` floats, grown
// geometrically: freeing memory waits for the whole device.
int reserve_points(cublox_batch *b, size_t floats) {
  int rc;
  if (floats > b->points_cap) {
    floats = std::max(floats, 2 * b->points_cap);
    cudaStreamSynchronize(b->stream);
    b->points_cap = 0;
    if ((rc = ensure_dev(reinterpret_cast<void **>(&b->d_points), floats * sizeof(float))))
      return rc;
    b->points_cap = floats;
  }
  if (floats > b->h_points_cap) {
    floats = std::max(floats, 2 * b->h_points_cap);
    cudaStreamSynchronize(b->stream);  // a walk may be reading the old buffer in place
    b->h_points_cap = 0;
    if ((rc = ensure_pinned(reinterpret_cast<void **>(&b->h_points), floats * sizeof(float))))
      return rc;
    b->h_points_cap = floats;
  }
  return CUBLOX_OK;
}

// The per-step launch sequence (captured into a graph when enabled, so it
// depends on nothing that changes between steps but the shape and the fold
// variant).  On failure *what names the call.
cudaError_t enqueue_step(cublox_batch *b, int shape, const char **what) {
  const Shape &sh = kShapes[shape];
  cudaError_t e;
  *what = "an earlier CUDA call left an error";
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  *what = "counter reset";
  if ((e = cudaMemsetAsync(b->d_counters, 0, sizeof(int), b->stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(b->d_counters + 2, 0, sizeof(int), b->stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(b->d_counters + 4, 0, sizeof(int), b->stream)) != cudaSuccess)
    return e;
  if ((sh.fused || sh.wq) &&
      (e = cudaMemsetAsync(b->d_done, 0, sizeof(int) * b->maps_cap, b->stream)) != cudaSuccess)
    return e;
  *what = "timing event";
  if (b->timed && (e = cudaEventRecord(b->ev[0], b->stream)) != cudaSuccess) return e;
  *what = sh.fused ? "fused walk+fold launch" : "walk launch";
  if ((e = launch_walk(b->d_maps, b->d_witems, b->d_fitems, b->d_counters, b->d_done, shape,
                       b->stream)) != cudaSuccess)
    return e;
  *what = "timing event";
  if (b->timed && (e = cudaEventRecord(b->ev[1], b->stream)) != cudaSuccess) return e;
  if (!sh.fused) {
    *what = "fold launch";
    if ((e = launch_fold(b->d_maps, b->d_fitems, b->d_counters, b->fold_variant, b->stream)) !=
        cudaSuccess)
      return e;
  }
  *what = "timing event";
  if (b->timed && (e = cudaEventRecord(b->ev[2], b->stream)) != cudaSuccess) return e;
  return cudaSuccess;
}

void drop_graph(cublox_batch *b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  b->graph_shape = -1;
}

}  // namespace

extern "C" {

int cublox_batch_create(void *stream, cublox_batch **out) {
  if (!out) return fail(CUBLOX_ERR_INVALID, "batch_create: null argument");
  *out = nullptr;
  cublox_batch *b = new cublox_batch();
  if (stream) {
    b->stream = static_cast<cudaStream_t>(stream);
  } else {
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      delete b;
      return fail(CUBLOX_ERR_CUDA, "batch_create: stream creation failed");
    }
    b->own_stream = true;
  }
  if (cublox_b200::detail::dmalloc(&b->d_counters, sizeof(int) * kCounters) != cudaSuccess ||
      cublox_b200::detail::hmalloc(&b->h_counters, sizeof(int) * kCounters) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->staged, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->points_read, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    delete b;
    return fail(CUBLOX_ERR_NOMEM, "batch_create: allocation failed");
  }
  for (int i = 0; i < 4; ++i) cudaEventCreate(&b->ev[i]);
  for (int i = 0; i < kNumShapes; ++i) shape_grid(i);
  *out = b;
  return CUBLOX_OK;
}

int cublox_batch_destroy(cublox_batch *b) {
  if (!b) return CUBLOX_OK;
  cudaStreamSynchronize(b->stream);
  for (cublox_grid *g : b->grids) cublox_grid_destroy(g);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  cublox_b200::detail::dfree(b->d_maps);
  cublox_b200::detail::dfree(b->d_witems);
  cublox_b200::detail::dfree(b->d_fitems);
  cublox_b200::detail::dfree(b->d_counters);
  cublox_b200::detail::dfree(b->d_done);
  cublox_b200::detail::dfree(b->d_points);
  if (b->h_maps) cublox_b200::detail::hfree(b->h_maps);
  if (b->h_witems) cublox_b200::detail::hfree(b->h_witems);
  if (b->h_fitems) cublox_b200::detail::hfree(b->h_fitems);
  if (b->h_counters) cublox_b200::detail::hfree(b->h_counters);
  if (b->h_points) cublox_b200::detail::hfree(b->h_points);
  if (b->staged) cudaEventDestroy(b->staged);
  if (b->points_read) cudaEventDestroy(b->points_read);
  for (int i = 0; i < 4; ++i)
    if (b->ev[i]) cudaEventDestroy(b->ev[i]);
  if (b->own_stream) cudaStreamDestroy(b->stream);
  delete b;
  return CUBLOX_OK;
}

int cublox_batch_add_grid(cublox_batch *b, const int half_map_size[3], float resolution,
                          int origin_at_center, int has_recenter_threshold,
                          double recenter_threshold, const float origin[3], cublox_grid **out) {
  if (!b || !out) return fail(CUBLOX_ERR_INVALID, "batch_add_grid: null argument");
  int rc = cublox_grid_create(half_map_size, resolution, origin_at_center,
                              has_recenter_threshold, recenter_threshold, origin, b->stream, out);
  if (rc) return rc;
  b->grids.push_back(*out);
  return CUBLOX_OK;
}

int cublox_batch_set_option(cublox_batch *b, int key, int value) {
  if (!b) return fail(CUBLOX_ERR_INVALID, "null batch");
  switch (key) {
    case CUBLOX_BATCH_OPT_GRAPHS:
      b->graphs = value != 0;
      return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_AUTOTUNE:
      b->autotune = value != 0;
      b->tune_step = 0;
      b->tune_ms.clear();
      return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_SHAPE:
      if (value < 0 || value >= kNumShapes) break;
      b->shape = value;
      b->autotune = false;
      return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_LAYOUT:
      if (!detail::layout_valid(value)) break;
      b->layout = value;
      b->autotune = false;
      return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_WAIT_LIMIT:
      if (value < 1) break;
      b->wait_limit = value;
      return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_INJECT_MISSING_WALK:
      b->inject_missing_walk = value != 0;
      return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_TIMING:
      b->timed = value != 0;
      return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_HOST_READ:
      b->host_read = value != 0;
      return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_FOLD:
      if (value < 0 || value > 2) break;
      b->fold_variant = value;
      drop_graph(b);
      return CUBLOX_OK;
    default:
      break;
  }
  return fail(CUBLOX_ERR_INVALID, "batch_set_option: unknown key or value");
}

int cublox_batch_get_option(const cublox_batch *b, int key, int *value) {
  if (!b || !value) return fail(CUBLOX_ERR_INVALID, "null argument");
  switch (key) {
    case CUBLOX_BATCH_OPT_GRAPHS: *value = b->graphs; return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_AUTOTUNE: *value = b->autotune; return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_SHAPE: *value = b->shape; return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_LAYOUT: *value = b->layout; return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_WAIT_LIMIT: *value = b->wait_limit; return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_INJECT_MISSING_WALK: *value = b->inject_missing_walk; return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_TIMING: *value = b->timed; return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_HOST_READ: *value = b->host_read; return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_NUM_SHAPES: *value = kNumShapes; return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_FOLD: *value = b->fold_variant; return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_TUNING:
      *value = b->autotune && b->tune_step < kNumCandidates * b->tune_rounds;
      return CUBLOX_OK;
    default: break;
  }
  return fail(CUBLOX_ERR_INVALID, "batch_get_option: unknown key");
}

int cublox_batch_update(cublox_batch *b, int n, cublox_grid *const *grids, const float *xyz,
                        const int64_t *offsets, const float *sensors) {
  if (!b || (n > 0 && (!grids || !xyz || !offsets || !sensors)))
    return fail(CUBLOX_ERR_INVALID, "batch_update: null argument");
  if (n <= 0) return CUBLOX_OK;
  for (int i = 0; i < n; ++i) {
    if (!grids[i]) return fail(CUBLOX_ERR_INVALID, "batch_update: null grid");
    if (grids[i]->stream != b->stream)
      return fail(CUBLOX_ERR_INVALID, "batch_update: grid not created by this batch");
    if (offsets[i + 1] < offsets[i]) return fail(CUBLOX_ERR_INVALID, "batch_update: bad offsets");
    for (int j = 0; j < i; ++j)
      if (grids[j] == grids[i])
        return fail(CUBLOX_ERR_INVALID, "batch_update: a grid appears twice in one update");
  }
  const int64_t total = offsets[n] - offsets[0];
  if (total <= 0) return CUBLOX_OK;  // every scan empty: nothing changes
  const bool tuning = b->autotune && b->tune_step < kNumCandidates * b->tune_rounds;
  const int cand = tuning ? (b->tune_step / b->tune_rounds) % kNumCandidates : -1;
  const int active_shape = tuning ? kCandidates[cand].shape : b->shape;
  const int active_layout = tuning ? kCandidates[cand].layout : b->layout;
  // the grids' voxel layout (moved between scans, on the batch's stream)
  for (int i = 0; i < n; ++i) {
    if (grids[i]->lay_code == active_layout) continue;
    const int rc = detail::set_layout(grids[i], active_layout);
    if (rc) return rc;
  }
  const Shape &sh = kShapes[active_shape];
  const int rays_per_item = shape_rays(active_shape, total);
  // work items
  int n_w = 0, n_f = 0;
  for (int i = 0; i < n; ++i) {
    const int64_t c = offsets[i + 1] - offsets[i];
    n_w += static_cast<int>((c + rays_per_item - 1) / rays_per_item);
    n_f += (grids[i]->nlines + kFoldItemLines - 1) / kFoldItemLines;
  }
  // a fused shape queues walk and fold items in one list
  int rc = ensure_capacity(b, n, std::max(sh.fused ? n_w + n_f : n_w, 1), std::max(n_f, 1));
  if (rc) return rc;
  // points: one concatenated x0 y0 z0 ... buffer, host or device
  cudaPointerAttributes pa;
  const float *base = xyz + 3 * offsets[0];
  bool on_device = false, staged_read = false;
  if (cudaPointerGetAttributes(&pa, xyz) == cudaSuccess)
    on_device = pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged;
  else
    cudaGetLastError();
  // The pinned staging buffers are reused: wait until the last step's
  // copies out of them have run.
  if (cudaEventSynchronize(b->staged) != cudaSuccess) cudaGetLastError();
  if (!on_device && total > 0) {
    const size_t floats = 3 * static_cast<size_t>(total);
    const bool pinned = pa.type == cudaMemoryTypeHost && pa.devicePointer != nullptr;
    if (b->host_read && pinned) {
      // the walk reads the caller's pinned points over the bus, each once,
      // while it runs: no copy ahead of the launch
      base = static_cast<const float *>(pa.devicePointer) + 3 * offsets[0];
    } else {
      if ((rc = reserve_points(b, floats))) return rc;
      const float *src = base;
      if (!pinned) {
        // a walk that read the staged points in place must be done with them
        if (cudaEventSynchronize(b->points_read) != cudaSuccess) cudaGetLastError();
        std::memcpy(b->h_points, base, floats * sizeof(float));
        src = b->h_points;
      }
      if (b->host_read) {
        base = b->h_points;  // staged in pinned memory, read in place by the walk
        staged_read = true;
      } else {
        cudaError_t e = cudaMemcpyAsync(b->d_points, src, floats * sizeof(float),
                                        cudaMemcpyHostToDevice, b->stream);
        if (e != cudaSuccess) return cuda_fail(e, "batch points copy", __LINE__);
        base = b->d_points;
      }
    }
  }
  // descriptors and items; an empty scan leaves its grid untouched, as
  // cublox_grid_update does (OccupancyGrid.cpp:183-190)
  int w = 0, f = 0, d = 0;
  auto &w_end = b->w_end, &f_end = b->f_end;  // per map: end of its walk / fold items
  w_end.clear();
  f_end.clear();
  for (int i = 0; i < n; ++i) {
    cublox_grid *g = grids[i];
    const int64_t off = offsets[i] - offsets[0];
    const int c = static_cast<int>(offsets[i + 1] - offsets[i]);
    if (c <= 0 || g->voxel_num <= 0) continue;
    detail::snap_first_run(g, sensors + 3 * i);
    MapDesc &md = b->h_maps[d];
    const float *px = base + 3 * off;
    md.ray = detail::ray_params(g, px, px + 1, px + 2, c, 3, sensors + 3 * i);
    if (g->stats_on) cudaMemsetAsync(g->d_stats, 0, 4 * sizeof(unsigned long long), b->stream);
    md.occ = g->d_occ;
    md.l_hit = g->l_hit;
    md.l_miss = g->l_miss;
    md.l_min = g->l_min;
    md.l_max = g->l_max;
    md.l_unknown = g->l_unknown;
    for (int a = 0; a < 3; ++a)
      md.clo[a] = pos_to_global_dev(sensors[3 * i + a], g->res_inv, g->ctr, g->fp) -
                  (a == 2 && sh.flat ? sh.cube / 4 : sh.cube / 2);
    md.n_walk = 0;
    for (int s0 = 0; s0 < c; s0 += rays_per_item, ++md.n_walk)
      b->h_witems[w++] = WalkItem{d, s0, std::min(rays_per_item, c - s0), 0};
    for (int l0 = 0; l0 < g->nlines; l0 += kFoldItemLines)
      b->h_fitems[f++] = FoldItem{d, l0, std::min(kFoldItemLines, g->nlines - l0), 0};
    // test hook: the map's folds wait for one walk item more than it has,
    // so a fused launch's bounded wait runs out (the walk items themselves
    // are unchanged)
    if (b->inject_missing_walk && d == 0) ++md.n_walk;
    w_end.push_back(w);
    f_end.push_back(f);
    ++d;
  }
  if (sh.fused) {
    // with lag L = sh.fused: walk(0) .. walk(L) fold(0) walk(L + 1) fold(1)
    // ... walk(d - 1) fold(d - 1 - L) .. fold(d - 1)
    const int lag = sh.fused;
    auto &order = b->order;
    order.clear();
    auto put_walk = [&](int map) {
      for (int i = map ? w_end[map - 1] : 0; i < w_end[map]; ++i) order.push_back(b->h_witems[i]);
    };
    auto put_fold = [&](int map) {
      for (int i = map ? f_end[map - 1] : 0; i < f_end[map]; ++i) {
        const FoldItem &fi = b->h_fitems[i];
        order.push_back(WalkItem{~fi.map, fi.start, fi.count, fi.pad});
      }
    };
    for (int map = 0; map < d; ++map) {
      put_walk(map);
      if (map >= lag) put_fold(map - lag);
    }
    for (int map = std::max(0, d - lag); map < d; ++map) put_fold(map);
    std::copy(order.begin(), order.end(), b->h_witems);
    w = static_cast<int>(order.size());
    f = 0;
  }
  b->h_counters[0] = b->h_counters[2] = b->h_counters[4] = 0;
  b->h_counters[5] = b->wait_limit;
  b->h_counters[1] = sh.wq ? d : w;  // the warp-queue walk reads maps, not items
  b->h_counters[3] = f;
  cudaError_t e;
  if ((e = cudaMemcpyAsync(b->d_maps, b->h_maps, sizeof(MapDesc) * d, cudaMemcpyHostToDevice,
                           b->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(b->d_witems, b->h_witems, sizeof(WalkItem) * w,
                           cudaMemcpyHostToDevice, b->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(b->d_fitems, b->h_fitems, sizeof(FoldItem) * f,
                           cudaMemcpyHostToDevice, b->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(b->d_counters, b->h_counters, sizeof(int) * kCounters,
                           cudaMemcpyHostToDevice, b->stream)) != cudaSuccess)
    return cuda_fail(e, "batch descriptor copy", __LINE__);
  if ((e = cudaEventRecord(b->staged, b->stream)) != cudaSuccess)
    return cuda_fail(e, "batch staging event", __LINE__);
  // launch: tuning steps are timed, the rest replayed from a graph if asked
  const bool timed_before = b->timed;
  if (tuning) b->timed = true;
  if (b->graphs && !tuning && !b->timed) {
    if (!b->graph || b->graph_shape != active_shape) {
      drop_graph(b);
      cudaGraph_t gr;
      if ((e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
        return cuda_fail(e, "batch graph capture", __LINE__);
      const char *what = "";
      cudaError_t le = enqueue_step(b, active_shape, &what);
      e = cudaStreamEndCapture(b->stream, &gr);
      if (le != cudaSuccess)
        return cuda_fail(le, (std::string("batch graph capture: ") + what).c_str(), __LINE__);
      if (e != cudaSuccess) return cuda_fail(e, "batch graph end capture", __LINE__);
      e = cudaGraphInstantiate(&b->graph, gr, 0);
      detail::count(detail::kGraphBuilds);
      cudaGraphDestroy(gr);
      if (e != cudaSuccess) return cuda_fail(e, "batch graph instantiate", __LINE__);
      b->graph_shape = active_shape;
    }
    if ((e = cudaGraphLaunch(b->graph, b->stream)) != cudaSuccess)
      return cuda_fail(e, "batch graph launch", __LINE__);
  } else {
    const char *what = "";
    if ((e = enqueue_step(b, active_shape, &what)) != cudaSuccess)
      return cuda_fail(e, (std::string("batch step (shape ") + std::to_string(active_shape) +
                           "): " + what).c_str(), __LINE__);
  }
  b->timed = timed_before;
  if (staged_read && (e = cudaEventRecord(b->points_read, b->stream)) != cudaSuccess)
    return cuda_fail(e, "batch staging event", __LINE__);
  if (tuning) {
    float ms = 0.0f;  // walk + fold
    cudaEventSynchronize(b->ev[2]);
    cudaEventElapsedTime(&ms, b->ev[0], b->ev[2]);
    if (static_cast<int>(b->tune_ms.size()) < kNumCandidates)
      b->tune_ms.assign(kNumCandidates, 0.0f);
    b->tune_ms[cand] += ms;
    ++b->tune_step;
    if (b->tune_step >= kNumCandidates * b->tune_rounds) {
      int best = 0;
      for (int c = 1; c < kNumCandidates; ++c)
        if (b->tune_ms[c] < b->tune_ms[best]) best = c;
      b->shape = kCandidates[best].shape;
      b->layout = kCandidates[best].layout;
    }
  }
  return CUBLOX_OK;
}

int cublox_batch_reserve(cublox_batch *b, int64_t points, int maps) {
  if (!b || points < 0 || maps < 0) return fail(CUBLOX_ERR_INVALID, "batch_reserve: bad argument");
  if (cudaEventSynchronize(b->staged) != cudaSuccess) cudaGetLastError();
  int rc = reserve_points(b, 3 * static_cast<size_t>(points));
  if (rc) return rc;
  const int items = maps + static_cast<int>(points / 256) + 1;
  return ensure_capacity(b, std::max(maps, 1), items + maps * 64, maps * 64 + 1);
}

int cublox_batch_reserve_maps(cublox_batch *b, int64_t points, int maps, int64_t voxels) {
  if (!b || points < 0 || maps < 0 || voxels < 0)
    return fail(CUBLOX_ERR_INVALID, "batch_reserve_maps: bad argument");
  if (cudaEventSynchronize(b->staged) != cudaSuccess) cudaGetLastError();
  int rc = reserve_points(b, 3 * static_cast<size_t>(points));
  if (rc) return rc;
  // fold items: per map ceil(voxels / 4 / groups per item) + 1 (the tail
  // item); walk items: at least 256 rays each (every shape), one partial
  // item per map, and a fused shape queues the fold items behind them
  const int64_t folds = voxels / (32 * static_cast<int64_t>(kFoldItemLines)) + 2 * maps + 1;
  const int64_t walks = points / 256 + maps + 1;
  if (folds + walks > (int64_t(1) << 30))
    return fail(CUBLOX_ERR_INVALID, "batch_reserve_maps: too many work items");
  return ensure_capacity(b, std::max(maps, 1), static_cast<int>(walks + folds),
                         static_cast<int>(folds));
}

int cublox_batch_recenter(cublox_batch *b, int n, cublox_grid *const *grids,
                          const float *positions, int *actions) {
  if (!b || (n > 0 && (!grids || !positions)))
    return fail(CUBLOX_ERR_INVALID, "batch_recenter: null argument");
  for (int i = 0; i < n; ++i) {
    int a = 0;
    const int rc = cublox_grid_recenter(grids[i], positions + 3 * i, &a);
    if (rc) return rc;
    if (actions) actions[i] = a;
  }
  return CUBLOX_OK;
}

int cublox_batch_synchronize(cublox_batch *b) {
  if (!b) return fail(CUBLOX_ERR_INVALID, "null batch");
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return cuda_fail(e, "batch synchronize", __LINE__);
  return CUBLOX_OK;
}

int cublox_batch_last_timing(cublox_batch *b, float *walk_ms, float *fold_ms) {
  if (!b) return fail(CUBLOX_ERR_INVALID, "null batch");
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return cuda_fail(e, "batch timing", __LINE__);
  if (walk_ms) cudaEventElapsedTime(walk_ms, b->ev[0], b->ev[1]);
  if (fold_ms) cudaEventElapsedTime(fold_ms, b->ev[1], b->ev[2]);
  return CUBLOX_OK;
}

int cublox_batch_stream(const cublox_batch *b, void **stream) {
  if (!b || !stream) return fail(CUBLOX_ERR_INVALID, "null argument");
  *stream = b->stream;
  return CUBLOX_OK;
}

}  // extern "C"

// Batched integration: scans of many grids in one walk launch and one fold
// launch (include/cublox_b200.h, cublox_batch_*).
//
//  walk  persistent CTAs take work items — a contiguous run of one map's
//        rays — from a device queue.  A CTA zeroes an S^3 shared-memory cube
//        centred on that map's sensor voxel, walks the run (one thread per
//        ray, the exact walk of ray_walk.cuh), and flushes the cube into the
//        map's counters.  Points are read in place from one concatenated
//        x0 y0 z0 x1 ... buffer.
//  fold  persistent CTAs take (map, voxel range) items and fold counters
//        into stored log-odds with 16-byte accesses.
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
#include "grid_internal.hpp"
#include "kernels.cuh"
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
  int pad;
};

struct WalkItem {
  int map, start, count, pad;
};

struct FoldItem {
  int map, g4_start, g4_count, tail;  // tail: handle the vnum % 4 voxels
};

// counters: [0] walk queue, [1] walk items, [2] fold queue, [3] fold items
constexpr int kCounters = 4;

template <int S>
__device__ __forceinline__ void emit(const RayParams &p, uint32_t *cube, const int clo[3],
                                     int g0, int g1, int g2, int h) {
  const int c0 = g0 - clo[0], c1 = g1 - clo[1], c2 = g2 - clo[2];
  if (S > 0 && static_cast<unsigned>(c0) < static_cast<unsigned>(S) &&
      static_cast<unsigned>(c1) < static_cast<unsigned>(S) &&
      static_cast<unsigned>(c2) < static_cast<unsigned>(S))
    atomicAdd(&cube[(c0 * S + c1) * S + c2], 1u);
  else
    atomicAdd(p.cnt + h, 1u);
}

template <int S>
__global__ void __launch_bounds__(1024) batch_walk_kernel(const MapDesc *maps,
                                                          const WalkItem *items,
                                                          int *counters) {
  extern __shared__ uint32_t cube[];
  constexpr int kCube = S * S * S;
  __shared__ int s_item;
  const int n_items = counters[1];
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(&counters[0], 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n_items) break;
    const WalkItem item = items[it];
    const MapDesc &md = maps[item.map];
    const RayParams p = md.ray;
    const int clo[3] = {md.clo[0], md.clo[1], md.clo[2]};
    for (int q = threadIdx.x; q < kCube / 4; q += blockDim.x)
      reinterpret_cast<uint4 *>(cube)[q] = make_uint4(0u, 0u, 0u, 0u);
    __syncthreads();
    uint32_t rays = 0, incs = 0, hits = 0;
    for (int i = item.start + threadIdx.x; i < item.start + item.count; i += blockDim.x) {
      const size_t k = static_cast<size_t>(i) * p.stride;
      RayWalk w;
      if (!ray_begin(p, p.x[k], p.y[k], p.z[k], w)) continue;
      ++rays;
      for (int step = 0; step < w.max_steps; ++step) {
        if (at_end(w)) break;
        if (in_window(w, p)) {
          emit<S>(p, cube, clo, w.id[0], w.id[1], w.id[2], walk_hash(w, p));
          ++incs;
        } else if (left_for_good(w, p)) {
          break;
        }
        ray_step(w, p);
      }
      const int h = end_hash(w, p);
      if (h >= 0) {
        emit<S>(p, cube, clo, w.en[0], w.en[1], w.en[2], h);
        ++incs;
        if (!w.clipped) {
          atomicOr(p.cnt + h, kHitFlag);
          atomicAdd(p.hit + h, 1u);
          ++hits;
        }
      }
    }
    __syncthreads();
    if constexpr (S > 0) {
      for (int q = threadIdx.x; q < kCube; q += blockDim.x) {
        const uint32_t v = cube[q];
        if (!v) continue;
        const int g[3] = {clo[0] + q / (S * S), clo[1] + (q / S) % S, clo[2] + q % S};
        const int h = ((global_to_local(g[0], p.map[0], p.half[0]) + p.half[0]) * p.map[1] +
                       (global_to_local(g[1], p.map[1], p.half[1]) + p.half[1])) *
                          p.map[2] +
                      (global_to_local(g[2], p.map[2], p.half[2]) + p.half[2]);
        atomicAdd(p.cnt + h, v);
      }
    }
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
}

__device__ __forceinline__ float fold_one(const MapDesc &m, int h, uint32_t c, float s0) {
  const int op = static_cast<int>(c & kOpMask);
  int hit = 0;
  if (c & kHitFlag) {
    hit = static_cast<int>(m.ray.hit[h]);
    m.ray.hit[h] = 0u;
  }
  const int miss = op > hit ? op - hit : 0;
  const unsigned fp = m.ray.fp;
  float l = fadd(s0, m.l_unknown);
  l = (fp & kFpMissFma) ? ffma(m.l_miss, static_cast<float>(miss), l)
                        : fadd(l, fmul(m.l_miss, static_cast<float>(miss)));
  l = (fp & kFpHitFma) ? ffma(m.l_hit, static_cast<float>(hit), l)
                       : fadd(l, fmul(m.l_hit, static_cast<float>(hit)));
  if (l < m.l_min) l = m.l_min;
  if (l > m.l_max) l = m.l_max;
  return fsub(l, m.l_unknown);
}

__global__ void __launch_bounds__(256) batch_fold_kernel(const MapDesc *maps,
                                                         const FoldItem *items,
                                                         int *counters) {
  __shared__ int s_item;
  const int n_items = counters[3];
  uint32_t touched = 0;
  unsigned long long *stats = nullptr;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(&counters[2], 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= n_items) break;
    const FoldItem item = items[it];
    const MapDesc &m = maps[item.map];
    stats = m.ray.stats;
    uint4 *c4 = reinterpret_cast<uint4 *>(m.ray.cnt);
    float4 *o4 = reinterpret_cast<float4 *>(m.occ);
    const int g_end = item.g4_start + item.g4_count;
    for (int i0 = item.g4_start + threadIdx.x; i0 < g_end; i0 += 4 * blockDim.x) {
      uint4 c[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int i = i0 + u * blockDim.x;
        c[u] = i < g_end ? c4[i] : make_uint4(0u, 0u, 0u, 0u);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if ((c[u].x | c[u].y | c[u].z | c[u].w) == 0u) continue;
        const int i = i0 + u * blockDim.x;
        const int h = i << 2;
        float4 o = o4[i];
        if (c[u].x) { o.x = fold_one(m, h + 0, c[u].x, o.x); ++touched; }
        if (c[u].y) { o.y = fold_one(m, h + 1, c[u].y, o.y); ++touched; }
        if (c[u].z) { o.z = fold_one(m, h + 2, c[u].z, o.z); ++touched; }
        if (c[u].w) { o.w = fold_one(m, h + 3, c[u].w, o.w); ++touched; }
        o4[i] = o;
        c4[i] = make_uint4(0u, 0u, 0u, 0u);
      }
    }
    if (item.tail && threadIdx.x < (m.ray.vnum & 3)) {
      const int h = ((m.ray.vnum >> 2) << 2) + threadIdx.x;
      const uint32_t c = m.ray.cnt[h];
      if (c) {
        m.occ[h] = fold_one(m, h, c, m.occ[h]);
        m.ray.cnt[h] = 0u;
        ++touched;
      }
    }
    if (stats) {
      uint32_t t = touched;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
      if ((threadIdx.x & 31) == 0 && t) atomicAdd(stats + 3, static_cast<unsigned long long>(t));
    }
    touched = 0;
  }
}

struct Shape {
  int cube;   // 0, 16, 32
  int rays;   // rays per work item
  int block;  // walk CTA size
};

const Shape kShapes[] = {{32, 1024, 512}, {16, 512, 256}, {32, 2048, 1024},
                         {0, 1024, 512},  {32, 512, 512}, {16, 1024, 512}};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

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

// Resident CTAs per SM of batch_walk_kernel<S> at a CTA size; sets the
// shared-memory attribute on first use.  Called for every shape before any
// graph capture, so capture itself only enqueues launches.
template <int S>
int walk_ctas_per_sm(int block) {
  static int cached[3] = {0, 0, 0};  // block 256, 512, 1024
  const int slot = block >= 1024 ? 2 : (block >= 512 ? 1 : 0);
  if (cached[slot] == 0) {
    const size_t smem = sizeof(uint32_t) * S * S * S;
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(batch_walk_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(smem));
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_walk_kernel<S>, block,
                                                      smem) != cudaSuccess) {
      cudaGetLastError();
      per_sm = 1;
    }
    cached[slot] = per_sm < 1 ? 1 : per_sm;
  }
  return cached[slot];
}

template <int S>
cudaError_t launch_batch_walk(const MapDesc *maps, const WalkItem *items, int *counters,
                              int block, cudaStream_t s) {
  const size_t smem = sizeof(uint32_t) * S * S * S;
  batch_walk_kernel<S><<<sm_count_batch() * walk_ctas_per_sm<S>(block), block, smem, s>>>(
      maps, items, counters);
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
  // shape choice
  int shape = 0;
  bool autotune = true;
  int tune_step = 0;
  int tune_rounds = 2;
  std::vector<float> tune_ms;
  bool graphs = false;
  cudaGraphExec_t graph = nullptr;
  int graph_shape = -1;
  // timing
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  bool timed = false;
};

namespace {

int ensure_pinned(void **p, size_t bytes) {
  if (*p) cudaFreeHost(*p);
  *p = nullptr;
  if (cudaMallocHost(p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(CUBLOX_ERR_NOMEM, "batch: pinned allocation failed");
  }
  return CUBLOX_OK;
}

int ensure_dev(void **p, size_t bytes) {
  cudaFree(*p);
  *p = nullptr;
  if (cudaMalloc(p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(CUBLOX_ERR_NOMEM, "batch: device allocation failed");
  }
  return CUBLOX_OK;
}

int ensure_capacity(cublox_batch *b, int n_maps, int n_witems, int n_fitems) {
  if (n_maps > b->maps_cap || n_witems > b->witems_cap || n_fitems > b->fitems_cap) {
    if (b->staged) cudaEventSynchronize(b->staged);
    cudaStreamSynchronize(b->stream);
    const int mc = std::max(n_maps, 2 * b->maps_cap);
    const int wc = std::max(n_witems, 2 * b->witems_cap);
    const int fc = std::max(n_fitems, 2 * b->fitems_cap);
    int rc;
    if ((rc = ensure_dev(reinterpret_cast<void **>(&b->d_maps), sizeof(MapDesc) * mc)) ||
        (rc = ensure_dev(reinterpret_cast<void **>(&b->d_witems), sizeof(WalkItem) * wc)) ||
        (rc = ensure_dev(reinterpret_cast<void **>(&b->d_fitems), sizeof(FoldItem) * fc)) ||
        (rc = ensure_pinned(reinterpret_cast<void **>(&b->h_maps), sizeof(MapDesc) * mc)) ||
        (rc = ensure_pinned(reinterpret_cast<void **>(&b->h_witems), sizeof(WalkItem) * wc)) ||
        (rc = ensure_pinned(reinterpret_cast<void **>(&b->h_fitems), sizeof(FoldItem) * fc)))
      return rc;
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

// The per-step launch sequence (captured into a graph when enabled).
cudaError_t enqueue_step(cublox_batch *b, int shape) {
  const Shape &sh = kShapes[shape];
  cudaError_t e = cudaMemsetAsync(b->d_counters, 0, sizeof(int), b->stream);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(b->d_counters + 2, 0, sizeof(int), b->stream);
  if (e != cudaSuccess) return e;
  if (b->timed) cudaEventRecord(b->ev[0], b->stream);
  if (sh.cube >= 32)
    e = launch_batch_walk<32>(b->d_maps, b->d_witems, b->d_counters, sh.block, b->stream);
  else if (sh.cube >= 16)
    e = launch_batch_walk<16>(b->d_maps, b->d_witems, b->d_counters, sh.block, b->stream);
  else
    e = launch_batch_walk<0>(b->d_maps, b->d_witems, b->d_counters, sh.block, b->stream);
  if (e != cudaSuccess) return e;
  if (b->timed) cudaEventRecord(b->ev[1], b->stream);
  batch_fold_kernel<<<sm_count_batch() * 8, 256, 0, b->stream>>>(b->d_maps, b->d_fitems,
                                                                 b->d_counters);
  e = cudaGetLastError();
  if (b->timed) cudaEventRecord(b->ev[2], b->stream);
  return e;
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
  if (cudaMalloc(&b->d_counters, sizeof(int) * kCounters) != cudaSuccess ||
      cudaMallocHost(&b->h_counters, sizeof(int) * kCounters) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->staged, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    delete b;
    return fail(CUBLOX_ERR_NOMEM, "batch_create: allocation failed");
  }
  for (int i = 0; i < 4; ++i) cudaEventCreate(&b->ev[i]);
  sm_count_batch();
  for (const Shape &sh : kShapes) {
    if (sh.cube >= 32)
      walk_ctas_per_sm<32>(sh.block);
    else if (sh.cube >= 16)
      walk_ctas_per_sm<16>(sh.block);
    else
      walk_ctas_per_sm<0>(sh.block);
  }
  *out = b;
  return CUBLOX_OK;
}

int cublox_batch_destroy(cublox_batch *b) {
  if (!b) return CUBLOX_OK;
  cudaStreamSynchronize(b->stream);
  for (cublox_grid *g : b->grids) cublox_grid_destroy(g);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  cudaFree(b->d_maps);
  cudaFree(b->d_witems);
  cudaFree(b->d_fitems);
  cudaFree(b->d_counters);
  cudaFree(b->d_points);
  if (b->h_maps) cudaFreeHost(b->h_maps);
  if (b->h_witems) cudaFreeHost(b->h_witems);
  if (b->h_fitems) cudaFreeHost(b->h_fitems);
  if (b->h_counters) cudaFreeHost(b->h_counters);
  if (b->h_points) cudaFreeHost(b->h_points);
  if (b->staged) cudaEventDestroy(b->staged);
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
    case CUBLOX_BATCH_OPT_TIMING:
      b->timed = value != 0;
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
    case CUBLOX_BATCH_OPT_TIMING: *value = b->timed; return CUBLOX_OK;
    case CUBLOX_BATCH_OPT_NUM_SHAPES: *value = kNumShapes; return CUBLOX_OK;
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
  const int shape = b->autotune ? (b->tune_step / b->tune_rounds) % kNumShapes : b->shape;
  const bool tuning = b->autotune && b->tune_step < kNumShapes * b->tune_rounds;
  const int active_shape = tuning ? shape : b->shape;
  const Shape &sh = kShapes[active_shape];
  // work items
  int n_w = 0, n_f = 0;
  for (int i = 0; i < n; ++i) {
    const int64_t c = offsets[i + 1] - offsets[i];
    n_w += static_cast<int>((c + sh.rays - 1) / sh.rays);
    const int64_t g4 = grids[i]->voxel_num >> 2;
    n_f += static_cast<int>((g4 + (1 << 16) - 1) >> 16) + 1;
  }
  int rc = ensure_capacity(b, n, std::max(n_w, 1), std::max(n_f, 1));
  if (rc) return rc;
  // points: one concatenated x0 y0 z0 ... buffer, host or device
  cudaPointerAttributes pa;
  const float *base = xyz + 3 * offsets[0];
  bool on_device = false;
  if (cudaPointerGetAttributes(&pa, xyz) == cudaSuccess)
    on_device = pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged;
  else
    cudaGetLastError();
  // The pinned staging buffers are reused: wait until the last step's
  // copies out of them have run.
  if (cudaEventSynchronize(b->staged) != cudaSuccess) cudaGetLastError();
  if (!on_device && total > 0) {
    const size_t floats = 3 * static_cast<size_t>(total);
    if (floats > b->points_cap) {
      cudaStreamSynchronize(b->stream);
      if ((rc = ensure_dev(reinterpret_cast<void **>(&b->d_points), floats * sizeof(float))))
        return rc;
      b->points_cap = floats;
      if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
        b->graph_shape = -1;
      }
    }
    if (floats > b->h_points_cap) {
      if ((rc = ensure_pinned(reinterpret_cast<void **>(&b->h_points), floats * sizeof(float))))
        return rc;
      b->h_points_cap = floats;
    }
    if (pa.type != cudaMemoryTypeHost) {
      std::memcpy(b->h_points, base, floats * sizeof(float));
      cudaError_t e = cudaMemcpyAsync(b->d_points, b->h_points, floats * sizeof(float),
                                      cudaMemcpyHostToDevice, b->stream);
      if (e != cudaSuccess) return cuda_fail(e, "batch points copy", __LINE__);
    } else {
      cudaError_t e = cudaMemcpyAsync(b->d_points, base, floats * sizeof(float),
                                      cudaMemcpyHostToDevice, b->stream);
      if (e != cudaSuccess) return cuda_fail(e, "batch points copy", __LINE__);
    }
    base = b->d_points;
  }
  // descriptors and items; an empty scan leaves its grid untouched, as
  // cublox_grid_update does (OccupancyGrid.cpp:183-190)
  int w = 0, f = 0, d = 0;
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
      md.clo[a] = pos_to_global_dev(sensors[3 * i + a], g->res_inv, g->ctr, g->fp) - sh.cube / 2;
    md.pad = 0;
    for (int s0 = 0; s0 < c; s0 += sh.rays)
      b->h_witems[w++] = WalkItem{d, s0, std::min(sh.rays, c - s0), 0};
    const int g4 = g->voxel_num >> 2;
    for (int s0 = 0; s0 < g4 || (s0 == 0 && g4 == 0); s0 += (1 << 16)) {
      b->h_fitems[f++] = FoldItem{d, s0, std::min(1 << 16, g4 - s0), s0 == 0 ? 1 : 0};
      if (g4 == 0) break;
    }
    ++d;
  }
  b->h_counters[1] = w;
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
      if (b->graph) cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
      cudaGraph_t gr;
      if ((e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
        return cuda_fail(e, "batch graph capture", __LINE__);
      cudaError_t le = enqueue_step(b, active_shape);
      e = cudaStreamEndCapture(b->stream, &gr);
      if (le != cudaSuccess) return cuda_fail(le, "batch graph capture launch", __LINE__);
      if (e != cudaSuccess) return cuda_fail(e, "batch graph end capture", __LINE__);
      e = cudaGraphInstantiate(&b->graph, gr, 0);
      cudaGraphDestroy(gr);
      if (e != cudaSuccess) return cuda_fail(e, "batch graph instantiate", __LINE__);
      b->graph_shape = active_shape;
    }
    if ((e = cudaGraphLaunch(b->graph, b->stream)) != cudaSuccess)
      return cuda_fail(e, "batch graph launch", __LINE__);
  } else {
    if ((e = enqueue_step(b, active_shape)) != cudaSuccess)
      return cuda_fail(e, "batch step launch", __LINE__);
  }
  b->timed = timed_before;
  if (tuning) {
    float ms = 0.0f;
    cudaEventSynchronize(b->ev[1]);
    cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]);
    if (static_cast<int>(b->tune_ms.size()) < kNumShapes) b->tune_ms.assign(kNumShapes, 0.0f);
    b->tune_ms[active_shape] += ms;
    ++b->tune_step;
    if (b->tune_step >= kNumShapes * b->tune_rounds) {
      int best = 0;
      for (int s = 1; s < kNumShapes; ++s)
        if (b->tune_ms[s] < b->tune_ms[best]) best = s;
      b->shape = best;
    }
  }
  return CUBLOX_OK;
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

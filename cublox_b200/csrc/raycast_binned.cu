// Direction-binned raycast with near-sensor shared-memory staging (sm_100a).
//
// 1. bin:     each ray gets an octahedral direction bin (64 x 64, Morton
//             ordered) and the bins are counted;
// 2. scan:    exclusive scan of the 4096 bin counts (one block);
// 3. scatter: rays are written, bin by bin, into a sorted SoA copy;
// 4. walk:    each CTA takes a contiguous run of sorted rays (a compact cone
//             of directions), its warps walk 32 rays at a time in lockstep.
//             Every in-window voxel increment is keyed by its hash; lanes of
//             a warp holding the same voxel are merged with __match_any_sync
//             and one leader adds the group's count.  Increments inside an
//             S^3 cube around the sensor voxel — where every ray passes —
//             go to a shared-memory counter cube, flushed to the global
//             counters once per CTA; the rest go straight to the global
//             counters.  The walk itself is the exact one of ray_walk.cuh.
//
// Counts are integers, so the order rays are walked in cannot change them.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"
#include "far_walk.cuh"
#include "ray_walk.cuh"

namespace cublox_b200 {

namespace {

constexpr int kBinSide = 64;
constexpr int kBins = kBinSide * kBinSide;
constexpr uint32_t kNoKey = 0x80000000u;  // never a hash (hash < 2^31)

__device__ __forceinline__ uint32_t spread2(uint32_t v) {
  v &= 0xffffu;
  v = (v | (v << 8)) & 0x00ff00ffu;
  v = (v | (v << 4)) & 0x0f0f0f0fu;
  v = (v | (v << 2)) & 0x33333333u;
  v = (v | (v << 1)) & 0x55555555u;
  return v;
}

// Octahedral direction bin of (e - o); any bin for degenerate rays.
__device__ __forceinline__ int dir_bin(float dx, float dy, float dz) {
  const float s = fabsf(dx) + fabsf(dy) + fabsf(dz);
  if (!(s > 0.0f) || !isfinite(s)) return 0;
  float u = dx / s, v = dy / s;
  if (dz < 0.0f) {
    const float uu = (1.0f - fabsf(v)) * (u < 0.0f ? -1.0f : 1.0f);
    const float vv = (1.0f - fabsf(u)) * (v < 0.0f ? -1.0f : 1.0f);
    u = uu;
    v = vv;
  }
  int bu = static_cast<int>((u * 0.5f + 0.5f) * kBinSide);
  int bv = static_cast<int>((v * 0.5f + 0.5f) * kBinSide);
  bu = min(max(bu, 0), kBinSide - 1);
  bv = min(max(bv, 0), kBinSide - 1);
  return static_cast<int>(spread2(bu) | (spread2(bv) << 1));
}

__global__ void __launch_bounds__(256) bin_kernel(const RayParams p, int *bins,
                                                  int *hist) {
  __shared__ int sh[kBins];
  for (int i = threadIdx.x; i < kBins; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n;
       i += gridDim.x * blockDim.x) {
    const size_t k = static_cast<size_t>(i) * p.stride;
    const int b = dir_bin(p.x[k] - p.o[0], p.y[k] - p.o[1], p.z[k] - p.o[2]);
    bins[i] = b;
    atomicAdd(&sh[b], 1);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kBins; i += blockDim.x)
    if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// Exclusive scan of kBins counts by one block of 1024 threads.
__global__ void __launch_bounds__(1024) bin_scan_kernel(const int *hist, int *cursor) {
  __shared__ int part[1024];
  const int t = threadIdx.x;
  constexpr int per = kBins / 1024;
  int loc[per];
  int sum = 0;
#pragma unroll
  for (int k = 0; k < per; ++k) {
    loc[k] = hist[t * per + k];
    sum += loc[k];
  }
  part[t] = sum;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const int v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int run = part[t] - sum;
#pragma unroll
  for (int k = 0; k < per; ++k) {
    cursor[t * per + k] = run;
    run += loc[k];
  }
}

__global__ void __launch_bounds__(256) scatter_kernel(const RayParams p,
                                                      const int *bins, int *cursor,
                                                      float *sorted) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n;
       i += gridDim.x * blockDim.x) {
    const size_t k = static_cast<size_t>(i) * p.stride;
    const int d = atomicAdd(&cursor[bins[i]], 1);
    sorted[d] = p.x[k];
    sorted[p.n + d] = p.y[k];
    sorted[2 * static_cast<size_t>(p.n) + d] = p.z[k];
  }
}

// Lockstep walk of 32 sorted rays per warp chunk.
template <int S, bool kMatch>
__global__ void __launch_bounds__(512, 1) walk_kernel(const RayParams p, const int cl0,
                                                      const int cl1, const int cl2,
                                                      const int rays_per_cta) {
  extern __shared__ uint32_t cube[];
  constexpr int kCube = S * S * S;
  __shared__ int next;
  for (int i = threadIdx.x; i < kCube / 4; i += blockDim.x)
    reinterpret_cast<uint4 *>(cube)[i] = make_uint4(0u, 0u, 0u, 0u);
  if (threadIdx.x == 0) next = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int r0 = blockIdx.x * rays_per_cta;
  const int r1 = min(p.n, r0 + rays_per_cta);
  const int clo[3] = {cl0, cl1, cl2};
  uint32_t rays = 0, incs = 0, hits = 0;
  int last = -1;  // line this thread flagged last
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(&next, 32);
    base = __shfl_sync(0xffffffffu, base, 0) + r0;
    if (base >= r1) break;
    const int i = base + lane;
    RayWalk w;
    bool valid = false;
    if (i < r1) valid = ray_begin(p, p.x[i], p.y[i], p.z[i], w);
    bool alive = valid;
    int c[3] = {0, 0, 0};
    if (valid) {
      ++rays;
#pragma unroll
      for (int a = 0; a < 3; ++a) c[a] = w.id[a] - clo[a];
    }
    for (int step = 0;; ++step) {
      bool live = alive && step < w.max_steps && !at_end(w);
      const bool inw = live && in_window(w, p);
      if (live && !inw && left_for_good(w, p)) live = false;
      alive = live;
      if (!__any_sync(0xffffffffu, live)) break;
      uint32_t key = kNoKey | lane;
      bool incube = false;
      if (live && inw) {
        key = static_cast<uint32_t>(walk_hash(w, p));
        incube = static_cast<unsigned>(c[0]) < static_cast<unsigned>(S) &&
                 static_cast<unsigned>(c[1]) < static_cast<unsigned>(S) &&
                 static_cast<unsigned>(c[2]) < static_cast<unsigned>(S);
        ++incs;
      }
      if (kMatch) {
        const uint32_t peers = __match_any_sync(0xffffffffu, key);
        if (!(key & kNoKey) && lane == __ffs(peers) - 1) {
          const uint32_t n = __popc(peers);
          if (incube) {
            atomicAdd(&cube[(c[0] * S + c[1]) * S + c[2]], n);
          } else {
            atomicAdd(p.cnt + key, n);
            mark_line(p, static_cast<int>(key), last);
          }
        }
      } else if (!(key & kNoKey)) {
        if (incube) {
          atomicAdd(&cube[(c[0] * S + c[1]) * S + c[2]], 1u);
        } else {
          atomicAdd(p.cnt + key, 1u);
          mark_line(p, static_cast<int>(key), last);
        }
      }
      if (live) {
        const int a = ray_step(w, p);
        if (a == 0)
          c[0] += w.st[0];
        else if (a == 1)
          c[1] += w.st[1];
        else
          c[2] += w.st[2];
      }
    }
    // Endpoints (kernels.cu:139-151): op for an in-window endpoint, and a
    // hit unless the ray was clipped.
    uint32_t ekey = kNoKey | lane;
    bool e_incube = false;
    int e_idx = 0;
    if (valid) {
      const int h = end_hash(w, p);
      if (h >= 0) {
        ekey = static_cast<uint32_t>(h);
        int ec[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) ec[a] = w.en[a] - clo[a];
        e_incube = static_cast<unsigned>(ec[0]) < static_cast<unsigned>(S) &&
                   static_cast<unsigned>(ec[1]) < static_cast<unsigned>(S) &&
                   static_cast<unsigned>(ec[2]) < static_cast<unsigned>(S);
        e_idx = (ec[0] * S + ec[1]) * S + ec[2];
        ++incs;
      }
    }
    const bool e_hit = !(ekey & kNoKey) && !w.clipped;
    if (e_hit) ++hits;
    {
      const uint32_t peers = __match_any_sync(0xffffffffu, ekey);
      if (!(ekey & kNoKey) && lane == __ffs(peers) - 1) {
        const uint32_t n = __popc(peers);
        if (e_incube) {
          atomicAdd(&cube[e_idx], n);
        } else {
          atomicAdd(p.cnt + ekey, n);
          mark_line(p, static_cast<int>(ekey), last);
        }
      }
      const uint32_t hkey = e_hit ? ekey : (kNoKey | lane);
      const uint32_t hp = __match_any_sync(0xffffffffu, hkey);
      if (e_hit && lane == __ffs(hp) - 1) {
        atomicOr(p.cnt + hkey, kHitFlag);
        atomicAdd(p.hit + hkey, static_cast<uint32_t>(__popc(hp)));
      }
    }
  }
  __syncthreads();
  // Flush the cube: every staged voxel was in the window when counted.
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
}

int sms() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

template <int S, bool kMatch>
void launch_walk(const RayParams &p, const int clo[3], cudaStream_t s) {
  const size_t smem = sizeof(uint32_t) * S * S * S;
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(walk_kernel<S, kMatch>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(smem));
    configured = true;
  }
  int ctas = sms();
  int per = (p.n + ctas - 1) / ctas;
  per = ((per + 31) / 32) * 32;
  if (per < 32) per = 32;
  const int grid = (p.n + per - 1) / per;
  walk_kernel<S, kMatch><<<grid, 512, smem, s>>>(p, clo[0], clo[1], clo[2], per);
}

}  // namespace

void launch_raycast_binned(const RayParams &p_in, const BinnedScratch &b, int cube,
                           bool match, bool sort, cudaStream_t s) {
  if (p_in.n <= 0) return;
  RayParams p = p_in;
  if (sort) {
    cudaMemsetAsync(b.hist, 0, sizeof(int) * kBins, s);
    const int grid = min((p.n + 255) / 256, sms() * 4);
    bin_kernel<<<grid, 256, 0, s>>>(p, b.bins, b.hist);
    bin_scan_kernel<<<1, 1024, 0, s>>>(b.hist, b.cursor);
    scatter_kernel<<<grid, 256, 0, s>>>(p, b.bins, b.cursor, b.sorted);
    p.x = b.sorted;
    p.y = b.sorted + p.n;
    p.z = b.sorted + 2 * static_cast<size_t>(p.n);
    p.stride = 1;
  } else if (p.stride != 1) {
    // The walk reads x[i], y[i], z[i]; an AoS cloud is read with stride 3
    // by the bin/scatter path only, so force the sort for it.
    return launch_raycast_binned(p_in, b, cube, match, true, s);
  }
  // Cube around the sensor voxel (device binning of the sensor origin).
  int clo[3];
  const int half_cube = cube / 2;
  for (int a = 0; a < 3; ++a)
    clo[a] = pos_to_global_dev(p.o[a], p.inv, p.ctr != 0, p.fp) - half_cube;
  if (cube >= 32) {
    if (match)
      launch_walk<32, true>(p, clo, s);
    else
      launch_walk<32, false>(p, clo, s);
  } else if (cube >= 16) {
    if (match)
      launch_walk<16, true>(p, clo, s);
    else
      launch_walk<16, false>(p, clo, s);
  } else {
    if (match)
      launch_walk<4, true>(p, clo, s);  // a token cube: almost all global
    else
      launch_walk<4, false>(p, clo, s);
  }
}

int binned_bins() { return kBins; }

void launch_direction_sort(const RayParams &p, const BinnedScratch &b, cudaStream_t s) {
  if (p.n <= 0) return;
  cudaMemsetAsync(b.hist, 0, sizeof(int) * kBins, s);
  const int grid = min((p.n + 255) / 256, sms() * 4);
  bin_kernel<<<grid, 256, 0, s>>>(p, b.bins, b.hist);
  bin_scan_kernel<<<1, 1024, 0, s>>>(b.hist, b.cursor);
  scatter_kernel<<<grid, 256, 0, s>>>(p, b.bins, b.cursor, b.sorted);
}

}  // namespace cublox_b200

// Warp-cooperative exact raycast: long rays are split between lanes.
//
// The reference walks each ray sequentially in one thread (kernels.cu:106-
// 137), so a scan's latency is set by its longest ray (~900 dependent steps
// at README scale).  Here a warp takes 32 rays, estimates each one's
// in-window length, and cuts it into K time segments; every lane then walks
// one segment.  Bit-exactness:
//
//  * The walk is a merge of three per-axis event sequences T_a(j) (the
//    rounded running sums tM += tD), ordered by (T, axis rank z<y<x) — the
//    reference's tie rule.  A segment [tau_k, tau_k+1) owns the states
//    produced by the events with T in that range; its start state is the
//    one after all events with T < tau_k, which first_at_or_above()
//    (dda_jump.cuh) computes exactly per axis.
//  * The reference stops at the first state equal to the end voxel, which
//    can only be state |dx|+|dy|+|dz| (= L1); whether it is reached follows
//    from comparing the last needed event of every axis with the first
//    extra one.  States past L1 are skipped when it is.
//  * Degenerate rays (an axis with infinite or stalling times, huge index
//    spans) are never split.
//
// Increments inside the S^3 cube around the sensor are staged in shared
// memory and flushed once per CTA, as in raycast_binned.cu.
#include <cuda_runtime.h>

#include <cstdint>

#include "dda_jump.cuh"
#include "kernels.cuh"
#include "ray_walk.cuh"

namespace cublox_b200 {

namespace {

constexpr int kMaxSegs = 32;

struct Cuts {
  float t_lo, t_hi;  // window interval along the ray (parametric metres)
  int K;
};

// Window entry/exit of the ray (o + t*u, t in [0, L]) — only used to place
// the segment cuts, so a padded float slab test is enough.
__device__ __forceinline__ Cuts plan_cuts(const RayParams &p, const RayWalk &w,
                                          float ex, float ey, float ez, int seg_len) {
  Cuts c{0.0f, 0.0f, 1};
  const float o[3] = {p.o[0], p.o[1], p.o[2]};
  float e[3] = {ex, ey, ez};
  float d[3] = {e[0] - o[0], e[1] - o[1], e[2] - o[2]};
  const float L = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  if (!(L > 0.0f) || !isfinite(L)) return c;
  const float Lc = fminf(L, p.max_range);
  float t0 = 0.0f, t1 = Lc;
  float rate = 0.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float ua = d[a] / L;
    const float off = p.ctr ? -0.5f : 0.0f;
    const float lo = (static_cast<float>(p.win[a] - p.half[a] - 1) + off) * p.res;
    const float hi = (static_cast<float>(p.win[a] + p.half[a] + 2) + off) * p.res;
    if (fabsf(ua) < 1e-12f) {
      if (o[a] < lo || o[a] > hi) return c;
      continue;
    }
    float ta = (lo - o[a]) / ua, tb = (hi - o[a]) / ua;
    if (ta > tb) {
      const float t = ta;
      ta = tb;
      tb = t;
    }
    t0 = fmaxf(t0, ta);
    t1 = fminf(t1, tb);
    rate += fabsf(ua);
  }
  if (!(t1 > t0)) return c;
  const float steps = (t1 - t0) * rate / p.res;
  int K = static_cast<int>(steps / static_cast<float>(seg_len));
  K = K < 1 ? 1 : (K > kMaxSegs ? kMaxSegs : K);
  // Splitting needs finite per-axis times and moderate spans.
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (w.st[a] != 0 && (!isfinite(w.tM[a]) || !isfinite(w.tD[a]))) K = 1;
    if (abs(w.en[a] - w.id[a]) > (1 << 20)) K = 1;
  }
  c.t_lo = t0;
  c.t_hi = t1;
  c.K = K;
  return c;
}

__device__ __forceinline__ float cut_time(const Cuts &c, int k) {
  if (k <= 0) return -inf_f();
  if (k >= c.K) return inf_f();
  return c.t_lo + (c.t_hi - c.t_lo) * (static_cast<float>(k) / static_cast<float>(c.K));
}

// (T, rank) order of the reference's step choice: z before y before x.
__device__ __forceinline__ bool ev_less(float t1, int r1, float t2, int r2) {
  return t1 < t2 || (t1 == t2 && r1 < r2);
}

// Does the walk's state number L1 (= |dx|+|dy|+|dz|) equal the end voxel?
__device__ bool reaches_end(const RayWalk &w0) {
  float need_t = -inf_f(), extra_t = inf_f();
  int need_r = -1, extra_r = 3;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int D = w0.en[a] - w0.id[a];
    const int rank = 2 - a;
    if (D != 0 && (w0.st[a] == 0 || (D > 0) != (w0.st[a] > 0))) return false;
    const int n = abs(D);
    if (w0.st[a] == 0) continue;  // never steps: extra events at +inf
    if (n > 0) {
      const JumpResult v = value_at(w0.tM[a], w0.tD[a], n - 1);
      if (!v.ok) return false;
      if (ev_less(need_t, need_r, v.s, rank)) {
        need_t = v.s;
        need_r = rank;
      }
    }
    const JumpResult x = value_at(w0.tM[a], w0.tD[a], n);
    if (!x.ok) return false;
    if (ev_less(x.s, rank, extra_t, extra_r)) {
      extra_t = x.s;
      extra_r = rank;
    }
  }
  return ev_less(need_t, need_r, extra_t, extra_r);
}

__device__ __forceinline__ int pick_axis(const RayWalk &w) {
  if (w.tM[0] < w.tM[1]) return w.tM[0] < w.tM[2] ? 0 : 2;
  return w.tM[1] < w.tM[2] ? 1 : 2;
}

__device__ __forceinline__ float axis_time(const RayWalk &w, int a) {
  return a == 0 ? w.tM[0] : (a == 1 ? w.tM[1] : w.tM[2]);
}

template <int S>
struct Emitter {
  const RayParams &p;
  uint32_t *cube;
  int clo0, clo1, clo2;
  uint32_t incs;

  __device__ __forceinline__ void voxel(const RayWalk &w) {
    const int c0 = w.id[0] - clo0, c1 = w.id[1] - clo1, c2 = w.id[2] - clo2;
    if (S > 0 && static_cast<unsigned>(c0) < static_cast<unsigned>(S) &&
        static_cast<unsigned>(c1) < static_cast<unsigned>(S) &&
        static_cast<unsigned>(c2) < static_cast<unsigned>(S)) {
      atomicAdd(&cube[(c0 * S + c1) * S + c2], 1u);
    } else {
      atomicAdd(p.cnt + walk_hash(w, p), 1u);
    }
    ++incs;
  }
};

// Walk segment k of K of one ray.  Returns false if the ray is dropped.
template <int S>
__device__ bool walk_segment(const RayParams &p, float ex, float ey, float ez, int k,
                             const Cuts &cuts, Emitter<S> &em, uint32_t &hits) {
  RayWalk w;
  if (!ray_begin(p, ex, ey, ez, w)) return false;
  const int L1 = abs(w.en[0] - w.id[0]) + abs(w.en[1] - w.id[1]) + abs(w.en[2] - w.id[2]);
  int64_t i = 0;  // index of the current state
  int ended = -1; // unknown
  RayWalk w0;
  if (k > 0) {
    w0 = w;
    const float tau = cut_time(cuts, k);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (w.st[a] == 0) continue;
      const JumpResult r = first_at_or_above(w0.tM[a], w0.tD[a], tau, w.max_steps);
      if (!r.ok) atomicOr(p.err, kErrJumpStall);  // excluded by plan_cuts
      const int c = static_cast<int>(r.j);
      i += c;
      w.tM[a] = r.s;
      w.id[a] = w0.id[a] + w0.st[a] * c;
      w.rel[a] = w.id[a] - p.win[a];
      w.slot[a] = global_to_local(w.id[a], p.map[a], p.half[a]) + p.half[a];
    }
  }
  const float tau_next = cut_time(cuts, k + 1);
  // process the current state (lane 0 owns the initial one)
  bool go = true;
  if (k == 0) {
    if (i >= w.max_steps || at_end(w)) {
      go = false;
    } else if (in_window(w, p)) {
      em.voxel(w);
    } else if (left_for_good(w, p)) {
      go = false;
    }
  }
  while (go) {
    const int a = pick_axis(w);
    if (axis_time(w, a) >= tau_next) break;
    if (a == 0) {
      w.id[0] += w.st[0];
      w.rel[0] += w.st[0];
      w.slot[0] = wrap_slot(w.slot[0] + w.st[0], p.map[0]);
      w.tM[0] = fadd(w.tM[0], w.tD[0]);
    } else if (a == 1) {
      w.id[1] += w.st[1];
      w.rel[1] += w.st[1];
      w.slot[1] = wrap_slot(w.slot[1] + w.st[1], p.map[1]);
      w.tM[1] = fadd(w.tM[1], w.tD[1]);
    } else {
      w.id[2] += w.st[2];
      w.rel[2] += w.st[2];
      w.slot[2] = wrap_slot(w.slot[2] + w.st[2], p.map[2]);
      w.tM[2] = fadd(w.tM[2], w.tD[2]);
    }
    ++i;
    if (i >= w.max_steps) break;
    if (i >= L1) {
      // Only state L1 can be the end voxel; past it, the walk went on only
      // if state L1 was not the end.
      if (i == L1) {
        if (at_end(w)) break;
      } else {
        if (ended < 0) ended = (k == 0) ? 0 : (reaches_end(w0) ? 1 : 0);
        if (ended) break;
      }
    }
    if (in_window(w, p)) {
      em.voxel(w);
    } else if (left_for_good(w, p)) {
      break;
    }
  }
  if (k == 0) {
    // Endpoint (kernels.cu:139-151).
    const int h = end_hash(w, p);
    if (h >= 0) {
      const int c0 = w.en[0] - em.clo0, c1 = w.en[1] - em.clo1, c2 = w.en[2] - em.clo2;
      if (S > 0 && static_cast<unsigned>(c0) < static_cast<unsigned>(S) &&
          static_cast<unsigned>(c1) < static_cast<unsigned>(S) &&
          static_cast<unsigned>(c2) < static_cast<unsigned>(S))
        atomicAdd(&em.cube[(c0 * S + c1) * S + c2], 1u);
      else
        atomicAdd(p.cnt + h, 1u);
      ++em.incs;
      if (!w.clipped) {
        atomicOr(p.cnt + h, kHitFlag);
        atomicAdd(p.hit + h, 1u);
        ++hits;
      }
    }
  }
  return true;
}

template <int S>
__global__ void __launch_bounds__(512, 1) split_walk_kernel(const RayParams p, const int cl0,
                                                            const int cl1, const int cl2,
                                                            const int seg_len,
                                                            int *work_counter) {
  extern __shared__ uint32_t cube[];
  constexpr int kCube = S * S * S;
  for (int i = threadIdx.x; i < kCube / 4; i += blockDim.x)
    reinterpret_cast<uint4 *>(cube)[i] = make_uint4(0u, 0u, 0u, 0u);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  Emitter<S> em{p, cube, cl0, cl1, cl2, 0u};
  uint32_t rays = 0, hits = 0;
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(work_counter, 32);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= p.n) break;
    const int i = base + lane;
    float ex = 0.0f, ey = 0.0f, ez = 0.0f;
    int K = 0;
    Cuts cuts{0.0f, 0.0f, 1};
    if (i < p.n) {
      ex = p.x[i];
      ey = p.y[i];
      ez = p.z[i];
      RayWalk w;
      if (ray_begin(p, ex, ey, ez, w)) {
        cuts = plan_cuts(p, w, ex, ey, ez, seg_len);
        K = cuts.K;
        ++rays;
      }
    }
    // Inclusive warp scan of the segment counts.
    int incl = K;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= off) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    for (int g0 = 0; g0 < total; g0 += 32) {
      const int g = g0 + lane;
      // Smallest ray r of the chunk with incl[r] > g.
      int r = 0;
#pragma unroll
      for (int step = 16; step >= 1; step >>= 1) {
        const int v = __shfl_sync(0xffffffffu, incl, r + step - 1);
        if (v <= g) r += step;
      }
      const int kr = __shfl_sync(0xffffffffu, K, r);
      const float rx = __shfl_sync(0xffffffffu, ex, r);
      const float ry = __shfl_sync(0xffffffffu, ey, r);
      const float rz = __shfl_sync(0xffffffffu, ez, r);
      const float tlo = __shfl_sync(0xffffffffu, cuts.t_lo, r);
      const float thi = __shfl_sync(0xffffffffu, cuts.t_hi, r);
      const int excl = __shfl_sync(0xffffffffu, incl, r) - kr;
      if (g < total) {
        const Cuts rc{tlo, thi, kr};
        walk_segment<S>(p, rx, ry, rz, g - excl, rc, em, hits);
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kCube; i += blockDim.x) {
    const uint32_t v = cube[i];
    if (!v) continue;
    const int g[3] = {cl0 + i / (S * S), cl1 + (i / S) % S, cl2 + i % S};
    const int h = ((global_to_local(g[0], p.map[0], p.half[0]) + p.half[0]) * p.map[1] +
                   (global_to_local(g[1], p.map[1], p.half[1]) + p.half[1])) *
                      p.map[2] +
                  (global_to_local(g[2], p.map[2], p.half[2]) + p.half[2]);
    atomicAdd(p.cnt + h, v);
  }
  if (p.stats) {
    uint32_t incs = em.incs;
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

int sm_count_split() {
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
void launch_split(const RayParams &p, const int clo[3], int seg_len, int *counter,
                  cudaStream_t s) {
  const size_t smem = sizeof(uint32_t) * S * S * S;
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(split_walk_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(smem));
  static int per_sm = 0;
  if (per_sm == 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, split_walk_kernel<S>, 512, smem);
    if (per_sm < 1) per_sm = 1;
  }
  const int grid = sm_count_split() * per_sm;
  split_walk_kernel<S><<<grid, 512, smem, s>>>(p, clo[0], clo[1], clo[2], seg_len, counter);
}

}  // namespace

void launch_raycast_split(const RayParams &p, int cube, int seg_len, int *counter,
                          cudaStream_t s) {
  if (p.n <= 0) return;
  cudaMemsetAsync(counter, 0, sizeof(int), s);
  int clo[3];
  const int hc = cube / 2;
  for (int a = 0; a < 3; ++a)
    clo[a] = pos_to_global_dev(p.o[a], p.inv, p.ctr != 0, p.fp) - hc;
  if (cube >= 32)
    launch_split<32>(p, clo, seg_len, counter, s);
  else if (cube >= 16)
    launch_split<16>(p, clo, seg_len, counter, s);
  else
    launch_split<0>(p, clo, seg_len, counter, s);
}

}  // namespace cublox_b200

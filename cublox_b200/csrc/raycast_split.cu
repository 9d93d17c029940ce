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

// T_a(j) continuing from a known (j0, s0) of the same sequence when j >= j0,
// else from the start (t0).
__device__ __forceinline__ JumpResult value_from(float t0, float d, int64_t j0, float s0,
                                                 int64_t j) {
  if (j >= j0) {
    JumpResult r = value_at(s0, d, j - j0);
    r.j += j0;
    return r;
  }
  return value_at(t0, d, j);
}

// Does the walk's state number L1 (= |dx|+|dy|+|dz|) equal the end voxel?
// It does iff every event needed to reach the end voxel (the first |D_a|
// of each axis) precedes, in (T, rank) order, every further event.  (j0,
// s0) are known positions of each axis's sequence to continue from.
__device__ bool reaches_end(const RayWalk &w0, const int64_t j0[3], const float s0[3]) {
  float need_t = -inf_f(), extra_t = inf_f();
  int need_r = -1, extra_r = 3;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int D = w0.en[a] - w0.id[a];
    const int rank = 2 - a;
    if (D != 0 && (w0.st[a] == 0 || (D > 0) != (w0.st[a] > 0))) return false;
    const int n = abs(D);
    if (w0.st[a] == 0) continue;  // never steps: extra events at +inf
    float tn;
    if (n > 0) {
      const JumpResult v = value_from(w0.tM[a], w0.tD[a], j0[a], s0[a], n - 1);
      if (!v.ok) return false;
      if (ev_less(need_t, need_r, v.s, rank)) {
        need_t = v.s;
        need_r = rank;
      }
      tn = fadd(v.s, w0.tD[a]);
    } else {
      tn = w0.tM[a];
    }
    if (ev_less(tn, rank, extra_t, extra_r)) {
      extra_t = tn;
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

// ---- planned split ------------------------------------------------------
// Per ray (plan kernel, one thread per ray): the exact setup, the cuts, and
// every segment's start state, computed by continuing each axis's jump from
// the previous cut (so each axis's binades are walked once per ray).  Per
// segment (walk kernel, one lane per segment from a global queue): load the
// start state and walk until the next cut.

struct SegRec {     // 48 bytes
  int ray;
  int i;            // index of the start state
  int id[3];        // start voxel
  float tM[3];      // per-axis next event times
  float tau_next;   // the segment owns events with T < tau_next
  int k;            // segment number within the ray
  int pad[2];
};

struct RayRec {     // 48 bytes
  int en[3];
  int st[3];
  float tD[3];
  int max_steps;
  int L1;
  int flags;        // bit0 clipped, bit1 state L1 is the end voxel
};

__global__ void __launch_bounds__(256) seg_plan_kernel(const RayParams p, int seg_len,
                                                       int max_segs, SegRec *segs,
                                                       RayRec *rays, int *seg_count,
                                                       int seg_cap) {
  __shared__ int warp_tot[8];
  __shared__ int block_base;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  RayWalk w;
  bool valid = false;
  Cuts cuts{0.0f, 0.0f, 0};
  float ex = 0.0f, ey = 0.0f, ez = 0.0f;
  if (i < p.n) {
    const size_t k = static_cast<size_t>(i) * p.stride;
    ex = p.x[k];
    ey = p.y[k];
    ez = p.z[k];
    valid = ray_begin(p, ex, ey, ez, w);
    if (valid) {
      cuts = plan_cuts(p, w, ex, ey, ez, seg_len);
      if (cuts.K > max_segs) cuts.K = max_segs;
    }
  }
  int K = valid ? cuts.K : 0;
  // block-wide exclusive scan of K, one global reservation per block
  int incl = K;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += v;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int q = 0; q < static_cast<int>(blockDim.x >> 5); ++q) {
      const int t = warp_tot[q];
      warp_tot[q] = run;
      run += t;
    }
    block_base = atomicAdd(seg_count, run);
  }
  __syncthreads();
  int base = block_base + warp_tot[warp] + incl - K;
  if (!valid) return;
  if (base + K > seg_cap) {  // never expected: capacity is n * max_segs
    atomicOr(p.err, kErrFetchOverflow);
    return;
  }
  RayRec rr;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    rr.en[a] = w.en[a];
    rr.st[a] = w.st[a];
    rr.tD[a] = w.tD[a];
  }
  rr.max_steps = w.max_steps;
  rr.L1 = abs(w.en[0] - w.id[0]) + abs(w.en[1] - w.id[1]) + abs(w.en[2] - w.id[2]);
  // segment start states, cut by cut
  int64_t jc[3] = {0, 0, 0};
  float sc[3] = {w.tM[0], w.tM[1], w.tM[2]};
  for (int k = 0; k < K; ++k) {
    SegRec sr;
    sr.ray = i;
    sr.k = k;
    sr.tau_next = cut_time(cuts, k + 1);
    int64_t idx = 0;
    if (k > 0) {
      const float tau = cut_time(cuts, k);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        if (w.st[a] == 0) continue;
        const JumpResult r =
            first_at_or_above(sc[a], w.tD[a], tau, static_cast<int64_t>(w.max_steps) - jc[a]);
        if (!r.ok) atomicOr(p.err, kErrJumpStall);  // excluded by plan_cuts
        jc[a] += r.j;
        sc[a] = r.s;
      }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      idx += jc[a];
      sr.id[a] = w.id[a] + w.st[a] * static_cast<int>(jc[a]);
      sr.tM[a] = sc[a];
    }
    sr.i = idx > w.max_steps ? w.max_steps : static_cast<int>(idx);
    sr.pad[0] = sr.pad[1] = 0;
    segs[base + k] = sr;
  }
  rr.flags = (w.clipped ? 1 : 0) | ((K > 1 && reaches_end(w, jc, sc)) ? 2 : 0);
  rays[i] = rr;
}

template <int S>
__global__ void __launch_bounds__(1024) seg_walk_kernel(const RayParams p, const int cl0,
                                                       const int cl1, const int cl2,
                                                       const SegRec *segs, const RayRec *rays,
                                                       const int *seg_count, int *work,
                                                       const int contiguous) {
  extern __shared__ uint32_t cube[];
  constexpr int kCube = S * S * S;
  __shared__ int cta_next;
  for (int q = threadIdx.x; q < kCube / 4; q += blockDim.x)
    reinterpret_cast<uint4 *>(cube)[q] = make_uint4(0u, 0u, 0u, 0u);
  if (threadIdx.x == 0) cta_next = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int total = *seg_count;
  // contiguous: CTA c owns segments [lo, hi); warps share them via cta_next.
  const int per = (total + gridDim.x - 1) / gridDim.x;
  const int lo = contiguous ? min(total, blockIdx.x * per) : 0;
  const int hi = contiguous ? min(total, lo + per) : total;
  Emitter<S> em{p, cube, cl0, cl1, cl2, 0u};
  uint32_t nrays = 0, hits = 0;
  for (;;) {
    int b = 0;
    if (lane == 0) b = contiguous ? lo + atomicAdd(&cta_next, 32) : atomicAdd(work, 32);
    b = __shfl_sync(0xffffffffu, b, 0);
    if (b >= hi) break;
    const int g = b + lane;
    if (g >= hi) continue;
    const SegRec sr = segs[g];
    const RayRec rr = rays[sr.ray];
    RayWalk w;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      w.id[a] = sr.id[a];
      w.en[a] = rr.en[a];
      w.st[a] = rr.st[a];
      w.tD[a] = rr.tD[a];
      w.tM[a] = sr.tM[a];
      w.rel[a] = w.id[a] - p.win[a];
      w.slot[a] = global_to_local(w.id[a], p.map[a], p.half[a]) + p.half[a];
    }
    w.max_steps = rr.max_steps;
    w.clipped = rr.flags & 1;
    const bool ends_at_l1 = (rr.flags & 2) != 0;
    int i = sr.i;
    bool go = i < w.max_steps;
    if (sr.k == 0) {
      ++nrays;
      if (!go || at_end(w)) {
        go = false;
      } else if (in_window(w, p)) {
        em.voxel(w);
      } else if (left_for_good(w, p)) {
        go = false;
      }
    }
    while (go) {
      const int a = pick_axis(w);
      if (axis_time(w, a) >= sr.tau_next) break;
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
      // Only state L1 can be the end voxel; past it the walk continues only
      // if state L1 was not the end (a segment that started past L1 learns
      // that from the plan).
      if (i == rr.L1) {
        if (at_end(w)) break;
      } else if (i > rr.L1 && sr.i >= rr.L1 && ends_at_l1) {
        break;
      }
      if (in_window(w, p)) {
        em.voxel(w);
      } else if (left_for_good(w, p)) {
        break;
      }
    }
    if (sr.k == 0) {
      // Endpoint (kernels.cu:139-151).
      const int h = end_hash(w, p);
      if (h >= 0) {
        const int c0 = w.en[0] - cl0, c1 = w.en[1] - cl1, c2 = w.en[2] - cl2;
        if (S > 0 && static_cast<unsigned>(c0) < static_cast<unsigned>(S) &&
            static_cast<unsigned>(c1) < static_cast<unsigned>(S) &&
            static_cast<unsigned>(c2) < static_cast<unsigned>(S))
          atomicAdd(&cube[(c0 * S + c1) * S + c2], 1u);
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
  }
  __syncthreads();
  if constexpr (S > 0)
  for (int q = threadIdx.x; q < kCube; q += blockDim.x) {
    const uint32_t v = cube[q];
    if (!v) continue;
    const int gg[3] = {cl0 + q / (S * S), cl1 + (q / S) % S, cl2 + q % S};
    const int h = ((global_to_local(gg[0], p.map[0], p.half[0]) + p.half[0]) * p.map[1] +
                   (global_to_local(gg[1], p.map[1], p.half[1]) + p.half[1])) *
                      p.map[2] +
                  (global_to_local(gg[2], p.map[2], p.half[2]) + p.half[2]);
    atomicAdd(p.cnt + h, v);
  }
  if (p.stats) {
    uint32_t incs = em.incs;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      nrays += __shfl_down_sync(0xffffffffu, nrays, off);
      incs += __shfl_down_sync(0xffffffffu, incs, off);
      hits += __shfl_down_sync(0xffffffffu, hits, off);
    }
    if (lane == 0) {
      atomicAdd(p.stats + 0, static_cast<unsigned long long>(nrays));
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
void launch_seg_walk(const RayParams &p, const int clo[3], const SplitScratch &sc,
                     cudaStream_t s) {
  const size_t smem = sizeof(uint32_t) * S * S * S;
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(seg_walk_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(smem));
  const int block = sc.block == 256 || sc.block == 1024 ? sc.block : 512;
  static int per_sm[3] = {0, 0, 0};
  int &ps = per_sm[block == 256 ? 0 : (block == 512 ? 1 : 2)];
  if (ps == 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ps, seg_walk_kernel<S>, block, smem);
    if (ps < 1) ps = 1;
  }
  const int grid = sm_count_split() * ps;
  seg_walk_kernel<S><<<grid, block, smem, s>>>(
      p, clo[0], clo[1], clo[2], reinterpret_cast<const SegRec *>(sc.segs),
      reinterpret_cast<const RayRec *>(sc.rays), sc.counters, sc.counters + 1, sc.contiguous);
}

}  // namespace

size_t split_seg_bytes() { return sizeof(SegRec); }
size_t split_ray_bytes() { return sizeof(RayRec); }

void launch_raycast_split(const RayParams &p, int cube, int seg_len, const SplitScratch &sc,
                          cudaStream_t s) {
  if (p.n <= 0) return;
  cudaMemsetAsync(sc.counters, 0, 2 * sizeof(int), s);
  seg_plan_kernel<<<(p.n + 255) / 256, 256, 0, s>>>(
      p, seg_len, sc.max_segs, reinterpret_cast<SegRec *>(sc.segs),
      reinterpret_cast<RayRec *>(sc.rays), sc.counters, sc.seg_cap);
  int clo[3];
  const int hc = cube / 2;
  for (int a = 0; a < 3; ++a)
    clo[a] = pos_to_global_dev(p.o[a], p.inv, p.ctr != 0, p.fp) - hc;
  if (cube >= 32)
    launch_seg_walk<32>(p, clo, sc, s);
  else if (cube >= 16)
    launch_seg_walk<16>(p, clo, sc, s);
  else if (cube >= 8)
    launch_seg_walk<8>(p, clo, sc, s);
  else
    launch_seg_walk<0>(p, clo, sc, s);
}

}  // namespace cublox_b200

// Segmented exact raycast: long rays are split between lanes.
//
// The reference walks each ray sequentially in one thread (kernels.cu:106-
// 137), so a scan's latency is set by its longest ray (~900 dependent steps
// at README scale).  Here each ray's in-window length is estimated and the
// ray is cut into K time segments of about the same number of steps; every
// lane then walks one segment.  Bit-exactness:
//
//  * The walk is a merge of three per-axis event sequences T_a(j) (the
//    rounded running sums tM += tD), ordered by (T, axis rank z<y<x) — the
//    reference's tie rule.  Segment k starts at the state after all events
//    with T < tau_k, which first_at_or_above() (dda_jump.cuh) computes
//    exactly per axis, and walks up to the next segment's start state.
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
#include "far_walk.cuh"
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
// of each axis) precedes, in (T, rank) order, every further event.  Each
// axis contributes its last needed event and its first extra one
// (end_events), computed from a known position (j0, s0) of its sequence
// when that is not past the event, else from the start (tM0); end_combine
// orders the contributions.
struct EndEvents {
  float need_t, extra_t;
  bool ok;        // false: this axis alone rules the end voxel out
  bool has_need;  // the axis must step to reach the end voxel
  bool has_extra; // the axis steps at all
};

__device__ __forceinline__ EndEvents end_events(int D, int st, float tM0, float tD, int64_t j0,
                                                float s0) {
  EndEvents r{-inf_f(), inf_f(), true, false, false};
  if (D != 0 && (st == 0 || (D > 0) != (st > 0))) {
    r.ok = false;
    return r;
  }
  if (st == 0) return r;  // never steps: extra events at +inf
  r.has_extra = true;
  const int n = abs(D);
  if (n > 0) {
    const JumpResult v = value_from(tM0, tD, j0, s0, n - 1);
    if (!v.ok) {
      r.ok = false;
      return r;
    }
    r.has_need = true;
    r.need_t = v.s;
    r.extra_t = fadd(v.s, tD);
  } else {
    r.extra_t = tM0;
  }
  return r;
}

__device__ __forceinline__ bool end_combine(const EndEvents ev[3]) {
  float need_t = -inf_f(), extra_t = inf_f();
  int need_r = -1, extra_r = 3;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int rank = 2 - a;
    if (!ev[a].ok) return false;
    if (ev[a].has_need && ev_less(need_t, need_r, ev[a].need_t, rank)) {
      need_t = ev[a].need_t;
      need_r = rank;
    }
    if (ev[a].has_extra && ev_less(ev[a].extra_t, rank, extra_t, extra_r)) {
      extra_t = ev[a].extra_t;
      extra_r = rank;
    }
  }
  return ev_less(need_t, need_r, extra_t, extra_r);
}

// ---- planned split ------------------------------------------------------
// A ray's loop states 0, 1, 2, ... are cut at K times tau_1 < ... <
// tau_{K-1}: segment k owns the states i_k .. i_{k+1} - 1, where i_k counts
// the events with T < tau_k (i_0 = 0; the last segment runs to the ray's
// end).  Two launches:
//   seg_plan_kernel  32 rays per CTA, one warp per axis: the exact set-up
//                    and the cuts (every warp computes them), then warp a
//                    follows axis a's event sequence from cut to cut with
//                    the exact jump of dda_jump.cuh (advance_to: a cut in
//                    the binade run the previous one ended in costs one
//                    division), so each axis's binades are walked once per
//                    ray, and writes that axis's part of every segment
//                    record;
//   seg_walk_kernel  one lane per segment from a queue: walk i_{k+1} - i_k
//                    loop iterations from the start state, near phase then
//                    far phase (far_walk.cuh).
// Segment records: slot r holds ray r's first segment (the one that starts
// at the sensor and crosses the shared-memory cube); the later segments of
// all rays follow, so warps of the walk see segments of one kind.

struct SegAxis {    // 16 bytes: one axis of a segment's start, written in one store
  int j;            // events before the segment (start state index = sum over axes)
  int nj;           // events in the segment (-1: last segment)
  int id;           // start voxel coordinate
  float tM;         // next event time
};

struct __align__(16) SegRec {  // 64 bytes
  int ray;          // -1: the ray was dropped (first-segment slots only)
  int k;            // segment number within the ray
  int pad[2];
  SegAxis ax[3];
};

struct RayRec {     // 48 bytes
  int en[3];
  int st[3];
  float tD[3];
  int max_steps;
  int L1;
  int flags;        // bit0 clipped, bit1 state L1 is the end voxel
};

constexpr int kFlagClipped = 1, kFlagEndsAtL1 = 2;
constexpr int kPlanRays = 32;

template <typename T>
__device__ __forceinline__ T pick3(const T (&v)[3], int a) {
  return a == 0 ? v[0] : (a == 1 ? v[1] : v[2]);
}

__global__ void __launch_bounds__(3 * kPlanRays) seg_plan_kernel(const RayParams p, int seg_len,
                                                                 int max_segs, SegRec *segs,
                                                                 RayRec *rays, int *seg_count,
                                                                 int seg_cap) {
  __shared__ int s_base;
  __shared__ EndEvents s_end[3][kPlanRays];
  const int a = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * kPlanRays + lane;
  RayWalk w;
  bool valid = false;
  Cuts cuts{0.0f, 0.0f, 0};
  if (i < p.n) {
    const size_t k = static_cast<size_t>(i) * p.stride;
    const float ex = p.x[k], ey = p.y[k], ez = p.z[k];
    valid = ray_begin(p, ex, ey, ez, w);
    if (valid) {
      cuts = plan_cuts(p, w, ex, ey, ez, seg_len);
      if (cuts.K > max_segs) cuts.K = max_segs;
    }
  }
  // Later segments (k >= 1) of the CTA's rays: one reservation per CTA.
  const int more = valid ? cuts.K - 1 : 0;
  int incl = more;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += v;
  }
  if (threadIdx.x == 31) s_base = atomicAdd(seg_count, incl);
  __syncthreads();
  const int base = p.n + s_base + incl - more;  // record of segment 1
  if (valid && base + more > seg_cap) {         // never expected: capacity is n * max_segs
    atomicOr(p.err, kErrFetchOverflow);
    valid = false;
  }
  if (!valid && a == 0 && i < p.n) segs[i].ray = -1;
  long long jc = 0;
  float sc = 0.0f;
  if (valid) {
    const int st = pick3(w.st, a), id0 = pick3(w.id, a);
    const float tD = pick3(w.tD, a);
    sc = pick3(w.tM, a);
    JumpStretch run{};
    run.valid = false;
    const int K = cuts.K;
    for (int k = 0; k < K; ++k) {
      SegRec *r = segs + (k == 0 ? i : base + k - 1);
      long long jn = jc;
      float sn = sc;
      if (k + 1 < K && st != 0) {
        const JumpResult q = advance_to(jc, sc, tD, cut_time(cuts, k + 1), w.max_steps, run);
        if (!q.ok) atomicOr(p.err, kErrJumpStall);  // excluded by plan_cuts
        jn = q.j;
        sn = q.s;
      }
      if (a == 0) *reinterpret_cast<int2 *>(r) = make_int2(i, k);
      *reinterpret_cast<int4 *>(&r->ax[a]) =
          make_int4(static_cast<int>(jc), k + 1 < K ? static_cast<int>(jn - jc) : -1,
                    id0 + st * static_cast<int>(jc), __float_as_int(sc));
      if (k + 1 < K) {
        jc = jn;
        sc = sn;
      }
    }
  }
  // (jc, sc): axis a at the last cut; its share of the end test
  if (valid && cuts.K > 1)
    s_end[a][lane] = end_events(pick3(w.en, a) - pick3(w.id, a), pick3(w.st, a),
                                pick3(w.tM, a), pick3(w.tD, a), jc, sc);
  __syncthreads();
  if (!valid || a != 0) return;
  RayRec rr;
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    rr.en[b] = w.en[b];
    rr.st[b] = w.st[b];
    rr.tD[b] = w.tD[b];
  }
  rr.max_steps = w.max_steps;
  rr.L1 = abs(w.en[0] - w.id[0]) + abs(w.en[1] - w.id[1]) + abs(w.en[2] - w.id[2]);
  bool ends = false;
  if (cuts.K > 1) {
    const EndEvents ev[3] = {s_end[0][lane], s_end[1][lane], s_end[2][lane]};
    ends = end_combine(ev);
  }
  rr.flags = (w.clipped ? kFlagClipped : 0) | (ends ? kFlagEndsAtL1 : 0);
  rays[i] = rr;
}

// Near phase of a segment: the exact loop while the voxel is in the cube or
// outside the window, for at most `budget` iterations.  Returns true if the
// segment ended in it; false once the walk is in the window and outside the
// cube (f then holds it).
template <int S, int SZ = S>
__device__ __forceinline__ bool seg_near(const RayParams &p, uint32_t *cube, const int clo[3],
                                         RayWalk &w, int i, int &budget, FarWalk &f,
                                         uint32_t &incs) {
  for (;; ++i, --budget) {
    if (budget <= 0 || i >= w.max_steps || at_end(w)) return true;
    if (in_window(w, p)) {
      const int c = cube_cell<S, SZ>(w.id[0], w.id[1], w.id[2], clo);
      if (c < 0) {
        to_far(p, w, i, f);
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

template <int S, int SZ = S>
__global__ void __launch_bounds__(1024) seg_walk_kernel(const RayParams p, const int cl0,
                                                       const int cl1, const int cl2,
                                                       const SegRec *segs, const RayRec *rays,
                                                       const int *seg_count, int *work,
                                                       const int contiguous) {
  extern __shared__ uint32_t cube[];
  constexpr int kCube = S * S * SZ;
  __shared__ int cta_next;
  for (int q = threadIdx.x; q < kCube / 4; q += blockDim.x)
    reinterpret_cast<uint4 *>(cube)[q] = make_uint4(0u, 0u, 0u, 0u);
  if (threadIdx.x == 0) cta_next = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int total = p.n + *seg_count;  // first-segment slots, then later segments
  const int clo[3] = {cl0, cl1, cl2};
  // contiguous: CTA c owns segments [lo, hi); warps share them via cta_next.
  const int per = (total + gridDim.x - 1) / gridDim.x;
  const int lo = contiguous ? min(total, blockIdx.x * per) : 0;
  const int hi = contiguous ? min(total, lo + per) : total;
  uint32_t nrays = 0, hits = 0, incs = 0;
  for (;;) {
    int b = 0;
    if (lane == 0) b = contiguous ? lo + atomicAdd(&cta_next, 32) : atomicAdd(work, 32);
    b = __shfl_sync(0xffffffffu, b, 0);
    if (b >= hi) break;
    // Every lane runs the round, live or not, and the warp meets after the
    // near phase, so that its far phases run together rather than in groups
    // that entered the far loop at different times.
    const int g = b + lane;
    bool live = g < hi;
    SegRec sr;
    if (live) {
      sr = segs[g];
      live = sr.ray >= 0;
    }
    RayWalk w;
    FarWalk f;
    bool far = false;
    int budget = 0;
    if (live) {
      const RayRec rr = rays[sr.ray];
      const int j_sum = sr.ax[0].j + sr.ax[1].j + sr.ax[2].j;
      const int i0 = min(j_sum, rr.max_steps);
      budget = sr.ax[0].nj < 0
                   ? 0x7fffffff
                   : min(j_sum + sr.ax[0].nj + sr.ax[1].nj + sr.ax[2].nj, rr.max_steps) - i0;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        w.id[a] = sr.ax[a].id;
        w.en[a] = rr.en[a];
        w.st[a] = rr.st[a];
        w.tD[a] = rr.tD[a];
        w.tM[a] = sr.ax[a].tM;
        w.rel[a] = w.id[a] - p.win[a];
        w.slot[a] = global_to_local(w.id[a], p.map[a], p.half[a]) + p.half[a];
      }
      w.max_steps = rr.max_steps;
      w.clipped = (rr.flags & kFlagClipped) != 0;
      // A ray whose state L1 is the end voxel stops there: segments past it
      // have nothing to walk.
      if (!((rr.flags & kFlagEndsAtL1) && i0 > rr.L1))
        far = !seg_near<S, SZ>(p, cube, clo, w, i0, budget, f, incs);
    }
    __syncwarp();
    if (far) walk_far(p, f, budget, incs);
    if (live && sr.k == 0) {
      // Endpoint (kernels.cu:139-151).
      ++nrays;
      apply_end<S>(p, cube, ray_end_of<S, SZ>(p, w, clo), incs, hits);
    }
  }
  __syncthreads();
  flush_cube<S, SZ>(p, cube, clo);
  if (p.stats) {
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

template <int S, int SZ = S>
void launch_seg_walk(const RayParams &p, const int clo[3], const SplitScratch &sc,
                     cudaStream_t s) {
  const size_t smem = sizeof(uint32_t) * S * S * SZ;
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(seg_walk_kernel<S, SZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(smem));
  const int block = sc.block == 256 || sc.block == 1024 ? sc.block : 512;
  static int per_sm[3] = {0, 0, 0};
  int &ps = per_sm[block == 256 ? 0 : (block == 512 ? 1 : 2)];
  if (ps == 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ps, seg_walk_kernel<S, SZ>, block, smem);
    if (ps < 1) ps = 1;
  }
  const int grid = sm_count_split() * ps;
  seg_walk_kernel<S, SZ><<<grid, block, smem, s>>>(
      p, clo[0], clo[1], clo[2], reinterpret_cast<const SegRec *>(sc.segs),
      reinterpret_cast<const RayRec *>(sc.rays), sc.counters, sc.counters + 1, sc.contiguous);
}

}  // namespace

size_t split_seg_bytes() { return sizeof(SegRec); }
size_t split_ray_bytes() { return sizeof(RayRec); }

void launch_raycast_split(const RayParams &p, int cube, bool flat, int seg_len,
                          const SplitScratch &sc, cudaStream_t s) {
  if (p.n <= 0) return;
  cudaMemsetAsync(sc.counters, 0, 2 * sizeof(int), s);
  seg_plan_kernel<<<(p.n + kPlanRays - 1) / kPlanRays, 3 * kPlanRays, 0, s>>>(
      p, seg_len, sc.max_segs, reinterpret_cast<SegRec *>(sc.segs),
      reinterpret_cast<RayRec *>(sc.rays), sc.counters, sc.seg_cap);
  int clo[3];
  flat = flat && cube >= 32;
  for (int a = 0; a < 3; ++a)
    clo[a] = pos_to_global_dev(p.o[a], p.inv, p.ctr != 0, p.fp) -
             (a == 2 && flat ? cube / 4 : cube / 2);
  if (flat)
    launch_seg_walk<32, 16>(p, clo, sc, s);
  else if (cube >= 32)
    launch_seg_walk<32>(p, clo, sc, s);
  else if (cube >= 16)
    launch_seg_walk<16>(p, clo, sc, s);
  else if (cube >= 8)
    launch_seg_walk<8>(p, clo, sc, s);
  else
    launch_seg_walk<0>(p, clo, sc, s);
}

}  // namespace cublox_b200

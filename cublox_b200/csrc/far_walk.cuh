// Two-phase form of the exact ray walk (ray_walk.cuh), shared by the
// batched walk (batch.cu) and the split single-grid walk (raycast_split.cu).
#pragma once

#include <cstdint>

#include "exact_fp.cuh"
#include "kernels.cuh"
#include "ray_walk.cuh"

namespace cublox_b200 {

// Near phase: the exact walk of ray_walk.cuh (the reference's loop,
// kernels.cu:105-137) while the voxel is inside the S^3 shared-memory cube
// around the sensor, or outside the window.  Far phase, from the first
// in-window voxel outside the cube on: the same loop on per-axis step
// counters.  The cube and the window are boxes and a ray moves monotonically
// on every axis, so once it has left either it never comes back: the far
// phase needs no per-step box tests, only "steps left on this axis"
// counters, and keeps the voxel's address as a sum of per-axis terms
// (VoxLayout), each updated from its ring-buffer slot when the walk steps on
// that axis.  The voxels visited, and so the counts, are those of the single
// loop.

struct FarWalk {
  float tM[3], tD[3];  // as in RayWalk
  int e[3];     // steps to the endpoint's coordinate on the axis (all 0: at the endpoint)
  int out[3];   // steps the walk can still take on the axis inside the window
  int slot[3];  // ring-buffer slot of the current voxel on the axis
  int st[3];    // step on the axis (-1, 0, 1)
  int off[3];   // the axis's term of the current voxel's address
  int left;     // loop iterations left (max_steps - k)
  int h;        // address of the current voxel
  int line;     // line this thread flagged last (mark_line)
};

// The update after the loop (kernels.cu:138-151), fixed at the ray's start:
// endpoint hash (-1: endpoint outside the window), its cube cell (-1: not in
// the cube), and whether it counts a hit (not clipped at max range).
struct RayEnd {
  int h, c;
  bool hit;
};

constexpr int kNever = 0x7fffffff;  // counters of an axis the ray never steps on

// Cell of a global voxel in the S x S x SZ shared-memory cube with corner
// clo (z fastest), or -1 outside it.
template <int S, int SZ = S>
__device__ __forceinline__ int cube_cell(int g0, int g1, int g2, const int clo[3]) {
  const int c0 = g0 - clo[0], c1 = g1 - clo[1], c2 = g2 - clo[2];
  if (S > 0 && static_cast<unsigned>(c0) < static_cast<unsigned>(S) &&
      static_cast<unsigned>(c1) < static_cast<unsigned>(S) &&
      static_cast<unsigned>(c2) < static_cast<unsigned>(SZ))
    return (c0 * S + c1) * SZ + c2;
  return -1;
}

template <int S, int SZ = S>
__device__ __forceinline__ RayEnd ray_end_of(const RayParams &p, const RayWalk &w,
                                             const int clo[3]) {
  RayEnd r;
  r.h = end_hash(w, p);
  r.c = r.h >= 0 ? cube_cell<S, SZ>(w.en[0], w.en[1], w.en[2], clo) : -1;
  r.hit = !w.clipped;
  return r;
}

template <int S>
__device__ __forceinline__ void apply_end(const RayParams &p, uint32_t *cube, const RayEnd &r,
                                          uint32_t &incs, uint32_t &hits) {
  if (r.h < 0) return;
  if (S > 0 && r.c >= 0) {
    atomicAdd(&cube[r.c], 1u);
  } else {
    atomicAdd(p.cnt + r.h, 1u);
    int last = -1;
    mark_line(p, r.h, last);
  }
  ++incs;
  if (r.hit) {
    atomicOr(p.cnt + r.h, kHitFlag);
    atomicAdd(p.hit + r.h, 1u);
    ++hits;
  }
}

// Add an S^3 shared-memory cube of counts (corner clo, global voxel index)
// into the map's counters and flag their lines.  Only in-window voxels reach
// the cube, so every non-zero cell has an address in the map.
template <int S, int SZ = S>
__device__ __forceinline__ void flush_cube(const RayParams &p, const uint32_t *cube,
                                           const int clo[3]) {
  if constexpr (S > 0) {
    for (int q = threadIdx.x; q < S * S * SZ; q += blockDim.x) {
      const uint32_t v = cube[q];
      if (!v) continue;
      const int h =
          global_addr(p, clo[0] + q / (S * SZ), clo[1] + (q / SZ) % S, clo[2] + q % SZ);
      atomicAdd(p.cnt + h, v);
      if (p.dirty) p.dirty[h >> kLineShift] = 1;
    }
  }
}

// Far-phase state of a walk whose current voxel (loop iteration k, not yet
// counted) is inside the window.
__device__ __forceinline__ void to_far(const RayParams &p, const RayWalk &w, int k, FarWalk &f) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int d = w.en[a] - w.id[a];
    const int st = w.st[a];
    f.tM[a] = w.tM[a];
    f.tD[a] = w.tD[a];
    f.e[a] = st > 0 ? d : (st < 0 ? -d : d);
    f.out[a] = st > 0 ? p.half[a] - w.rel[a] : (st < 0 ? p.half[a] + w.rel[a] : kNever);
    f.slot[a] = w.slot[a];
    f.st[a] = st;
    f.off[a] = vox_axis(p.lay, a, w.slot[a]);
  }
  f.left = w.max_steps - k;
  f.h = f.off[0] + f.off[1] + f.off[2];
  f.line = -1;
}

// One step on axis A (the tie rule picked it): the slot moves with the ring
// buffer's wrap and the axis's address term follows it (a few integer
// operations, no memory access on the way to the next atomic's address).
// Returns true if the new voxel is outside the window, which ends the loop:
// the next iteration would break at its step limit, at the endpoint or as
// out of the window for good.
template <int A>
__device__ __forceinline__ bool far_step(FarWalk &f, const RayParams &p) {
  f.tM[A] = fadd(f.tM[A], f.tD[A]);
  --f.e[A];
  int s = f.slot[A] + f.st[A];
  s = s == p.map[A] ? 0 : (s < 0 ? p.map[A] - 1 : s);
  f.slot[A] = s;
  const int o = vox_axis(p.lay, A, s);
  f.h += o - f.off[A];
  f.off[A] = o;
  return f.out[A]-- == 0;
}

// Far phase for at most `budget` loop iterations; the ray's own step limit,
// window exit and endpoint end it earlier.  The endpoint test costs nothing
// per step: every step lowers one e counter by one, so the walk can stand on
// the endpoint only after exactly e0 + e1 + e2 steps (an axis it never steps
// on must already match), and not at all once a counter went negative.
// Until then only the limits and the window exit end the loop.  Every
// iteration counts the current voxel, then steps.  Returns true if the ray's
// loop is over (window left, endpoint reached or step limit spent), false
// if only the budget stopped it.
__device__ __forceinline__ bool walk_far(const RayParams &p, FarWalk &f, int budget,
                                         uint32_t &incs) {
  const int lim = min(budget, f.left);
  bool reachable = true;
  int to_end = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (f.st[a] == 0 ? f.e[a] != 0 : f.e[a] < 0) reachable = false;
    to_end += f.e[a];
  }
  int n = reachable ? min(lim, to_end) : lim;
  int done = 0;
  for (int pass = 0; pass < 2; ++pass) {
    for (; n > 0; --n) {
      atomicAdd(p.cnt + f.h, 1u);
      mark_line(p, f.h, f.line);
      ++done;
      bool gone;
      if (f.tM[0] < f.tM[1]) {
        gone = f.tM[0] < f.tM[2] ? far_step<0>(f, p) : far_step<2>(f, p);
      } else {
        gone = f.tM[1] < f.tM[2] ? far_step<1>(f, p) : far_step<2>(f, p);
      }
      if (gone) {
        f.left -= done;
        incs += static_cast<uint32_t>(done);
        return true;
      }
    }
    // At a limit, or where the endpoint could be: stop if on it, else (a
    // counter overshot) only the limits and the window remain.
    if (done >= lim || (f.e[0] | f.e[1] | f.e[2]) == 0) break;
    n = lim - done;
  }
  f.left -= done;
  incs += static_cast<uint32_t>(done);
  return f.left == 0 || (f.e[0] | f.e[1] | f.e[2]) == 0;
}
// ---- rays of an item ordered by length ----
// A warp runs until its longest ray ends, and rays of one azimuth column of
// a spinning LiDAR differ several-fold in how far they walk (beams that
// hit the ground near the sensor, beams that leave the window's top, beams
// clipped at max range).  A CTA therefore walks its item's rays in order of
// an estimate of their loop length (a counting sort on kOrderBins bins of
// kOrderStep iterations), so that the lanes of a warp end at about the same
// time.  Counts are sums of integer increments, so the order changes no
// result; the estimate only has to be cheap.

constexpr int kOrderBins = 32;
constexpr int kOrderStep = 32;   // loop iterations per bin
constexpr int kOrderCap = 1024;  // rays per item the CTA orders

struct RayOrder {
  float x[kOrderCap], y[kOrderCap], z[kOrderCap];  // the item's points, in input order
  uint16_t idx[kOrderCap];  // the item's rays, shortest estimate first
  int base[kOrderBins];
};

// Estimated loop iterations of the ray to (x, y, z): the L1 length in voxels
// of its segment, clipped at max range and at the window's box.
__device__ __forceinline__ int ray_len_estimate(const RayParams &p, float x, float y, float z) {
  const float d[3] = {x - p.o[0], y - p.o[1], z - p.o[2]};
  const float r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  if (!(r2 < 1e30f)) return 0;  // non-finite: the walk drops the ray at once
  float t = 1.0f;
  if (r2 > p.max_range * p.max_range) t = p.max_range * rsqrtf(r2);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float lo = static_cast<float>(p.win[a] - p.half[a]) * p.res;
    const float hi = static_cast<float>(p.win[a] + p.half[a] + 1) * p.res;
    if (d[a] > 0.0f) t = fminf(t, fmaxf(0.0f, (hi - p.o[a]) / d[a]));
    if (d[a] < 0.0f) t = fminf(t, fmaxf(0.0f, (lo - p.o[a]) / d[a]));
  }
  const float l1 = (fabsf(d[0]) + fabsf(d[1]) + fabsf(d[2])) * t * p.inv;
  return l1 < 1e9f ? static_cast<int>(l1) : 1 << 30;
}

// Fills `o` with the item's points start .. start + count - 1 and their
// order (count <= min(2 blockDim.x, kOrderCap)): o.idx[j] is the j-th
// shortest.  Each point is read once, here (the points may sit in host
// memory and be read over the bus).  Contains CTA barriers; every thread of
// the CTA calls it.
__device__ __forceinline__ void order_rays(const RayParams &p, int start, int count, RayOrder &o) {
  const int t = threadIdx.x, nt = blockDim.x;
  if (t < kOrderBins) o.base[t] = 0;
  __syncthreads();
  int bin[2] = {0, 0}, slot[2] = {0, 0};
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int j = t + r * nt;
    if (j < count) {
      const size_t k = static_cast<size_t>(start + j) * p.stride;
      const float x = p.x[k], y = p.y[k], z = p.z[k];
      o.x[j] = x;
      o.y[j] = y;
      o.z[j] = z;
      bin[r] = min(kOrderBins - 1, ray_len_estimate(p, x, y, z) / kOrderStep);
      slot[r] = atomicAdd(&o.base[bin[r]], 1);
    }
  }
  __syncthreads();
  if (t < 32) {  // exclusive prefix sum of the bin sizes
    const int c = o.base[t];
    int incl = c;
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, s);
      if (t >= s) incl += v;
    }
    o.base[t] = incl - c;
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int j = t + r * nt;
    if (j < count) o.idx[o.base[bin[r]] + slot[r]] = static_cast<uint16_t>(j);
  }
  __syncthreads();
}

}  // namespace cublox_b200

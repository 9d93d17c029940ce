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
// counters, and keeps the voxel's hash incrementally, with the ring
// buffer's wrap.  The voxels visited, and so the counts, are those of the
// single loop.

struct FarWalk {
  float tM[3], tD[3];  // as in RayWalk
  int e[3];     // steps to the endpoint's coordinate on the axis (all 0: at the endpoint)
  int out[3];   // steps the walk can still take on the axis inside the window
  int wrap[3];  // steps on the axis before its ring-buffer slot wraps
  int dh[3];    // hash change of one step on the axis
  int left;     // loop iterations left (max_steps - k)
  int h;        // hash of the current voxel
};

// The update after the loop (kernels.cu:138-151), fixed at the ray's start:
// endpoint hash (-1: endpoint outside the window), its cube cell (-1: not in
// the cube), and whether it counts a hit (not clipped at max range).
struct RayEnd {
  int h, c;
  bool hit;
};

constexpr int kNever = 0x7fffffff;  // counters of an axis the ray never steps on

template <int S>
__device__ __forceinline__ int cube_cell(int g0, int g1, int g2, const int clo[3]) {
  const int c0 = g0 - clo[0], c1 = g1 - clo[1], c2 = g2 - clo[2];
  if (S > 0 && static_cast<unsigned>(c0) < static_cast<unsigned>(S) &&
      static_cast<unsigned>(c1) < static_cast<unsigned>(S) &&
      static_cast<unsigned>(c2) < static_cast<unsigned>(S))
    return (c0 * S + c1) * S + c2;
  return -1;
}

template <int S>
__device__ __forceinline__ RayEnd ray_end_of(const RayParams &p, const RayWalk &w,
                                             const int clo[3]) {
  RayEnd r;
  r.h = end_hash(w, p);
  r.c = r.h >= 0 ? cube_cell<S>(w.en[0], w.en[1], w.en[2], clo) : -1;
  r.hit = !w.clipped;
  return r;
}

template <int S>
__device__ __forceinline__ void apply_end(const RayParams &p, uint32_t *cube, const RayEnd &r,
                                          uint32_t &incs, uint32_t &hits) {
  if (r.h < 0) return;
  if (S > 0 && r.c >= 0)
    atomicAdd(&cube[r.c], 1u);
  else
    atomicAdd(p.cnt + r.h, 1u);
  ++incs;
  if (r.hit) {
    atomicOr(p.cnt + r.h, kHitFlag);
    atomicAdd(p.hit + r.h, 1u);
    ++hits;
  }
}

// Far-phase state of a walk whose current voxel (loop iteration k, not yet
// counted) is inside the window.
__device__ __forceinline__ void to_far(const RayParams &p, const RayWalk &w, int k, FarWalk &f) {
  const int stride[3] = {p.map[1] * p.map[2], p.map[2], 1};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int d = w.en[a] - w.id[a];
    const int st = w.st[a];
    f.tM[a] = w.tM[a];
    f.tD[a] = w.tD[a];
    f.e[a] = st > 0 ? d : (st < 0 ? -d : d);
    f.out[a] = st > 0 ? p.half[a] - w.rel[a] : (st < 0 ? p.half[a] + w.rel[a] : kNever);
    f.wrap[a] = st > 0 ? p.map[a] - 1 - w.slot[a] : (st < 0 ? w.slot[a] : kNever);
    f.dh[a] = st * stride[a];
  }
  f.left = w.max_steps - k;
  f.h = walk_hash(w, p);
}

// One step on axis A (the tie rule picked it).  Returns true if the new
// voxel is outside the window, which ends the loop: the next iteration would
// break at its step limit, at the endpoint or as out of the window for good.
template <int A>
__device__ __forceinline__ bool far_step(FarWalk &f, int map_a) {
  f.tM[A] = fadd(f.tM[A], f.tD[A]);
  --f.e[A];
  if (f.wrap[A] == 0) {
    f.h += f.dh[A] * (1 - map_a);
    f.wrap[A] = map_a - 1;
  } else {
    f.h += f.dh[A];
    --f.wrap[A];
  }
  return f.out[A]-- == 0;
}

// Far phase for at most `budget` loop iterations; the ray's own step limit,
// window exit and endpoint end it earlier.  The endpoint test costs nothing
// per step: every step lowers one e counter by one, so the walk can stand on
// the endpoint only after exactly e0 + e1 + e2 steps (an axis it never steps
// on must already match), and not at all once a counter went negative.
// Until then only the limits and the window exit end the loop.  Every
// iteration counts the current voxel, then steps.
__device__ __forceinline__ void walk_far(const RayParams &p, FarWalk &f, int budget,
                                         uint32_t &incs) {
  const int lim = min(budget, f.left);
  bool reachable = true;
  int to_end = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (f.dh[a] == 0 ? f.e[a] != 0 : f.e[a] < 0) reachable = false;
    to_end += f.e[a];
  }
  int n = reachable ? min(lim, to_end) : lim;
  int done = 0;
  for (int pass = 0; pass < 2; ++pass) {
    for (; n > 0; --n) {
      atomicAdd(p.cnt + f.h, 1u);
      ++done;
      bool gone;
      if (f.tM[0] < f.tM[1]) {
        gone = f.tM[0] < f.tM[2] ? far_step<0>(f, p.map[0]) : far_step<2>(f, p.map[2]);
      } else {
        gone = f.tM[1] < f.tM[2] ? far_step<1>(f, p.map[1]) : far_step<2>(f, p.map[2]);
      }
      if (gone) {
        f.left -= done;
        incs += static_cast<uint32_t>(done);
        return;
      }
    }
    // At a limit, or where the endpoint could be: stop if on it, else (a
    // counter overshot) only the limits and the window remain.
    if (done >= lim || (f.e[0] | f.e[1] | f.e[2]) == 0) break;
    n = lim - done;
  }
  f.left -= done;
  incs += static_cast<uint32_t>(done);
}
}  // namespace cublox_b200

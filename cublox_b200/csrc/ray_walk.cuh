// Exact Amanatides–Woo walk state of one ray, as the reference sets it up
// (src/kernels.cu:44-137), shared by every raycast kernel.
#pragma once

#include <cstdint>

#include "exact_fp.cuh"
#include "kernels.cuh"

namespace cublox_b200 {

__device__ __forceinline__ float inf_f() { return __int_as_float(0x7f800000); }

__device__ __forceinline__ int wrap_slot(int s, int map) {
  return s >= map ? s - map : (s < 0 ? s + map : s);
}

struct RayWalk {
  int id[3];    // current global voxel
  int en[3];    // endpoint global voxel
  int st[3];    // step per axis (-1, 0, 1)
  int rel[3];   // id - window origin
  int slot[3];  // ring-buffer slot of id per axis, in [0, map)
  float tD[3], tM[3];
  int max_steps;
  bool clipped;
};

// Set up one ray (kernels.cu:44-105).  Returns false if the reference drops it.
__device__ __forceinline__ bool ray_begin(const RayParams &p, float ex,
                                          float ey, float ez, RayWalk &w) {
  const float ox = p.o[0], oy = p.o[1], oz = p.o[2];
  float dx = fsub(ex, ox), dy = fsub(ey, oy), dz = fsub(ez, oz);
  float L = fsqrt(sos(dx, dy, dz, (p.fp >> kFpRaySosShift) & 7u));
  if (L < 1e-6f || !isfinite(L) || !isfinite(ex) || !isfinite(ey) ||
      !isfinite(ez))
    return false;
  w.clipped = L > p.max_range;
  if (w.clipped) {
    const float s = fdiv(p.max_range, L);
    if (p.fp & kFpClipFma) {
      ex = ffma(dx, s, ox);
      ey = ffma(dy, s, oy);
      ez = ffma(dz, s, oz);
    } else {
      ex = fadd(ox, fmul(dx, s));
      ey = fadd(oy, fmul(dy, s));
      ez = fadd(oz, fmul(dz, s));
    }
    dx = fmul(dx, s);
    dy = fmul(dy, s);
    dz = fmul(dz, s);
    L = p.max_range;
  }
  const float invL = fdiv(1.0f, L);
  const float u[3] = {fmul(dx, invL), fmul(dy, invL), fmul(dz, invL)};
  const float oo[3] = {ox, oy, oz};
  const float ee[3] = {ex, ey, ez};
  const bool ctr = p.ctr != 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    w.id[a] = pos_to_global_dev(oo[a], p.inv, ctr, p.fp);
    w.en[a] = pos_to_global_dev(ee[a], p.inv, ctr, p.fp);
    w.st[a] = (u[a] > 0.0f) - (u[a] < 0.0f);
    w.tD[a] = w.st[a] == 0 ? inf_f() : fabsf(fdiv(p.res, u[a]));
    float t;
    if (ctr) {
      t = fadd(static_cast<float>(w.id[a]), fmul(0.5f, static_cast<float>(w.st[a])));
    } else {
      t = fadd(static_cast<float>(w.id[a]), static_cast<float>(w.st[a] > 0));
    }
    const float num = (p.fp & kFpBoundFma) ? ffma(t, p.res, -oo[a])
                                           : fsub(fmul(t, p.res), oo[a]);
    w.tM[a] = w.st[a] == 0 ? inf_f() : fdiv(num, u[a]);
    w.rel[a] = w.id[a] - p.win[a];
    w.slot[a] = global_to_local(w.id[a], p.map[a], p.half[a]) + p.half[a];
  }
  w.max_steps = abs(w.en[0] - w.id[0]) + abs(w.en[1] - w.id[1]) +
                abs(w.en[2] - w.id[2]) + 4;
  return true;
}

__device__ __forceinline__ bool at_end(const RayWalk &w) {
  return w.id[0] == w.en[0] && w.id[1] == w.en[1] && w.id[2] == w.en[2];
}

__device__ __forceinline__ bool in_window(const RayWalk &w, const RayParams &p) {
  return abs(w.rel[0]) <= p.half[0] && abs(w.rel[1]) <= p.half[1] &&
         abs(w.rel[2]) <= p.half[2];
}

// Outside on some axis and not moving back: no later voxel is inside.
__device__ __forceinline__ bool left_for_good(const RayWalk &w, const RayParams &p) {
  return (abs(w.rel[0]) > p.half[0] && w.rel[0] * w.st[0] >= 0) ||
         (abs(w.rel[1]) > p.half[1] && w.rel[1] * w.st[1] >= 0) ||
         (abs(w.rel[2]) > p.half[2] && w.rel[2] * w.st[2] >= 0);
}

// Address of the current voxel in the map's arrays.
__device__ __forceinline__ int walk_hash(const RayWalk &w, const RayParams &p) {
  return vox_addr(p.lay, w.slot[0], w.slot[1], w.slot[2]);
}

// Flag the line of address h as holding a counted voxel (a plain byte
// store: every writer stores the same 1).  `last` is the line this thread
// flagged last, so a run of increments on one line stores once.
__device__ __forceinline__ void mark_line(const RayParams &p, int h, int &last) {
  const int line = h >> kLineShift;
  if (line != last) {
    last = line;
    if (p.dirty) p.dirty[line] = 1;
  }
}

// One step, tie rule of kernels.cu:120-136.  Returns the axis stepped.
__device__ __forceinline__ int ray_step(RayWalk &w, const RayParams &p) {
  int a;
  if (w.tM[0] < w.tM[1]) {
    a = w.tM[0] < w.tM[2] ? 0 : 2;
  } else {
    a = w.tM[1] < w.tM[2] ? 1 : 2;
  }
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
  return a;
}

// Address of an in-window voxel given by its global index.
__device__ __forceinline__ int global_addr(const RayParams &p, int g0, int g1, int g2) {
  return vox_addr(p.lay, global_to_local(g0, p.map[0], p.half[0]) + p.half[0],
                  global_to_local(g1, p.map[1], p.half[1]) + p.half[1],
                  global_to_local(g2, p.map[2], p.half[2]) + p.half[2]);
}

// Endpoint address if the endpoint voxel is in the window, else -1.
__device__ __forceinline__ int end_hash(const RayWalk &w, const RayParams &p) {
  if (abs(w.en[0] - p.win[0]) > p.half[0] || abs(w.en[1] - p.win[1]) > p.half[1] ||
      abs(w.en[2] - p.win[2]) > p.half[2])
    return -1;
  return global_addr(p, w.en[0], w.en[1], w.en[2]);
}

}  // namespace cublox_b200

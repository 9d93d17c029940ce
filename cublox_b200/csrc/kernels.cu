// Device kernels of the map-integration path (sm_100a).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "fold.cuh"
#include "kernels.cuh"
#include "ray_walk.cuh"

namespace cublox_b200 {

namespace {

// One ray, op for op as rayCastUpdateKernel (kernels.cu:44-151), with the
// window test and hash kept incrementally and the walk cut short once the
// ray has left the window for good (indices are monotone per axis, so no
// later voxel of the loop can be inside).  Returns false if dropped.
// kAccount: count the reference loop's iterations instead (no early exit,
// no counters touched); u_incs gets iterations + 1.
template <bool kAccount = false>
__device__ __forceinline__ bool cast_one(const RayParams &p, float ex,
                                         float ey, float ez, uint32_t &u_incs,
                                         uint32_t &h_incs) {
  RayWalk w;
  if (!ray_begin(p, ex, ey, ez, w)) return false;
  uint32_t incs = 0;
  int last = -1;  // line flagged last
  for (int step = 0; step < w.max_steps; ++step) {
    if (at_end(w)) break;
    if (kAccount) {
      ++incs;
    } else if (in_window(w, p)) {
      const int h = walk_hash(w, p);
      atomicAdd(p.cnt + h, 1u);
      mark_line(p, h, last);
      ++incs;
    } else if (left_for_good(w, p)) {
      break;
    }
    ray_step(w, p);
  }
  if (kAccount) {
    u_incs += incs + 1;
    return true;
  }
  // Endpoint: op, and hit unless clipped (kernels.cu:139-151).
  const int h = end_hash(w, p);
  if (h >= 0) {
    atomicAdd(p.cnt + h, 1u);
    mark_line(p, h, last);
    if (!w.clipped) {
      atomicOr(p.cnt + h, kHitFlag);
      atomicAdd(p.hit + h, 1u);
      ++h_incs;
    }
    ++incs;
  }
  u_incs += incs;
  return true;
}

template <bool kStats>
__global__ void __launch_bounds__(256) raycast_kernel(const RayParams p) {
  uint32_t rays = 0, u = 0, hh = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n;
       i += gridDim.x * blockDim.x) {
    const size_t k = static_cast<size_t>(i) * p.stride;
    if (cast_one(p, p.x[k], p.y[k], p.z[k], u, hh)) ++rays;
  }
  if (kStats) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      rays += __shfl_down_sync(0xffffffffu, rays, off);
      u += __shfl_down_sync(0xffffffffu, u, off);
      hh += __shfl_down_sync(0xffffffffu, hh, off);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(p.stats + 0, static_cast<unsigned long long>(rays));
      atomicAdd(p.stats + 1, static_cast<unsigned long long>(u));
      atomicAdd(p.stats + 2, static_cast<unsigned long long>(hh));
    }
  }
}

__global__ void __launch_bounds__(256) step_count_kernel(const RayParams p) {
  uint32_t it = 0, hh = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n;
       i += gridDim.x * blockDim.x) {
    const size_t k = static_cast<size_t>(i) * p.stride;
    cast_one<true>(p, p.x[k], p.y[k], p.z[k], it, hh);
  }
  unsigned long long v = it;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(p.stats, v);
}

__device__ __forceinline__ FoldView fold_view(const ApplyParams &p) {
  return FoldView{p.occ, p.cnt, p.hit, p.vnum, p.l_hit, p.l_miss, p.l_min, p.l_max,
                  p.l_unknown, p.fp};
}

// Fold one voxel's counters in place (applyUpdateKernel, kernels.cu:179-200).
__device__ __forceinline__ void fold(const ApplyParams &p, int h, uint32_t c) {
  p.occ[h] = fold_counter(fold_view(p), h, c, p.occ[h]);
}

template <bool kStats>
__global__ void __launch_bounds__(256) apply_sweep_kernel(const ApplyParams p) {
  const int n4 = p.vnum >> 2;
  uint32_t touched = 0;
  uint4 *c4 = reinterpret_cast<uint4 *>(p.cnt);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n4;
       i += gridDim.x * blockDim.x) {
    const uint4 c = c4[i];
    if ((c.x | c.y | c.z | c.w) == 0u) continue;
    const int h = i << 2;
    if (c.x) { fold(p, h + 0, c.x); ++touched; }
    if (c.y) { fold(p, h + 1, c.y); ++touched; }
    if (c.z) { fold(p, h + 2, c.z); ++touched; }
    if (c.w) { fold(p, h + 3, c.w); ++touched; }
    c4[i] = make_uint4(0u, 0u, 0u, 0u);
  }
  // tail (vnum not a multiple of 4)
  if (blockIdx.x == 0 && threadIdx.x < (p.vnum & 3)) {
    const int h = (n4 << 2) + threadIdx.x;
    const uint32_t c = p.cnt[h];
    if (c) {
      fold(p, h, c);
      p.cnt[h] = 0u;
      ++touched;
    }
  }
  if (kStats) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
      touched += __shfl_down_sync(0xffffffffu, touched, off);
    if ((threadIdx.x & 31) == 0 && touched)
      atomicAdd(p.stats + 3, static_cast<unsigned long long>(touched));
  }
}

// Grid-stride sweep of 16-byte counter groups, four counter loads in flight
// per thread (fold_groups); the vnum % 4 tail by block 0.
template <bool kStats>
__global__ void __launch_bounds__(256) fold_vec_kernel(const ApplyParams p) {
  const FoldView v = fold_view(p);
  uint32_t touched = fold_groups<4, false>(v, blockIdx.x * blockDim.x + threadIdx.x,
                                           p.vnum >> 2, gridDim.x * blockDim.x);
  if (blockIdx.x == 0) touched += fold_tail(v);
  if (kStats) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
      touched += __shfl_down_sync(0xffffffffu, touched, off);
    if ((threadIdx.x & 31) == 0 && touched)
      atomicAdd(p.stats + 3, static_cast<unsigned long long>(touched));
  }
}

// Fold of the flagged lines only: each warp takes groups of 32 line flags,
// grid-stride (fold_lines).
template <bool kStats>
__global__ void __launch_bounds__(256) fold_lines_kernel(const ApplyParams p) {
  const FoldView v = fold_view(p);
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  uint32_t touched = fold_lines<8, false>(v, p.dirty, warp * 32, p.nlines, warps * 32);
  if (kStats) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
      touched += __shfl_down_sync(0xffffffffu, touched, off);
    if ((threadIdx.x & 31) == 0 && touched)
      atomicAdd(p.stats + 3, static_cast<unsigned long long>(touched));
  }
}

// Fold of the flagged lines through per-CTA line lists (fold.cuh,
// build_line_list / fold_line_list): CTA b takes items of kListLines lines
// b, b + grid, ... and loads the next item's flags before folding the
// current list.
template <bool kStats>
__global__ void __launch_bounds__(kListThreads, 4) fold_list_kernel(const ApplyParams p,
                                                                     int item_lines) {
  __shared__ LineList L;
  __shared__ HitQueue hq;
  if (threadIdx.x == 0) hq.n = 0;  // the first read follows build_line_list's barriers
  const FoldView v = fold_view(p);
  const int items = (p.nlines + item_lines - 1) / item_lines;
  auto count_of = [&](int it) { return min(item_lines, p.nlines - it * item_lines); };
  int it = blockIdx.x;
  uint4 f = make_uint4(0u, 0u, 0u, 0u);
  if (it < items) f = load_line_flags(p.dirty, it * item_lines, count_of(it));
  uint32_t touched = 0;
  for (; it < items; it += gridDim.x) {
    const int start = it * item_lines;
    const int n = build_line_list(line_flag_bits(f), L, p.dirty, start, count_of(it));
    const int next = it + gridDim.x;
    if (next < items) f = load_line_flags(p.dirty, next * item_lines, count_of(next));
    touched += fold_line_list<4, false>(v, L.line, n, start, &hq);
    __syncthreads();
    fold_hit_queue(v, hq);  // ends with a barrier: the list is rewritten next
  }
  if (kStats) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
      touched += __shfl_down_sync(0xffffffffu, touched, off);
    if ((threadIdx.x & 31) == 0 && touched)
      atomicAdd(p.stats + 3, static_cast<unsigned long long>(touched));
  }
}

// Union-of-slabs clear.  One block per x slot: a marked x slab is one
// contiguous run of ny*nz floats; otherwise every (x, y) column clears its
// whole run if y is marked, else the marked z slots.
__global__ void __launch_bounds__(256) clear_kernel(const ClearParams p) {
  extern __shared__ uint32_t sm[];
  const int nx = p.map[0], ny = p.map[1], nz = p.map[2];
  const int wy = (ny + 31) >> 5, wz = (nz + 31) >> 5;
  uint32_t *my = sm;
  int *zl = reinterpret_cast<int *>(sm + wy);
  __shared__ int nzl;
  for (int i = threadIdx.x; i < wy; i += blockDim.x) my[i] = p.ymask[i];
  if (threadIdx.x == 0) {
    int c = 0;
    if (p.any_z)
      for (int w = 0; w < wz; ++w) {
        uint32_t b = p.zmask[w];
        while (b) {
          const int k = __ffs(b) - 1;
          b &= b - 1;
          zl[c++] = w * 32 + k;
        }
      }
    nzl = c;
  }
  __syncthreads();
  for (int lx = blockIdx.x; lx < nx; lx += gridDim.x) {
    float *base = p.occ + static_cast<size_t>(lx) * ny * nz;
    if ((p.xmask[lx >> 5] >> (lx & 31)) & 1u) {
      if (p.x_done) continue;
      const int n = ny * nz;
      for (int i = threadIdx.x; i < n; i += blockDim.x) base[i] = 0.0f;
      continue;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nw = blockDim.x >> 5;
    for (int ly = warp; ly < ny; ly += nw) {
      float *col = base + static_cast<size_t>(ly) * nz;
      if ((my[ly >> 5] >> (ly & 31)) & 1u) {
        for (int z = lane; z < nz; z += 32) col[z] = 0.0f;
      } else {
        for (int k = lane; k < nzl; k += 32) col[zl[k]] = 0.0f;
      }
    }
  }
}

// Union-of-slabs clear for 32-voxel brick layouts.  A warp takes up to
// kClearZ bricks of one (x brick, y brick) column at a time, a lane per
// voxel of a brick: the columns of the listed x bricks crossed with every y
// brick, then of every x brick crossed with the listed y bricks (the warp
// walks consecutive 128-byte lines of the column), then of every (x, y)
// brick for the listed z bricks.  A lane clears its voxel if its x, y or z
// slot is marked; lanes of padding slots (past the map) do nothing; a brick
// on two lists is cleared twice, with the same result.  Index divisions are
// per run of lines, not per brick.
constexpr int kClearZ = 8;

__global__ void __launch_bounds__(256) clear_bricks_kernel(const ClearParams p) {
  const int lane = threadIdx.x & 31;
  const int chunks = (p.nbr[2] + kClearZ - 1) / kClearZ;  // runs of z bricks per column
  const int u0 = p.nb[0] * p.nbr[1] * chunks;  // listed x bricks x every y brick
  const int u1 = p.nbr[0] * p.nb[1] * chunks;  // every x brick x listed y bricks
  const int u2 = p.nb[2] > 0 ? p.nbr[0] * p.nbr[1] : 0;
  const int units = u0 + u1 + u2;
  const int l12 = p.lay.lb[1] + p.lay.lb[2];
  const int i0 = lane >> l12;
  const int i1 = (lane >> p.lay.lb[2]) & ((1 << p.lay.lb[1]) - 1);
  const int i2 = lane & ((1 << p.lay.lb[2]) - 1);
  auto marked = [](const uint32_t *m, int s) { return ((m[s >> 5] >> (s & 31)) & 1u) != 0u; };
  for (int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < units;
       u += (gridDim.x * blockDim.x) >> 5) {
    int bx, by, z0 = 0;
    if (u < u0) {
      const int col = u / chunks;
      z0 = (u - col * chunks) * kClearZ;
      bx = p.blist[col / p.nbr[1]];
      by = col % p.nbr[1];
    } else if (u < u0 + u1) {
      const int v = u - u0, col = v / chunks;
      z0 = (v - col * chunks) * kClearZ;
      bx = col / p.nb[1];
      by = p.blist[p.nb[0] + col % p.nb[1]];
    } else {
      const int v = u - u0 - u1;
      bx = v / p.nbr[1];
      by = v % p.nbr[1];
    }
    const int s0 = (bx << p.lay.lb[0]) + i0, s1 = (by << p.lay.lb[1]) + i1;
    if (s0 >= p.map[0] || s1 >= p.map[1]) continue;
    const bool xy = marked(p.xmask, s0) || marked(p.ymask, s1);
    float *col = p.occ + bx * p.lay.bs[0] + by * p.lay.bs[1] + lane;
    if (u < u0 + u1) {
      const int z1 = min(z0 + kClearZ, p.nbr[2]);
      for (int bz = z0; bz < z1; ++bz) {
        const int s2 = (bz << p.lay.lb[2]) + i2;
        if (s2 < p.map[2] && (xy || (p.any_z && marked(p.zmask, s2))))
          col[bz * p.lay.bs[2]] = 0.0f;
      }
    } else {
      for (int j = 0; j < p.nb[2]; ++j) {
        const int bz = p.blist[p.nb[0] + p.nb[1] + j];
        const int s2 = (bz << p.lay.lb[2]) + i2;
        if (s2 < p.map[2] && marked(p.zmask, s2)) col[bz * p.lay.bs[2]] = 0.0f;
      }
    }
  }
}

// Layout <-> the reference's hash order, one thread per hash.
__global__ void __launch_bounds__(256) relayout_kernel(const float *src, float *dst,
                                                       const VoxLayout lay, const int ny,
                                                       const int nz, const long long vnum,
                                                       const int to_ref) {
  const long long nyz = static_cast<long long>(ny) * nz;
  for (long long h = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; h < vnum;
       h += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int sx = static_cast<int>(h / nyz);
    const int r = static_cast<int>(h - sx * nyz);
    const int sy = r / nz, sz = r - sy * nz;
    const int a = vox_addr(lay, sx, sy, sz);
    if (to_ref)
      dst[h] = src[a];
    else
      dst[a] = src[h];
  }
}

// Sphere fetch over host-clipped candidate boxes, one block per query
// (grid-stride), candidates in (x, y, z) order with z fastest so that
// consecutive threads read consecutive voxels of one column.  Pass 1 counts,
// pass 2 writes the first `limits[q]` samples at `offsets[q]` in that order.
template <int kPass>
__global__ void __launch_bounds__(256) fetch_kernel(const FetchParams p) {
  __shared__ int warp_tot[8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int u = blockIdx.x; u < p.nu; u += gridDim.x) {
    const int q = p.uq[u];
    const int *b = p.qbox + 8 * q;
    const int gx0 = b[0], gy0 = b[2], gz0 = b[4];
    const int nx = b[1] - b[0] + 1, nyy = b[3] - b[2] + 1, nzz = b[5] - b[4] + 1;
    const float c[3] = {p.centers[3 * q], p.centers[3 * q + 1],
                        p.centers[3 * q + 2]};
    const float r2 = p.qr2[q];
    long long running = 0;
    const long long limit = kPass == 2 ? p.limits[u] : 0;
    const long long base_off = kPass == 2 ? p.offsets[u] : 0;
    const long long all = (nx > 0 && nyy > 0 && nzz > 0)
                              ? static_cast<long long>(nx) * nyy * nzz
                              : 0;
    const long long t_begin = p.ut0[u];
    const long long total = min(all, t_begin + p.unit);  // end of this unit
    for (long long t0 = t_begin; t0 < total; t0 += blockDim.x) {
      if (kPass == 2 && running >= limit) break;
      const long long t = t0 + threadIdx.x;
      bool keep = false;
      float pos[3];
      uint8_t state = 0;
      if (t < total) {
        const int iz = static_cast<int>(t % nzz);
        const long long r = t / nzz;
        const int iy = static_cast<int>(r % nyy);
        const int ix = static_cast<int>(r / nyy);
        const int g[3] = {gx0 + ix, gy0 + iy, gz0 + iz};
        float d[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const float tt = p.ctr ? static_cast<float>(g[a])
                                 : fadd(static_cast<float>(g[a]), 0.5f);
          pos[a] = fmul(tt, p.res);
          d[a] = (p.fp & kFpFetchDFma) ? ffma(tt, p.res, -c[a])
                                       : fsub(pos[a], c[a]);
        }
        const float s = sos(d[0], d[1], d[2], (p.fp >> kFpFetchSosShift) & 7u);
        if (!(s > r2)) {
          const int h = vox_addr(p.lay, global_to_local(g[0], p.map[0], p.half[0]) + p.half[0],
                                 global_to_local(g[1], p.map[1], p.half[1]) + p.half[1],
                                 global_to_local(g[2], p.map[2], p.half[2]) + p.half[2]);
          const float l = fadd(p.occ[h], p.l_unknown);
          state = l >= p.l_occ ? 2 : (l < p.l_free ? 1 : 0);
          keep = p.filter < 0 || static_cast<int>(state) == p.filter;
        }
      }
      const uint32_t bal = __ballot_sync(0xffffffffu, keep);
      if (lane == 0) warp_tot[warp] = __popc(bal);
      __syncthreads();
      int before = 0, blk = 0;
#pragma unroll
      for (int w = 0; w < 8; ++w) {
        const int v = warp_tot[w];
        before += w < warp ? v : 0;
        blk += v;
      }
      if (kPass == 2 && keep) {
        const long long rank =
            running + before + __popc(bal & ((1u << lane) - 1u));
        if (rank < limit) {
          const long long o = base_off + rank;
          p.out_pos[3 * o + 0] = pos[0];
          p.out_pos[3 * o + 1] = pos[1];
          p.out_pos[3 * o + 2] = pos[2];
          p.out_state[o] = state;
        }
      }
      running += blk;
      __syncthreads();
    }
    if (kPass == 1 && threadIdx.x == 0) p.counts[u] = running;
  }
}

// Host-side float->int of the reference's point queries (x86 cvttss2si:
// NaN or out of range gives INT_MIN).
__device__ __forceinline__ int f2i_hostlike(float v) {
  return (v >= -2147483648.0f && v < 2147483648.0f) ? static_cast<int>(v)
                                                    : (-2147483647 - 1);
}

__global__ void __launch_bounds__(256) query_kernel(const QueryParams p) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n;
       i += gridDim.x * blockDim.x) {
    int g[3];
    bool in = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float v = p.xyz[3 * static_cast<size_t>(i) + a];
      const float m = fmul(v, p.inv);
      g[a] = p.ctr ? f2i_hostlike(fadd(m, v < 0.0f ? -0.5f : 0.5f))
                   : f2i_hostlike(ffloor(m));
      in = in && abs(g[a] - p.win[a]) <= p.half[a];
    }
    uint8_t st = 0;
    if (in) {
      const int h = vox_addr(p.lay, global_to_local(g[0], p.map[0], p.half[0]) + p.half[0],
                             global_to_local(g[1], p.map[1], p.half[1]) + p.half[1],
                             global_to_local(g[2], p.map[2], p.half[2]) + p.half[2]);
      const float l = fadd(p.occ[h], p.l_unknown);
      st = l >= p.l_occ ? 2 : (l < p.l_free ? 1 : 0);
    }
    p.out[i] = st;
  }
}

__global__ void gather_soa_kernel(const float *xyz, int layout, int n,
                                  float *dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    if (layout == 1) {
      dst[i] = xyz[3 * static_cast<size_t>(i)];
      dst[n + i] = xyz[3 * static_cast<size_t>(i) + 1];
      dst[2 * static_cast<size_t>(n) + i] = xyz[3 * static_cast<size_t>(i) + 2];
    }
  }
}

// One point of buildCloudInOdomFrame (main.cpp:666-684), in its FP32 order
// on x86-64 without FMA: squaredNorm as (x*x + y*y) + z*z, the isometry as
// ((r0*x + r1*y) + r2*z) + t per row; a dropped point is written as NaN.
__device__ __forceinline__ void ingest_point(const IngestParams &p, int i, float x, float y,
                                             float z) {
  float w[3];
  bool keep = isfinite(x) && isfinite(y) && isfinite(z);
  if (keep) keep = !(fadd(fadd(fmul(x, x), fmul(y, y)), fmul(z, z)) > p.max_r2);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float *r = p.R + 3 * a;
    w[a] = keep ? fadd(fadd(fadd(fmul(r[0], x), fmul(r[1], y)), fmul(r[2], z)), p.t[a])
                : __int_as_float(0x7fc00000);
  }
  p.dst[i] = w[0];
  p.dst[p.n + i] = w[1];
  p.dst[2 * static_cast<size_t>(p.n) + i] = w[2];
  if (p.count && keep) atomicAdd(p.count, 1);
}

__global__ void __launch_bounds__(256) ingest_kernel(const IngestParams p) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n;
       i += gridDim.x * blockDim.x) {
    if (p.layout == 1)
      ingest_point(p, i, p.xyz[3 * static_cast<size_t>(i)], p.xyz[3 * static_cast<size_t>(i) + 1],
                   p.xyz[3 * static_cast<size_t>(i) + 2]);
    else
      ingest_point(p, i, p.xyz[i], p.xyz[p.col + i], p.xyz[2 * static_cast<size_t>(p.col) + i]);
  }
}

// One pixel of depthCallback (main.cpp:596-631): invalid depth (16-bit 0;
// float non-finite or <= 0) gives NaN; else z in metres, x = ((u - cx) * z)
// / fx, y = ((v - cy) * z) / fy, then ingest_point.
__global__ void __launch_bounds__(256) depth_kernel(const DepthParams p) {
  const int n = p.ingest.n;  // pixels used (the driver's cloud cap)
  const float nan = __int_as_float(0x7fc00000);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int v = i / p.width, u = i - v * p.width;
    const unsigned char *row = p.image + static_cast<long long>(v) * p.step;
    float z;
    bool valid;
    if (p.encoding == 0) {
      const uint16_t raw = reinterpret_cast<const uint16_t *>(row)[u];
      valid = raw != 0;
      z = fmul(static_cast<float>(raw), 0.001f);
    } else {
      z = reinterpret_cast<const float *>(row)[u];
      valid = isfinite(z) && z > 0.0f;
    }
    if (!valid) {
      ingest_point(p.ingest, i, nan, nan, nan);
      continue;
    }
    const float x = fdiv(fmul(fsub(static_cast<float>(u), p.cx), z), p.fx);
    const float y = fdiv(fmul(fsub(static_cast<float>(v), p.cy), z), p.fy);
    ingest_point(p.ingest, i, x, y, z);
  }
}

// occupancyVizDropBySubsample (main.cpp:71-84): the host's binning (no FMA)
// of the sample position, x ^ y ^ z of the global index, modulo step.
__device__ __forceinline__ bool viz_drop(const VizParams &p, const float *q) {
  if (p.step <= 1) return false;
  const unsigned mix = static_cast<unsigned>(pos_to_global_dev(q[0], p.inv, p.ctr != 0, 0u)) ^
                       static_cast<unsigned>(pos_to_global_dev(q[1], p.inv, p.ctr != 0, 0u)) ^
                       static_cast<unsigned>(pos_to_global_dev(q[2], p.inv, p.ctr != 0, 0u));
  return (mix % static_cast<unsigned>(p.step)) != 0u;
}

// distanceToOccupancyColor + packRGBFloat (main.cpp:275-304): distance by
// Eigen's norm, sqrt((dx*dx + dy*dy) + dz*dz).
__device__ __forceinline__ float viz_rgb(const VizParams &p, const float *q) {
  const float dx = fsub(q[0], p.o[0]), dy = fsub(q[1], p.o[1]), dz = fsub(q[2], p.o[2]);
  const float d = fsqrt(fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz)));
  const float dm = fmaxf(p.d_max, 1.0f);
  const float t = fminf(fmaxf(fdiv(d, dm), 0.0f), 1.0f);
  float r, g, b;
  if (t <= 0.5f) {
    const float k = fmul(t, 2.0f);
    r = 0.0f;
    g = fsub(1.0f, k);
    b = k;
  } else {
    const float k = fmul(fsub(t, 0.5f), 2.0f);
    r = k;
    g = 0.0f;
    b = fsub(1.0f, k);
  }
  auto c8 = [](float c) {
    return static_cast<uint32_t>(fmul(fminf(fmaxf(c, 0.0f), 1.0f), 255.0f));
  };
  return __uint_as_float((c8(r) << 16) | (c8(g) << 8) | c8(b));
}

// One block walks the samples in order, 1024 at a time, and compacts the
// kept ones with a block-wide prefix sum, so the output keeps the sample
// order; it stops at max_points.
__global__ void __launch_bounds__(1024) viz_kernel(const VizParams p) {
  __shared__ int warp_sum[32];
  __shared__ long long s_base;
  if (threadIdx.x == 0) s_base = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (long long c0 = 0; c0 < p.n; c0 += blockDim.x) {
    const long long i = c0 + threadIdx.x;
    const bool keep = i < p.n && !viz_drop(p, p.pos + 3 * i);
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) warp_sum[warp] = __popc(m);
    __syncthreads();
    if (warp == 0) {
      const int nw = blockDim.x >> 5;
      int v = lane < nw ? warp_sum[lane] : 0;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, v, off);
        if (lane >= off) v += y;
      }
      if (lane < nw) warp_sum[lane] = v;  // inclusive
    }
    __syncthreads();
    const long long base = s_base;
    const long long at = base + (warp ? warp_sum[warp - 1] : 0) + __popc(m & ((1u << lane) - 1u));
    if (keep && at < p.max_points) {
      const float *q = p.pos + 3 * i;
      float4 v;
      v.x = q[0];
      v.y = q[1];
      v.z = q[2];
      v.w = viz_rgb(p, q);
      reinterpret_cast<float4 *>(p.out)[at] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) s_base = base + warp_sum[(blockDim.x >> 5) - 1];
    __syncthreads();
    if (s_base >= p.max_points) break;
  }
  if (threadIdx.x == 0) *p.written = s_base < p.max_points ? s_base : p.max_points;
}

int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

}  // namespace

void launch_raycast(const RayParams &p, cudaStream_t s) {
  if (p.n <= 0) return;
  const int block = 256;
  int grid = (p.n + block - 1) / block;
  if (p.stats)
    raycast_kernel<true><<<grid, block, 0, s>>>(p);
  else
    raycast_kernel<false><<<grid, block, 0, s>>>(p);
}

int kernel_binary_version() {
  cudaFuncAttributes a{};
  if (cudaFuncGetAttributes(&a, step_count_kernel) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return a.binaryVersion;
}

void launch_step_count(const RayParams &p, cudaStream_t s) {
  if (p.n <= 0) return;
  step_count_kernel<<<(p.n + 255) / 256, 256, 0, s>>>(p);
}

void launch_apply(const ApplyParams &p, cudaStream_t s) {
  if (p.variant == 2) {
    if (p.nlines <= 0) return;
    // items of up to 4,096 lines, smaller for small maps so that every SM
    // gets some (a multiple of 16 lines keeps the 16-byte flag loads aligned)
    const int cap = sm_count() * 4;
    int item_lines = (p.nlines + cap - 1) / cap;
    item_lines = ((item_lines + 255) / 256) * 256;
    if (item_lines > kListLines) item_lines = kListLines;
    int grid = (p.nlines + item_lines - 1) / item_lines;
    if (grid > cap) grid = cap;
    if (p.stats)
      fold_list_kernel<true><<<grid, kListThreads, 0, s>>>(p, item_lines);
    else
      fold_list_kernel<false><<<grid, kListThreads, 0, s>>>(p, item_lines);
    return;
  }
  if (p.variant == 3) {
    if (p.nlines <= 0) return;
    const int groups = (p.nlines + 31) / 32;  // one warp per group of 32 lines
    int grid = (groups + 7) / 8;
    const int cap = sm_count() * 8;
    if (grid > cap) grid = cap;
    if (p.stats)
      fold_lines_kernel<true><<<grid, 256, 0, s>>>(p);
    else
      fold_lines_kernel<false><<<grid, 256, 0, s>>>(p);
    return;
  }
  if (p.vnum <= 0) return;
  const int block = 256;
  const int n4 = (p.vnum >> 2) + 1;
  int grid = (n4 + block - 1) / block;
  const int cap = sm_count() * 16;
  if (grid > cap) grid = cap;
  if (p.variant == 1) {
    if (p.stats)
      fold_vec_kernel<true><<<grid, block, 0, s>>>(p);
    else
      fold_vec_kernel<false><<<grid, block, 0, s>>>(p);
    return;
  }
  if (p.stats)
    apply_sweep_kernel<true><<<grid, block, 0, s>>>(p);
  else
    apply_sweep_kernel<false><<<grid, block, 0, s>>>(p);
}

void launch_relayout(const float *src, float *dst, const VoxLayout &lay, const int map[3],
                     int to_ref, cudaStream_t s) {
  const long long v = static_cast<long long>(map[0]) * map[1] * map[2];
  if (v <= 0) return;
  long long grid = (v + 255) / 256;
  if (grid > sm_count() * 32) grid = sm_count() * 32;
  relayout_kernel<<<static_cast<int>(grid), 256, 0, s>>>(src, dst, lay, map[1], map[2], v, to_ref);
}

void launch_clear(const ClearParams &p, cudaStream_t s) {
  if (p.blist) {
    const long long chunks = (p.nbr[2] + kClearZ - 1) / kClearZ;
    const long long units = static_cast<long long>(p.nb[0]) * p.nbr[1] * chunks +
                            static_cast<long long>(p.nbr[0]) * p.nb[1] * chunks +
                            (p.nb[2] > 0 ? static_cast<long long>(p.nbr[0]) * p.nbr[1] : 0);
    if (units <= 0) return;
    long long grid = (units + 7) / 8;  // a run of a column's bricks per warp
    if (grid > sm_count() * 16) grid = sm_count() * 16;
    clear_bricks_kernel<<<static_cast<int>(grid), 256, 0, s>>>(p);
    return;
  }
  const int wy = (p.map[1] + 31) >> 5;
  const size_t smem = sizeof(uint32_t) * wy + sizeof(int) * (p.map[2] + 1);
  int grid = p.map[0];
  clear_kernel<<<grid, 256, smem, s>>>(p);
}

void launch_fetch(const FetchParams &p, int pass, cudaStream_t s) {
  if (p.nu <= 0) return;
  int grid = p.nu;
  const int cap = sm_count() * 8;
  if (grid > cap) grid = cap;
  if (pass == 1)
    fetch_kernel<1><<<grid, 256, 0, s>>>(p);
  else
    fetch_kernel<2><<<grid, 256, 0, s>>>(p);
}

void launch_query(const QueryParams &p, cudaStream_t s) {
  if (p.n <= 0) return;
  int grid = (p.n + 255) / 256;
  query_kernel<<<grid, 256, 0, s>>>(p);
}

void launch_gather_soa(const float *xyz, int layout, int n, float *dst,
                       cudaStream_t s) {
  if (n <= 0) return;
  int grid = (n + 255) / 256;
  gather_soa_kernel<<<grid, 256, 0, s>>>(xyz, layout, n, dst);
}

void launch_ingest(const IngestParams &p, cudaStream_t s) {
  if (p.n <= 0) return;
  ingest_kernel<<<(p.n + 255) / 256, 256, 0, s>>>(p);
}

void launch_viz(const VizParams &p, cudaStream_t s) { viz_kernel<<<1, 1024, 0, s>>>(p); }

void launch_depth(const DepthParams &p, cudaStream_t s) {
  const int n = p.ingest.n;
  if (n <= 0) return;
  depth_kernel<<<(n + 255) / 256, 256, 0, s>>>(p);
}

}  // namespace cublox_b200

// Fold of a scan's per-voxel counters into the stored log-odds
// (the reference's applyUpdateKernel, src/kernels.cu:167-208), shared by the
// single-grid sweep and the batched launches.
//
// Counter word: bits 0..30 traversal count, bit 31 "has a hit"; the hit count
// itself sits in a second array, read only for flagged voxels.
#pragma once

#include <cstdint>

#include "exact_fp.cuh"
#include "kernels.cuh"

namespace cublox_b200 {

struct FoldView {
  float *occ;
  uint32_t *cnt;
  uint32_t *hit;
  int vnum;
  float l_hit, l_miss, l_min, l_max, l_unknown;
  unsigned fp;
};

// One voxel: miss = op - hit (never negative), stored value shifted by
// l_unknown, miss then hit added (fused or not as the pinned contraction
// says), clamped, shifted back (kernels.cu:179-200).  The hit count is read
// at L2 (ld.global.cg): in a fused launch other CTAs of the same kernel
// wrote it.
__device__ __forceinline__ float fold_counter(const FoldView &v, int h, uint32_t c, float s0) {
  const int op = static_cast<int>(c & kOpMask);
  int hit = 0;
  if (c & kHitFlag) {
    hit = static_cast<int>(__ldcg(v.hit + h));
    v.hit[h] = 0u;
  }
  const int miss = op > hit ? op - hit : 0;
  float l = fadd(s0, v.l_unknown);
  l = (v.fp & kFpMissFma) ? ffma(v.l_miss, static_cast<float>(miss), l)
                          : fadd(l, fmul(v.l_miss, static_cast<float>(miss)));
  l = (v.fp & kFpHitFma) ? ffma(v.l_hit, static_cast<float>(hit), l)
                         : fadd(l, fmul(v.l_hit, static_cast<float>(hit)));
  if (l < v.l_min) l = v.l_min;
  if (l > v.l_max) l = v.l_max;
  return fsub(l, v.l_unknown);
}

__device__ __forceinline__ bool any_set(const uint4 &c) { return (c.x | c.y | c.z | c.w) != 0u; }

// Sweep of 16-byte counter groups first, first + stride, ... (< end): the U
// counter loads of a round are issued together, then each group with a set
// counter loads its stored values, folds and writes them back with its
// counters zeroed.  kL2: counters are loaded at L2 (ld.global.cg), as a
// launch that also wrote them from other CTAs needs.  Returns the voxels
// folded.
template <int U, bool kL2>
__device__ __forceinline__ uint32_t fold_groups(const FoldView &v, int first, int end,
                                                int stride) {
  const uint4 *c4r = reinterpret_cast<const uint4 *>(v.cnt);
  uint4 *c4 = reinterpret_cast<uint4 *>(v.cnt);
  float4 *o4 = reinterpret_cast<float4 *>(v.occ);
  uint32_t touched = 0;
  for (int i0 = first; i0 < end; i0 += U * stride) {
    uint4 c[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * stride;
      c[u] = i < end ? (kL2 ? __ldcg(c4r + i) : c4r[i]) : make_uint4(0u, 0u, 0u, 0u);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (!any_set(c[u])) continue;
      const int i = i0 + u * stride;
      const int h = i << 2;
      float4 o = o4[i];
      if (c[u].x) { o.x = fold_counter(v, h + 0, c[u].x, o.x); ++touched; }
      if (c[u].y) { o.y = fold_counter(v, h + 1, c[u].y, o.y); ++touched; }
      if (c[u].z) { o.z = fold_counter(v, h + 2, c[u].z, o.z); ++touched; }
      if (c[u].w) { o.w = fold_counter(v, h + 3, c[u].w, o.w); ++touched; }
      o4[i] = o;
      c4[i] = make_uint4(0u, 0u, 0u, 0u);
    }
  }
  return touched;
}

// Fold of the flagged lines among lines [first, end) by one warp.  The warp
// looks at 32 line flags at a time (lines base + lane; kAll: every line
// counts as flagged); each flagged line's counters and stored values are
// read whole (one 128-byte access per array, kLines lines in flight),
// folded where a counter is set, written back whole (a full line, so no
// partial-sector write) with the counters zeroed, and its flag cleared.
// `stride` is the distance between the warp's successive groups of 32
// lines.  kL2: flags and counters are read at L2 (ld.global.cg), as a launch
// that also wrote them from other CTAs needs.  Returns the voxels folded.
template <int kLines, bool kL2, bool kAll = false>
__device__ __forceinline__ uint32_t fold_lines(const FoldView &v, uint8_t *dirty, int first,
                                               int end, int stride) {
  const int lane = threadIdx.x & 31;
  uint32_t touched = 0;
  auto flag = [&](int l) -> bool {
    return l < end && (kAll || (kL2 ? __ldcg(dirty + l) : dirty[l]) != 0);
  };
  bool next = flag(first + lane);  // the group's flags are read a group ahead
  for (int base = first; base < end; base += stride) {
    const int l = base + lane;
    const bool d = next;
    uint32_t mask = __ballot_sync(0xffffffffu, d);
    if (d) dirty[l] = 0;
    next = flag(base + stride + lane);
    while (mask) {
      int at[kLines];
#pragma unroll
      for (int k = 0; k < kLines; ++k) {
        at[k] = -1;
        if (mask) {
          at[k] = ((base + __ffs(mask) - 1) << kLineShift) + lane;
          mask &= mask - 1;
        }
      }
      uint32_t c[kLines];
      float o[kLines];
#pragma unroll
      for (int k = 0; k < kLines; ++k)
        if (at[k] >= 0) c[k] = kL2 ? __ldcg(v.cnt + at[k]) : v.cnt[at[k]];
#pragma unroll
      for (int k = 0; k < kLines; ++k)
        if (at[k] >= 0) o[k] = v.occ[at[k]];
#pragma unroll
      for (int k = 0; k < kLines; ++k) {
        if (at[k] < 0) continue;
        if (c[k]) {
          o[k] = fold_counter(v, at[k], c[k], o[k]);
          ++touched;
        }
        v.occ[at[k]] = o[k];
        v.cnt[at[k]] = 0u;
      }
    }
  }
  return touched;
}

// ---- flagged lines gathered into shared memory by asynchronous copies ----
// The register fold above keeps at most kLines lines in flight per warp, and
// the fold is bound by how many scattered 128-byte lines are in flight.
// Here each warp stages up to 32 flagged lines at a time in shared memory
// with cp.async (16 bytes a lane, the data never passes through registers):
// a stage of 32 lines x (counters, values) is 16 instructions for the warp,
// and the next stage's copies are in flight while the warp folds the
// current one out of shared memory.  (One cp.async.bulk per 128-byte line,
// tried first, ran at half the speed: the copy engine's per-copy cost
// dominates at this size.)

__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(
                   __cvta_generic_to_shared(smem_dst))),
               "l"(gmem_src)
               : "memory");
}

// Shared memory of one warp: two stages of 32 lines x (counters, values).
struct LineStage {
  uint32_t cnt[32][32];
  float occ[32][32];
};
constexpr size_t kStageWarpSmem = 2 * sizeof(LineStage);

// A warp's position in its line range: the next flag group to read and the
// flagged lines of the current group not taken yet.
struct LineCursor {
  int base;       // first line of the current group of 32
  uint32_t pend;  // bit j: line base + j is flagged and not taken yet
  bool read;      // pend holds the current group's flags
};

// Up to 32 flagged lines from [cursor, end): lane j of the warp gets the
// j-th line (or -1), flags are cleared as their groups are read.  Returns
// how many lines were taken.
__device__ __forceinline__ int collect_lines(uint8_t *dirty, int end, LineCursor &c,
                                             int &my_line) {
  const int lane = threadIdx.x & 31;
  int n = 0;
  my_line = -1;
  while (n < 32) {
    if (!c.read) {
      if (c.base >= end) break;
      const int l = c.base + lane;
      const bool d = l < end && dirty[l] != 0;
      c.pend = __ballot_sync(0xffffffffu, d);
      if (d) dirty[l] = 0;
      c.read = true;
    }
    if (c.pend) {
      const int take = min(__popc(c.pend), 32 - n);
      const int r = lane - n;
      if (r >= 0 && r < take) my_line = c.base + static_cast<int>(__fns(c.pend, 0, r + 1));
      const int last = static_cast<int>(__fns(c.pend, 0, take));  // bit of the take-th line
      c.pend &= ~((2u << last) - 1u);
      n += take;
    }
    if (!c.pend) {
      c.base += 32;
      c.read = false;
    }
  }
  return n;
}

// Copies of the n lines held by the lanes (my_line, slots 0..n-1) into
// stage `st`, as one commit group: 256 16-byte chunks per array, chunk
// k * 32 + lane being part (lane & 7) of slot 4 k + (lane >> 3).
__device__ __forceinline__ void stage_issue(const FoldView &v, int n, int my_line,
                                            LineStage *st) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int slot = 4 * k + (lane >> 3), part = lane & 7;
    const int line = __shfl_sync(0xffffffffu, my_line, slot);
    if (slot < n) {
      const size_t at = (static_cast<size_t>(line) << kLineShift) + 4 * part;
      cp_async16(&st->cnt[slot][4 * part], v.cnt + at);
      cp_async16(&st->occ[slot][4 * part], v.occ + at);
    }
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}

// The flagged lines of [first, end) by one warp with its two stages `st`.
// Returns the voxels folded.
__device__ __forceinline__ uint32_t fold_lines_staged(const FoldView &v, uint8_t *dirty,
                                                      int first, int end, LineStage *st) {
  const int lane = threadIdx.x & 31;
  uint32_t touched = 0;
  LineCursor c{first, 0u, false};
  int cur = 0, line = -1;
  int n = collect_lines(dirty, end, c, line);
  if (n) stage_issue(v, n, line, &st[cur]);
  while (n) {
    int nline = -1;
    const int nn = collect_lines(dirty, end, c, nline);
    if (nn) {
      stage_issue(v, nn, nline, &st[cur ^ 1]);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncwarp();
    for (int j = 0; j < n; ++j) {
      const int at = (__shfl_sync(0xffffffffu, line, j) << kLineShift) + lane;
      const uint32_t cv = st[cur].cnt[j][lane];
      float o = st[cur].occ[j][lane];
      if (cv) {
        o = fold_counter(v, at, cv, o);
        ++touched;
      }
      v.occ[at] = o;
      v.cnt[at] = 0u;
    }
    __syncwarp();
    cur ^= 1;
    n = nn;
    line = nline;
  }
  return touched;
}

// The vnum % 4 voxels after the last whole group, one per thread 0..2.
__device__ __forceinline__ uint32_t fold_tail(const FoldView &v) {
  if (threadIdx.x >= static_cast<unsigned>(v.vnum & 3)) return 0;
  const int h = ((v.vnum >> 2) << 2) + threadIdx.x;
  const uint32_t c = __ldcg(v.cnt + h);
  if (!c) return 0;
  v.occ[h] = fold_counter(v, h, c, v.occ[h]);
  v.cnt[h] = 0u;
  return 1;
}

}  // namespace cublox_b200

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
  for (int base = first; base < end; base += stride) {
    const int l = base + lane;
    const bool d = l < end && (kAll || (kL2 ? __ldcg(dirty + l) : dirty[l]) != 0);
    uint32_t mask = __ballot_sync(0xffffffffu, d);
    if (d) dirty[l] = 0;
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

// ---- flagged lines gathered by the bulk-copy engine -------------------------
// The register fold above keeps at most kLines lines in flight per warp, and
// the fold is bound by how many scattered 128-byte lines are in flight.
// Here each warp stages its flagged lines in shared memory with
// cp.async.bulk (the copy engine needs no registers): for a group of 32
// line flags, the lanes of flagged lines each issue two 128-byte copies
// (counters, stored values) completing on the stage's mbarrier, while the
// warp folds the previous group out of the other stage.  Waits are bounded:
// one that gives up flags kErrWaitTimeout and the warp stops folding (after
// a bounded wait for its own copies).

constexpr int kBulkWaitSpin = 1 << 22;  // try_wait polls before a wait gives up

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_copy(void *dst, const void *src, uint32_t bytes,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  for (int i = 0; i < kBulkWaitSpin; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Shared memory of one warp: two stages of 32 lines x (counters, values).
struct BulkStage {
  uint32_t cnt[32][32];
  float occ[32][32];
};
constexpr size_t kBulkWarpSmem = 2 * sizeof(BulkStage) + 2 * sizeof(uint64_t);

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

// Copies of the n lines held by the lanes (my_line) into stage `st`: lane 0
// arms the barrier with their bytes, then each lane with a line copies its
// counters and values into its own slot.
__device__ __forceinline__ void bulk_issue(const FoldView &v, int n, int my_line, BulkStage *st,
                                           uint64_t *bar) {
  const int lane = threadIdx.x & 31;
  if (lane == 0) mbar_expect(bar, 256u * static_cast<uint32_t>(n));
  __syncwarp();
  if (my_line >= 0) {
    const size_t at = static_cast<size_t>(my_line) << kLineShift;
    bulk_copy(st->cnt[lane], v.cnt + at, 128u, bar);
    bulk_copy(st->occ[lane], v.occ + at, 128u, bar);
  }
}

// The flagged lines of [first, end) by one warp with its two stages `st`
// and barriers `bar` (initialised; `phase` their parities, kept across
// calls).  Stages hold up to 32 lines each, collected across flag groups,
// so a warp keeps up to 64 lines (16 KB) in flight whatever the density.
// Returns the voxels folded; *ok = false if a wait gave up.
__device__ __forceinline__ uint32_t fold_lines_bulk(const FoldView &v, uint8_t *dirty, int first,
                                                    int end, BulkStage *st, uint64_t *bar,
                                                    uint32_t &phase, bool *ok) {
  const int lane = threadIdx.x & 31;
  uint32_t touched = 0;
  LineCursor c{first, 0u, false};
  int cur = 0, line = -1;
  int n = collect_lines(dirty, end, c, line);
  if (n) bulk_issue(v, n, line, &st[cur], &bar[cur]);
  while (n) {
    int nline = -1;
    const int nn = collect_lines(dirty, end, c, nline);
    if (nn) {
      // the other stage was last read by this warp's generic loads
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      bulk_issue(v, nn, nline, &st[cur ^ 1], &bar[cur ^ 1]);
    }
    if (!mbar_wait(&bar[cur], (phase >> cur) & 1u)) {
      *ok = false;
      // bounded waits for this warp's copies still in flight, then stop
      mbar_wait(&bar[cur], (phase >> cur) & 1u);
      if (nn) mbar_wait(&bar[cur ^ 1], (phase >> (cur ^ 1)) & 1u);
      return touched;
    }
    phase ^= 1u << cur;
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

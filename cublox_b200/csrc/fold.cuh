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
// says), clamped, shifted back (kernels.cu:179-200).  fold_counter reads the
// hit count of a flagged voxel at L2 (ld.global.cg): in a fused launch other
// CTAs of the same kernel wrote it.
__device__ __forceinline__ float fold_value(const FoldView &v, int op, int hit, float s0) {
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

__device__ __forceinline__ float fold_counter(const FoldView &v, int h, uint32_t c, float s0) {
  int hit = 0;
  if (c & kHitFlag) {
    hit = static_cast<int>(__ldcg(v.hit + h));
    v.hit[h] = 0u;
  }
  return fold_value(v, static_cast<int>(c & kOpMask), hit, s0);
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

// ---- flagged lines compacted into a list per CTA ----
// The per-warp fold above reads 32 flags, then folds only the flagged ones
// among them: about 9 of 32 lines at README scale, so a warp rarely has more
// than one batch of lines in flight and waits a full memory latency on every
// flag group.  Here a CTA (256 threads or more) takes up to 4096 lines at a
// time: one 16-byte flag load for each of its first 256 threads, a CTA-wide
// prefix sum turns the flagged lines into a
// dense list in shared memory (flags cleared on the way), and the warps then
// fold the list four lines per warp access (8 lanes x 16 bytes a line) with
// kQuads accesses in flight per warp, so every warp has 4 kQuads lines in
// flight until the list runs out.  The next item's flags are loaded before
// the current list is folded.

constexpr int kListThreads = 256;              // CTA size of the fold-only kernels
constexpr int kListLines = 16 * kListThreads;  // lines per item: 16 flags per thread

struct LineList {
  uint16_t line[kListLines];  // flagged lines, relative to the item's first line
  int warp_sum[32];
};

// The raw flags of this thread's lines start + 16 t .. + 15 (bytes of lines
// at or beyond `count` read as zero); `dirty + start` is 16-byte aligned.
// The value is used only by line_flag_bits, so the load can stay in flight
// across other work.  kL2: read at L2 (ld.global.cg), as flags that other
// CTAs of the same launch wrote need.
template <bool kL2 = false>
__device__ __forceinline__ uint4 load_line_flags(const uint8_t *dirty, int start, int count) {
  const int i = 16 * static_cast<int>(threadIdx.x);
  if (i + 16 <= count) {
    const uint4 *q = reinterpret_cast<const uint4 *>(dirty + start + i);
    return kL2 ? __ldcg(q) : *q;
  }
  uint32_t w[4] = {0u, 0u, 0u, 0u};
  for (int j = 0; i + j < count && j < 16; ++j) {
    const uint8_t d = kL2 ? __ldcg(dirty + start + i + j) : dirty[start + i + j];
    w[j >> 2] |= static_cast<uint32_t>(d != 0) << (8 * (j & 3));
  }
  return make_uint4(w[0], w[1], w[2], w[3]);
}

// One bit per non-zero flag byte: bit j for byte j of the 16.
__device__ __forceinline__ uint32_t line_flag_bits(const uint4 &f) {
  const uint32_t w[4] = {f.x, f.y, f.z, f.w};
  uint32_t m = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint32_t nz = __vcmpne4(w[k], 0u) & 0x01010101u;  // bits 0, 8, 16, 24
    m |= ((nz | (nz >> 7) | (nz >> 14) | (nz >> 21)) & 0xfu) << (4 * k);
  }
  return m;
}

// The CTA's list from every thread's flag bits `m` (item of `count` lines
// from line `start`); clears the flags it found.  Returns the list's
// length.  Contains two CTA barriers, the last at the end.
__device__ __forceinline__ int build_line_list(uint32_t m, LineList &L, uint8_t *dirty, int start,
                                               int count) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = __popc(m);
  int incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) L.warp_sum[warp] = incl;
  __syncthreads();
  int pos = incl - c, total = 0;
  const int warps = blockDim.x >> 5;
  for (int w = 0; w < warps; ++w) {
    const int s = L.warp_sum[w];
    pos += w < warp ? s : 0;
    total += s;
  }
  const int i = 16 * static_cast<int>(threadIdx.x);
  for (uint32_t r = m; r; r &= r - 1) L.line[pos++] = static_cast<uint16_t>(i + __ffs(r) - 1);
  if (m) {
    if (i + 16 <= count)  // the thread's 16 flags are one aligned 16-byte word
      *reinterpret_cast<uint4 *>(dirty + start + i) = make_uint4(0u, 0u, 0u, 0u);
    else
      for (uint32_t r = m; r; r &= r - 1) dirty[start + i + __ffs(r) - 1] = 0;
  }
  __syncthreads();
  return total;
}

// Voxels with a hit whose fold waits for the end of the item.  Their hit
// count lives in a second array; loaded where the voxel is met, it would
// stall the warp's whole batch of lines for one more memory round trip
// (most batches hold a hit voxel), so they are queued in shared memory
// and folded together once the list is done, every hit load in flight at
// once.  A full queue folds further hits where they are met.
constexpr int kHitCap = 1024;

struct HitQueue {
  int n;                 // voxels queued (may pass kHitCap: the rest were folded in place)
  int h[kHitCap];        // address
  uint32_t c[kHitCap];   // counter word
};

// Folds voxel h (counter word c, stored value o) now, or queues it if it has
// a hit and the queue has room (its stored value is then written back
// unchanged by the caller and replaced by fold_hit_queue).
__device__ __forceinline__ float fold_or_queue(const FoldView &v, HitQueue *hq, int h, uint32_t c,
                                               float o) {
  if (hq && (c & kHitFlag)) {
    const int slot = atomicAdd(&hq->n, 1);
    if (slot < kHitCap) {
      hq->h[slot] = h;
      hq->c[slot] = c;
      return o;
    }
  }
  return fold_counter(v, h, c, o);
}

// Fold of the CTA's list of n lines (relative to line `start`).  Warp w of
// W takes line quads w, w + W, ...; lane (q, s) = (lane / 8, lane % 8)
// handles 16-byte piece s of the quad's line q.  A piece whose counters are
// all zero is left as it is (its values do not change, its counters are
// zero already).  Hit voxels go to `hq` when it is given (fold_hit_queue
// folds them after a CTA barrier).  kL2: counters are read at L2.  Returns
// the voxels folded or queued.
template <int kQuads, bool kL2>
__device__ __forceinline__ uint32_t fold_line_list(const FoldView &v, const uint16_t *list, int n,
                                                   int start, HitQueue *hq = nullptr) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  const int q = lane >> 3, sub = lane & 7;
  const uint4 *c4r = reinterpret_cast<const uint4 *>(v.cnt);
  uint4 *c4 = reinterpret_cast<uint4 *>(v.cnt);
  float4 *o4 = reinterpret_cast<float4 *>(v.occ);
  uint32_t touched = 0;
  const int quads = (n + 3) >> 2;
  for (int i0 = warp; i0 < quads; i0 += kQuads * warps) {
    int at[kQuads];
#pragma unroll
    for (int u = 0; u < kQuads; ++u) {
      const int k = 4 * (i0 + u * warps) + q;
      at[u] = k < n ? ((start + list[k]) << 3) + sub : -1;  // index of the 16-byte piece
    }
    uint4 c[kQuads];
    float4 o[kQuads];
#pragma unroll
    for (int u = 0; u < kQuads; ++u)
      if (at[u] >= 0) c[u] = kL2 ? __ldcg(c4r + at[u]) : c4r[at[u]];
#pragma unroll
    for (int u = 0; u < kQuads; ++u)
      if (at[u] >= 0) o[u] = o4[at[u]];
#pragma unroll
    for (int u = 0; u < kQuads; ++u) {
      if (at[u] < 0 || !any_set(c[u])) continue;
      const int h = at[u] << 2;
      const uint32_t cc[4] = {c[u].x, c[u].y, c[u].z, c[u].w};
      float oo[4] = {o[u].x, o[u].y, o[u].z, o[u].w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        touched += cc[e] != 0u;
        if (cc[e] & kHitFlag) {  // rare: queued, or folded here with its hit count
          oo[e] = fold_or_queue(v, hq, h + e, cc[e], oo[e]);
        } else {
          // no hit: the same arithmetic for every lane, kept where counted
          const float f = fold_value(v, static_cast<int>(cc[e]), 0, oo[e]);
          oo[e] = cc[e] ? f : oo[e];
        }
      }
      o4[at[u]] = make_float4(oo[0], oo[1], oo[2], oo[3]);
      c4[at[u]] = make_uint4(0u, 0u, 0u, 0u);
    }
  }
  return touched;
}

// Folds the queued hit voxels (after a CTA barrier that follows every
// fold_line_list of the item) and empties the queue; ends with a CTA
// barrier.  The stored value is read back: the list fold wrote it unchanged.
__device__ __forceinline__ void fold_hit_queue(const FoldView &v, HitQueue &hq) {
  const int n = min(hq.n, kHitCap);
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    const int h = hq.h[e];
    v.occ[h] = fold_counter(v, h, hq.c[e], v.occ[h]);
  }
  __syncthreads();
  if (threadIdx.x == 0) hq.n = 0;
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

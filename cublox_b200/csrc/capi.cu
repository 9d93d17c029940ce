// C ABI of cublox_b200 (include/cublox_b200.h): host orchestration of one
// occupancy map on one B200.  Host arithmetic that the reference performs on
// the CPU (window geometry, fetch bounds, recenter gate) is restated here with
// plain float ops; this file is compiled with -ffp-contract=off so that the
// host compiler fuses nothing either.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "../../include/cublox_b200.h"
#include "exact_fp.cuh"
#include "grid_internal.hpp"
#include "kernels.cuh"

using namespace cublox_b200;

namespace {
thread_local std::string g_err;
std::atomic<int64_t> g_counters[cublox_b200::detail::kNumCounters];
}  // namespace

namespace cublox_b200 {
namespace detail {
void count(Counter c) { g_counters[c].fetch_add(1, std::memory_order_relaxed); }

// Test hook (cublox_test_fail_allocations): after g_fail_skip more
// allocations, the next g_fail_count fail without a CUDA call.
std::atomic<int64_t> g_fail_skip{0}, g_fail_count{0};

bool injected_failure() {
  if (g_fail_count.load(std::memory_order_relaxed) <= 0) return false;
  if (g_fail_skip.fetch_sub(1, std::memory_order_relaxed) > 0) return false;
  return g_fail_count.fetch_sub(1, std::memory_order_relaxed) > 0;
}

cudaError_t dev_alloc(void **p, size_t bytes) {
  if (injected_failure()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  count(kDevAllocs);
  return cudaMalloc(p, bytes);
}

cudaError_t dev_free(void *p) {
  if (!p) return cudaSuccess;
  count(kDevFrees);
  return cudaFree(p);
}

cudaError_t pinned_alloc(void **p, size_t bytes) {
  if (injected_failure()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  count(kPinnedAllocs);
  return cudaMallocHost(p, bytes);
}

cudaError_t pinned_free(void *p) {
  if (!p) return cudaSuccess;
  count(kPinnedFrees);
  return cudaFreeHost(p);
}

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char *what, int line) {
  g_err = std::string("cublox_b200: ") + what + ": " + cudaGetErrorString(e) +
          " (line " + std::to_string(line) + ")";
  return CUBLOX_ERR_CUDA;
}
}  // namespace detail
}  // namespace cublox_b200

using cublox_b200::detail::cuda_fail;
using cublox_b200::detail::fail;

namespace {

#define CK(call)                                                     \
  do {                                                               \
    cudaError_t e_ = (call);                                         \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call, __LINE__);    \
  } while (0)

#define CK_LAUNCH()                                                  \
  do {                                                               \
    cudaError_t e_ = cudaGetLastError();                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, "launch", __LINE__); \
  } while (0)

// Host-side posToGlobalIndex as the reference's x86-64 build computes it
// (utils.hpp:24-31): no FMA, cvttss2si (NaN/out of range -> INT_MIN).
int f2i_x86(float v) {
  if (v >= -2147483648.0f && v < 2147483648.0f) return static_cast<int>(v);
  return std::numeric_limits<int>::min();
}
int d2i_x86(double v) {
  if (v > -2147483649.0 && v < 2147483648.0) return static_cast<int>(v);
  return std::numeric_limits<int>::min();
}
int host_p2g(float p, float inv, bool ctr) {
  if (ctr) {
    const float s = p < 0.0f ? -1.0f : 1.0f;
    const float m = p * inv;
    return f2i_x86(m + s * 0.5f);
  }
  return f2i_x86(std::floor(p * inv));
}
float g2p(int g, float res, bool ctr) {
  return ctr ? static_cast<float>(g) * res
             : (static_cast<float>(g) + 0.5f) * res;
}

// 0: pageable host memory, 1: pinned host memory, 2: device-accessible.
int mem_kind(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) return 2;
  if (a.type == cudaMemoryTypeHost) return 1;
  return 0;
}

}  // namespace


extern "C" {

const char *cublox_last_error(void) { return g_err.c_str(); }
const char *cublox_version(void) { return "cublox_b200 0.2 (sm_100a)"; }

int cublox_test_fail_allocations(int64_t skip, int64_t count) {
  if (skip < 0 || count < 0) return fail(CUBLOX_ERR_INVALID, "test_fail_allocations: negative");
  cublox_b200::detail::g_fail_count.store(0);
  cublox_b200::detail::g_fail_skip.store(skip);
  cublox_b200::detail::g_fail_count.store(count);
  return CUBLOX_OK;
}

int cublox_runtime_counters(int64_t *out, int n) {
  if (!out || n < 0) return fail(CUBLOX_ERR_INVALID, "runtime_counters: bad argument");
  for (int i = 0; i < n; ++i)
    out[i] = i < cublox_b200::detail::kNumCounters ? g_counters[i].load() : 0;
  return CUBLOX_OK;
}

int cublox_binary_version(int *binary_version) {
  if (!binary_version) return fail(CUBLOX_ERR_INVALID, "binary_version: null argument");
  *binary_version = kernel_binary_version();
  if (*binary_version < 0) return fail(CUBLOX_ERR_CUDA, "binary_version: no kernel image for this device");
  return CUBLOX_OK;
}

static void free_all(cublox_grid *g) {
  cublox_b200::detail::dfree(g->d_dirty);
  cublox_b200::detail::dfree(g->d_occ);
  cublox_b200::detail::dfree(g->d_cnt);
  cublox_b200::detail::dfree(g->d_hit);
  cublox_b200::detail::dfree(g->d_stats);
  cublox_b200::detail::dfree(g->d_err);
  cublox_b200::detail::dfree(g->d_masks);
  if (g->h_masks) cublox_b200::detail::hfree(g->h_masks);
  for (cudaEvent_t e : g->mask_ev)
    if (e) cudaEventDestroy(e);
  cublox_b200::detail::dfree(g->d_cloud);
  cublox_b200::detail::dfree(g->d_world);
  cublox_b200::detail::dfree(g->d_kept);
  cublox_b200::detail::dfree(g->d_image);
  cublox_b200::detail::dfree(g->d_bins);
  cublox_b200::detail::dfree(g->d_work);
  cublox_b200::detail::dfree(g->d_segs);
  cublox_b200::detail::dfree(g->d_rays);
  cublox_b200::detail::dfree(g->d_hist);
  cublox_b200::detail::dfree(g->d_sorted);
  cublox_b200::detail::free_fetch(&g->fs);
  cublox_b200::detail::dfree(g->d_qout);
  cublox_b200::detail::dfree(g->d_qin);
  for (int i = 0; i < 2; ++i) {
    if (g->h_stage[i]) cublox_b200::detail::hfree(g->h_stage[i]);
    if (g->stage_ev[i]) cudaEventDestroy(g->stage_ev[i]);
  }
  for (int i = 0; i < 6; ++i)
    if (g->tev[i]) cudaEventDestroy(g->tev[i]);
  if (g->own_stream && g->stream) cudaStreamDestroy(g->stream);
}

// Per-stage device timing (raycast, fold, recenter clear), opt-in.
static void tmark(cublox_grid *g, int stage, int end) {
  if (!g->timing_on) return;
  cudaEventRecord(g->tev[2 * stage + end], g->stream);
  if (end) g->tev_used[stage] = true;
}

static void set_origin(cublox_grid *g, const int o[3]) {
  for (int a = 0; a < 3; ++a) {
    g->origin_i[a] = o[a];
    g->origin_f[a] = g2p(o[a], g->res, g->ctr);
  }
}

}  // extern "C"

// Layout of a map's arrays for a layout code (log2 brick sides as digits
// x y z; 0: the reference's hash order).  Returns the voxels each array
// needs (padding included, a multiple of 32) and sets the bricks per axis.
static int64_t make_layout(const int map[3], int code, VoxLayout *L, int nbr[3]) {
  if (code == 0) {
    for (int a = 0; a < 3; ++a) {
      L->lb[a] = 0;
      nbr[a] = map[a];
    }
    L->bs[0] = map[1] * map[2];
    L->bs[1] = map[2];
    L->bs[2] = 1;
    for (int a = 0; a < 3; ++a) L->is[a] = L->bs[a];
    const int64_t v = static_cast<int64_t>(map[0]) * map[1] * map[2];
    return (v + 31) & ~int64_t(31);
  }
  const int lb[3] = {code / 100, (code / 10) % 10, code % 10};
  for (int a = 0; a < 3; ++a) {
    L->lb[a] = lb[a];
    nbr[a] = (map[a] + (1 << lb[a]) - 1) >> lb[a];
  }
  const int vb = 1 << (lb[0] + lb[1] + lb[2]);
  const int64_t n = static_cast<int64_t>(nbr[0]) * nbr[1] * nbr[2] * vb;
  if (n > (int64_t(1) << 31)) return n;  // the caller refuses it
  L->bs[0] = nbr[1] * nbr[2] * vb;
  L->bs[1] = nbr[2] * vb;
  L->bs[2] = vb;
  L->is[0] = 1 << (lb[1] + lb[2]);
  L->is[1] = 1 << lb[2];
  L->is[2] = 1;
  return n;
}

int64_t cublox_b200::detail::nalloc_for(const int half[3]) {
  int map[3];
  for (int a = 0; a < 3; ++a) map[a] = 2 * half[a] + 1;
  int64_t nalloc = 0;
  for (int code : kLayouts) {
    VoxLayout l{};
    int nb[3];
    const int64_t n = make_layout(map, code, &l, nb);
    if (n <= (int64_t(1) << 31)) nalloc = std::max(nalloc, n);
  }
  return nalloc;
}

size_t cublox_b200::detail::voxel_bytes_for(const int half[3]) {
  const int64_t nalloc = nalloc_for(half);
  return 12 * static_cast<size_t>(nalloc) + static_cast<size_t>(nalloc >> kLineShift);
}

bool cublox_b200::detail::layout_valid(int code) {
  if (code == 0) return true;
  if (code < 0 || code > 999) return false;
  const int d[3] = {code / 100, (code / 10) % 10, code % 10};
  return d[0] + d[1] + d[2] == kLineShift;  // one brick = one 32-voxel line
}

// The address of the voxel with reference hash h.
static int hash_addr(const cublox_grid *g, int h) {
  const int nyz = g->map[1] * g->map[2];
  const int sx = h / nyz, r = h - sx * nyz;
  const int sy = r / g->map[2], sz = r - sy * g->map[2];
  return vox_addr(g->lay, sx, sy, sz);
}

void cublox_b200::detail::layout_to_reference(const cublox_grid *g, const float *arr,
                                              float *ref) {
  size_t h = 0;
  for (int sx = 0; sx < g->map[0]; ++sx) {
    const int ox = vox_axis(g->lay, 0, sx);
    for (int sy = 0; sy < g->map[1]; ++sy) {
      const int oxy = ox + vox_axis(g->lay, 1, sy);
      for (int sz = 0; sz < g->map[2]; ++sz) ref[h++] = arr[oxy + vox_axis(g->lay, 2, sz)];
    }
  }
}

int cublox_b200::detail::set_layout(cublox_grid *g, int code) {
  if (!layout_valid(code)) return fail(CUBLOX_ERR_INVALID, "layout: bricks must hold 32 voxels");
  if (code == g->lay_code) return CUBLOX_OK;
  VoxLayout nl{};
  int nbr[3];
  const int64_t n = make_layout(g->map, code, &nl, nbr);
  if (n > g->nalloc)
    return fail(CUBLOX_ERR_INVALID, "layout: needs more voxels than the grid holds");
  if (!g->d_occ) return fail(CUBLOX_ERR_INVALID, "layout: the grid's buffers are released");
  // occ -> the reference order in hit (zero between scans) -> occ
  float *tmp = reinterpret_cast<float *>(g->d_hit);
  launch_relayout(g->d_occ, tmp, g->lay, g->map, 1, g->stream);
  CK_LAUNCH();
  CK(cudaMemsetAsync(g->d_occ, 0, sizeof(float) * static_cast<size_t>(g->nalloc), g->stream));
  launch_relayout(tmp, g->d_occ, nl, g->map, 0, g->stream);
  CK_LAUNCH();
  CK(cudaMemsetAsync(g->d_hit, 0, sizeof(uint32_t) * static_cast<size_t>(g->nalloc), g->stream));
  g->lay = nl;
  g->lay_code = code;
  for (int a = 0; a < 3; ++a) g->nbr[a] = nbr[a];
  return CUBLOX_OK;
}

extern "C" {

int cublox_grid_create(const int half_map_size[3], float resolution,
                       int origin_at_center, int has_recenter_threshold,
                       double recenter_threshold, const float origin[3],
                       void *stream, cublox_grid **out) {
  if (!half_map_size || !origin || !out)
    return fail(CUBLOX_ERR_INVALID, "cublox_grid_create: null argument");
  *out = nullptr;
  if (!(resolution > 0.0f) || !std::isfinite(resolution))
    return fail(CUBLOX_ERR_INVALID, "cublox_grid_create: resolution must be > 0");
  int64_t total = 1;
  for (int a = 0; a < 3; ++a) {
    if (half_map_size[a] < 0)
      return fail(CUBLOX_ERR_INVALID, "cublox_grid_create: negative half size");
    total *= 2 * static_cast<int64_t>(half_map_size[a]) + 1;
  }
  if (total > std::numeric_limits<int>::max())
    return fail(CUBLOX_ERR_RANGE,
                "cublox_grid_create: requested voxel_num = " +
                    std::to_string(total) + " exceeds int32 max (" +
                    std::to_string(std::numeric_limits<int>::max()) +
                    "). Pick a smaller half_map_size_i.");
  cublox_grid *g = new cublox_grid();
  g->res = resolution;
  g->res_inv = 1.0f / resolution;
  for (int a = 0; a < 3; ++a) {
    g->half[a] = half_map_size[a];
    g->map[a] = 2 * half_map_size[a] + 1;
  }
  g->voxel_num = static_cast<int>(total);
  // arrays sized for every layout the grid may switch to (that fits int32
  // addresses); the default layout unless it alone does not fit
  g->nalloc = 0;
  for (int code : cublox_b200::detail::kLayouts) {
    VoxLayout l{};
    int nb[3];
    const int64_t n = make_layout(g->map, code, &l, nb);
    if (n <= (int64_t(1) << 31)) g->nalloc = std::max(g->nalloc, n);
  }
  {
    int nb[3];
    int code = cublox_b200::detail::kDefaultLayout;
    if (make_layout(g->map, code, &g->lay, nb) > g->nalloc) code = 0;
    make_layout(g->map, code, &g->lay, nb);
    g->lay_code = code;
    for (int a = 0; a < 3; ++a) g->nbr[a] = nb[a];
  }
  g->nlines = static_cast<int>(g->nalloc >> kLineShift);
  g->has_thr = has_recenter_threshold != 0;
  if (g->has_thr) {
    const float t = static_cast<float>(recenter_threshold);
    g->thr_sq = t * t;
  }
  g->ctr = origin_at_center != 0;
  int o[3];
  for (int a = 0; a < 3; ++a) o[a] = host_p2g(origin[a], g->res_inv, g->ctr);
  set_origin(g, o);
  cudaGetDevice(&g->device);

  auto bail = [&](cudaError_t e, const char *what) {
    int rc = cuda_fail(e, what, __LINE__);
    if (e == cudaErrorMemoryAllocation) {
      rc = CUBLOX_ERR_NOMEM;
      g_err = std::string("cublox_grid_create: failed to allocate voxel buffers: ") +
              cudaGetErrorString(e);
    }
    cudaGetLastError();
    free_all(g);
    delete g;
    return rc;
  };
  cudaError_t e;
  if (stream) {
    g->stream = static_cast<cudaStream_t>(stream);
  } else {
    if ((e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking)) != cudaSuccess)
      return bail(e, "cudaStreamCreate");
    g->own_stream = true;
  }
  const size_t n = static_cast<size_t>(g->nalloc);
  if ((e = cublox_b200::detail::dmalloc(&g->d_dirty, static_cast<size_t>(g->nlines))) != cudaSuccess) return bail(e, "cudaMalloc line flags");
  if ((e = cudaMemsetAsync(g->d_dirty, 0, static_cast<size_t>(g->nlines), g->stream)) != cudaSuccess) return bail(e, "memset line flags");
  if ((e = cublox_b200::detail::dmalloc(&g->d_occ, n * sizeof(float))) != cudaSuccess) return bail(e, "cudaMalloc occ");
  if ((e = cublox_b200::detail::dmalloc(&g->d_cnt, n * sizeof(uint32_t))) != cudaSuccess) return bail(e, "cudaMalloc cnt");
  if ((e = cublox_b200::detail::dmalloc(&g->d_hit, n * sizeof(uint32_t))) != cudaSuccess) return bail(e, "cudaMalloc hit");
  if ((e = cublox_b200::detail::dmalloc(&g->d_stats, 4 * sizeof(unsigned long long))) != cudaSuccess) return bail(e, "cudaMalloc stats");
  if ((e = cublox_b200::detail::dmalloc(&g->d_err, sizeof(uint32_t))) != cudaSuccess) return bail(e, "cudaMalloc err");
  // recenter plan: slab masks, then (brick layouts) brick lists of up to
  // map[a] entries per axis
  int words = 0;
  for (int a = 0; a < 3; ++a) {
    g->mask_words[a] = (g->map[a] + 31) / 32;
    words += g->mask_words[a] + g->map[a];
  }
  if ((e = cublox_b200::detail::dmalloc(&g->d_masks, words * sizeof(uint32_t))) != cudaSuccess) return bail(e, "cudaMalloc masks");
  // pinned staging of the recenter masks, two halves used in turn
  g->mask_stage_words = words;
  if ((e = cublox_b200::detail::hmalloc(&g->h_masks, 2 * words * sizeof(uint32_t))) != cudaSuccess) return bail(e, "pinned masks");
  for (int i = 0; i < 2; ++i)
    if ((e = cudaEventCreateWithFlags(&g->mask_ev[i], cudaEventDisableTiming)) != cudaSuccess)
      return bail(e, "mask event");
  if ((e = cudaMemsetAsync(g->d_occ, 0, n * sizeof(float), g->stream)) != cudaSuccess) return bail(e, "memset occ");
  if ((e = cudaMemsetAsync(g->d_cnt, 0, n * sizeof(uint32_t), g->stream)) != cudaSuccess) return bail(e, "memset cnt");
  if ((e = cudaMemsetAsync(g->d_hit, 0, n * sizeof(uint32_t), g->stream)) != cudaSuccess) return bail(e, "memset hit");
  if ((e = cudaMemsetAsync(g->d_stats, 0, 4 * sizeof(unsigned long long), g->stream)) != cudaSuccess) return bail(e, "memset stats");
  if ((e = cudaMemsetAsync(g->d_err, 0, sizeof(uint32_t), g->stream)) != cudaSuccess) return bail(e, "memset err");
  if ((e = cudaStreamSynchronize(g->stream)) != cudaSuccess) return bail(e, "sync");
  *out = g;
  return CUBLOX_OK;
}

int cublox_grid_destroy(cublox_grid *g) {
  if (!g) return CUBLOX_OK;
  if (g->stream) cudaStreamSynchronize(g->stream);
  free_all(g);
  delete g;
  return CUBLOX_OK;
}

int cublox_grid_reset(cublox_grid *g) {
  if (!g) return fail(CUBLOX_ERR_INVALID, "null grid");
  const size_t n = static_cast<size_t>(g->nalloc);
  CK(cudaMemsetAsync(g->d_occ, 0, n * sizeof(float), g->stream));
  CK(cudaMemsetAsync(g->d_cnt, 0, n * sizeof(uint32_t), g->stream));
  CK(cudaMemsetAsync(g->d_hit, 0, n * sizeof(uint32_t), g->stream));
  CK(cudaMemsetAsync(g->d_dirty, 0, static_cast<size_t>(g->nlines), g->stream));
  CK(cudaStreamSynchronize(g->stream));
  g->first_run = true;
  return CUBLOX_OK;
}

int cublox_grid_reset_voxel(cublox_grid *g, int hash_id) {
  if (!g) return fail(CUBLOX_ERR_INVALID, "null grid");
  if (hash_id < 0 || hash_id >= g->voxel_num) return CUBLOX_OK;
  const int a = hash_addr(g, hash_id);
  CK(cudaMemsetAsync(g->d_occ + a, 0, sizeof(float), g->stream));
  CK(cudaMemsetAsync(g->d_cnt + a, 0, sizeof(uint32_t), g->stream));
  CK(cudaMemsetAsync(g->d_hit + a, 0, sizeof(uint32_t), g->stream));
  CK(cudaStreamSynchronize(g->stream));
  return CUBLOX_OK;
}

int cublox_grid_set_max_range(cublox_grid *g, float range) {
  if (!g) return fail(CUBLOX_ERR_INVALID, "null grid");
  g->max_range = range;
  return CUBLOX_OK;
}

int cublox_grid_get_max_range(const cublox_grid *g, float *range) {
  if (!g || !range) return fail(CUBLOX_ERR_INVALID, "null argument");
  *range = g->max_range;
  return CUBLOX_OK;
}

int cublox_grid_set_log_odds(cublox_grid *g, float l_hit, float l_miss,
                             float l_min, float l_max, float l_free,
                             float l_occupied) {
  if (!g) return fail(CUBLOX_ERR_INVALID, "null grid");
  g->l_hit = l_hit;
  g->l_miss = l_miss;
  g->l_min = l_min;
  g->l_max = l_max;
  g->l_free = l_free;
  g->l_occ = l_occupied;
  g->l_unknown = 0.0f;
  return CUBLOX_OK;
}

int cublox_grid_set_option(cublox_grid *g, int key, int value) {
  if (!g) return fail(CUBLOX_ERR_INVALID, "null grid");
  switch (key) {
    case CUBLOX_OPT_RAYCAST:
      if (value < 0 || value > 2) break;
      g->opt_raycast = value;
      return CUBLOX_OK;
    case CUBLOX_OPT_SEGMENT:
      if (value < 4 || value > 100000) break;
      g->opt_seg = value;
      return CUBLOX_OK;
    case CUBLOX_OPT_FOLD:
      if (value < 0 || value > 3) break;
      g->opt_fold = value;
      return CUBLOX_OK;
    case CUBLOX_OPT_LAYOUT:
      if (!cublox_b200::detail::layout_valid(value)) break;
      return cublox_b200::detail::set_layout(g, value);
    case CUBLOX_OPT_BLOCK:
      if (value != 256 && value != 512 && value != 1024) break;
      g->opt_block = value;
      return CUBLOX_OK;
    case CUBLOX_OPT_CONTIGUOUS:
      g->opt_contig = value != 0;
      return CUBLOX_OK;
    case CUBLOX_OPT_CUBE:
      if (value != 0 && value != 8 && value != 16 && value != 32) break;
      g->opt_cube = value;
      return CUBLOX_OK;
    case CUBLOX_OPT_FLAT_CUBE:
      g->opt_flat = value != 0;
      return CUBLOX_OK;
    case CUBLOX_OPT_MATCH:
      g->opt_match = value != 0;
      return CUBLOX_OK;
    case CUBLOX_OPT_SORT:
      g->opt_sort = value != 0;
      return CUBLOX_OK;
    default:
      break;
  }
  return fail(CUBLOX_ERR_INVALID, "set_option: unknown key or value");
}

int cublox_grid_get_option(const cublox_grid *g, int key, int *value) {
  if (!g || !value) return fail(CUBLOX_ERR_INVALID, "null argument");
  switch (key) {
    case CUBLOX_OPT_RAYCAST: *value = g->opt_raycast; return CUBLOX_OK;
    case CUBLOX_OPT_CUBE: *value = g->opt_cube; return CUBLOX_OK;
    case CUBLOX_OPT_FLAT_CUBE: *value = g->opt_flat; return CUBLOX_OK;
    case CUBLOX_OPT_MATCH: *value = g->opt_match; return CUBLOX_OK;
    case CUBLOX_OPT_SORT: *value = g->opt_sort; return CUBLOX_OK;
    case CUBLOX_OPT_SEGMENT: *value = g->opt_seg; return CUBLOX_OK;
    case CUBLOX_OPT_FOLD: *value = g->opt_fold; return CUBLOX_OK;
    case CUBLOX_OPT_BLOCK: *value = g->opt_block; return CUBLOX_OK;
    case CUBLOX_OPT_CONTIGUOUS: *value = g->opt_contig; return CUBLOX_OK;
    case CUBLOX_OPT_LAYOUT: *value = g->lay_code; return CUBLOX_OK;
    default: break;
  }
  return fail(CUBLOX_ERR_INVALID, "get_option: unknown key");
}

int cublox_grid_set_fp_mode(cublox_grid *g, unsigned mode) {
  if (!g) return fail(CUBLOX_ERR_INVALID, "null grid");
  g->fp = mode;
  return CUBLOX_OK;
}

int cublox_grid_get_fp_mode(const cublox_grid *g, unsigned *mode) {
  if (!g || !mode) return fail(CUBLOX_ERR_INVALID, "null argument");
  *mode = g->fp;
  return CUBLOX_OK;
}

static int ensure_cloud(cublox_grid *g, int n) {
  if (n <= g->cloud_cap) return CUBLOX_OK;
  CK(cudaStreamSynchronize(g->stream));
  cublox_b200::detail::dfree(g->d_cloud);
  g->d_cloud = nullptr;
  g->cloud_cap = 0;
  cudaError_t e = cublox_b200::detail::dmalloc(&g->d_cloud, sizeof(float) * 3 * static_cast<size_t>(n));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(CUBLOX_ERR_NOMEM, "cublox_grid_update: cloud buffer allocation failed");
  }
  g->cloud_cap = n;
  return CUBLOX_OK;
}

static int ensure_stage(cublox_grid *g, int n) {
  if (n <= g->stage_cap) return CUBLOX_OK;
  for (int i = 0; i < 2; ++i) {
    if (g->stage_ev[i]) CK(cudaEventSynchronize(g->stage_ev[i]));
    if (g->h_stage[i]) cublox_b200::detail::hfree(g->h_stage[i]);
    g->h_stage[i] = nullptr;
  }
  g->stage_cap = 0;
  for (int i = 0; i < 2; ++i) {
    cudaError_t e = cublox_b200::detail::hmalloc(&g->h_stage[i], sizeof(float) * 3 * static_cast<size_t>(n));
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(CUBLOX_ERR_NOMEM, "cublox_grid_update: pinned staging allocation failed");
    }
    if (!g->stage_ev[i]) CK(cudaEventCreateWithFlags(&g->stage_ev[i], cudaEventDisableTiming));
  }
  g->stage_cap = n;
  return CUBLOX_OK;
}

// Launch raycast (+ fold unless count_only) on a device SoA cloud.
static int integrate(cublox_grid *g, const float *dx, const float *dy,
                     const float *dz, int n, int stride,
                     const float sensor[3], bool count_only = false) {
  if (g->stats_on)
    CK(cudaMemsetAsync(g->d_stats, 0, 4 * sizeof(unsigned long long), g->stream));
  RayParams p{};
  p.x = dx;
  p.y = dy;
  p.z = dz;
  p.n = n;
  p.stride = stride;
  for (int a = 0; a < 3; ++a) {
    p.o[a] = sensor[a];
    p.win[a] = g->origin_i[a];
    p.half[a] = g->half[a];
    p.map[a] = g->map[a];
  }
  p.res = g->res;
  p.inv = g->res_inv;
  p.max_range = g->max_range;
  p.vnum = g->voxel_num;
  p.ctr = g->ctr ? 1 : 0;
  p.fp = g->fp;
  p.cnt = g->d_cnt;
  p.hit = g->d_hit;
  p.stats = g->stats_on ? g->d_stats : nullptr;
  p.err = g->d_err;
  p.lay = g->lay;
  p.dirty = g->d_dirty;
  if ((g->opt_raycast == 1 || (g->opt_raycast == 2 && g->opt_sort)) && n > g->bin_cap) {
    CK(cudaStreamSynchronize(g->stream));
    cublox_b200::detail::dfree(g->d_bins);
    cublox_b200::detail::dfree(g->d_sorted);
    g->d_bins = nullptr;
    g->d_sorted = nullptr;
    g->bin_cap = 0;
    if (!g->d_hist && cublox_b200::detail::dmalloc(&g->d_hist, sizeof(int) * 2 * binned_bins()) != cudaSuccess) {
      cudaGetLastError();
      return fail(CUBLOX_ERR_NOMEM, "update: bin buffer allocation failed");
    }
    if (cublox_b200::detail::dmalloc(&g->d_bins, sizeof(int) * static_cast<size_t>(n)) != cudaSuccess ||
        cublox_b200::detail::dmalloc(&g->d_sorted, sizeof(float) * 3 * static_cast<size_t>(n)) != cudaSuccess) {
      cudaGetLastError();
      return fail(CUBLOX_ERR_NOMEM, "update: sort buffer allocation failed");
    }
    g->bin_cap = n;
  }
  tmark(g, 0, 0);
  if (g->opt_raycast == 2 && p.stride != 1) {
    // the split walk reads SoA: gather an AoS cloud first
    int rc = ensure_cloud(g, n);
    if (rc) return rc;
    if (dx != g->d_cloud) {
      launch_gather_soa(dx, CUBLOX_LAYOUT_AOS, n, g->d_cloud, g->stream);
      CK_LAUNCH();
      p.x = g->d_cloud;
      p.y = g->d_cloud + n;
      p.z = g->d_cloud + 2 * static_cast<size_t>(n);
      p.stride = 1;
    }
  }
  constexpr int kMaxSegsPerRay = 16;
  if (g->opt_raycast == 2 && (n > g->split_cap || !g->d_work)) {
    CK(cudaStreamSynchronize(g->stream));
    cublox_b200::detail::dfree(g->d_segs);
    cublox_b200::detail::dfree(g->d_rays);
    g->d_segs = nullptr;
    g->d_rays = nullptr;
    g->split_cap = 0;
    if ((!g->d_work && cublox_b200::detail::dmalloc(&g->d_work, 2 * sizeof(int)) != cudaSuccess) ||
        cublox_b200::detail::dmalloc(&g->d_segs, split_seg_bytes() * kMaxSegsPerRay * static_cast<size_t>(n)) !=
            cudaSuccess ||
        cublox_b200::detail::dmalloc(&g->d_rays, split_ray_bytes() * static_cast<size_t>(n)) != cudaSuccess) {
      cudaGetLastError();
      return fail(CUBLOX_ERR_NOMEM, "update: split-walk scratch allocation failed");
    }
    g->split_cap = n;
  }
  if (g->opt_raycast == 2) {
    SplitScratch sc{g->d_segs, g->d_rays, g->d_work, kMaxSegsPerRay * n, kMaxSegsPerRay,
                    g->opt_block, g->opt_contig};
    RayParams ps = p;
    if (g->opt_sort) {
      BinnedScratch b{g->d_bins, g->d_hist, g->d_hist + binned_bins(), g->d_sorted};
      launch_direction_sort(p, b, g->stream);
      ps.x = g->d_sorted;
      ps.y = g->d_sorted + n;
      ps.z = g->d_sorted + 2 * static_cast<size_t>(n);
      ps.stride = 1;
    }
    launch_raycast_split(ps, g->opt_cube, g->opt_flat, g->opt_seg, sc, g->stream);
  } else if (g->opt_raycast == 1) {
    BinnedScratch b{g->d_bins, g->d_hist, g->d_hist + binned_bins(), g->d_sorted};
    launch_raycast_binned(p, b, g->opt_cube, g->opt_match != 0, g->opt_sort != 0, g->stream);
  } else {
    launch_raycast(p, g->stream);
  }
  CK_LAUNCH();
  tmark(g, 0, 1);
  if (count_only) return CUBLOX_OK;
  ApplyParams a{};
  a.occ = g->d_occ;
  a.cnt = g->d_cnt;
  a.hit = g->d_hit;
  a.vnum = g->voxel_num;
  a.l_hit = g->l_hit;
  a.l_miss = g->l_miss;
  a.l_min = g->l_min;
  a.l_max = g->l_max;
  a.l_unknown = g->l_unknown;
  a.fp = g->fp;
  a.stats = g->stats_on ? g->d_stats : nullptr;
  a.variant = g->opt_fold;
  a.dirty = g->d_dirty;
  a.nlines = g->nlines;
  a.err = g->d_err;
  a.vnum = static_cast<int>(std::min<int64_t>(g->nalloc, std::numeric_limits<int>::max()));
  tmark(g, 1, 0);
  launch_apply(a, g->stream);
  CK_LAUNCH();
  // the full sweeps leave the line flags set: clear them
  if (a.variant < 2)
    CK(cudaMemsetAsync(g->d_dirty, 0, static_cast<size_t>(g->nlines), g->stream));
  tmark(g, 1, 1);
  return CUBLOX_OK;
}

}  // extern "C"

void cublox_b200::detail::snap_first_run(cublox_grid *g, const float sensor[3]) {
  if (!g->first_run) return;
  int o[3];
  for (int a = 0; a < 3; ++a) o[a] = host_p2g(sensor[a], g->res_inv, g->ctr);
  set_origin(g, o);
  g->first_run = false;
}

RayParams cublox_b200::detail::ray_params(const cublox_grid *g, const float *x,
                                          const float *y, const float *z, int n, int stride,
                                          const float sensor[3]) {
  RayParams p{};
  p.x = x;
  p.y = y;
  p.z = z;
  p.n = n;
  p.stride = stride;
  for (int a = 0; a < 3; ++a) {
    p.o[a] = sensor[a];
    p.win[a] = g->origin_i[a];
    p.half[a] = g->half[a];
    p.map[a] = g->map[a];
  }
  p.res = g->res;
  p.inv = g->res_inv;
  p.max_range = g->max_range;
  p.vnum = g->voxel_num;
  p.ctr = g->ctr ? 1 : 0;
  p.fp = g->fp;
  p.cnt = g->d_cnt;
  p.hit = g->d_hit;
  p.stats = g->stats_on ? g->d_stats : nullptr;
  p.err = g->d_err;
  p.lay = g->lay;
  p.dirty = g->d_dirty;
  return p;
}

size_t cublox_b200::detail::device_bytes(const cublox_grid *g) {
  size_t b = 12 * static_cast<size_t>(g->d_occ ? g->nalloc : 0) + static_cast<size_t>(g->nlines);
  b += sizeof(float) * 3 * (static_cast<size_t>(g->cloud_cap) + static_cast<size_t>(g->world_cap));
  b += g->image_cap;
  b += g->fs.fq_bytes + 13 * static_cast<size_t>(g->fs.fcap) + 13 * static_cast<size_t>(g->qcap);
  b += static_cast<size_t>(g->split_cap) * (16 * split_seg_bytes() + split_ray_bytes());
  b += static_cast<size_t>(g->bin_cap) * 16;
  return b;
}

int cublox_b200::detail::release_scratch(cublox_grid *g) {
  const cudaError_t e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess) return cuda_fail(e, "release_scratch", __LINE__);
  cublox_b200::detail::dfree(g->d_world);
  g->d_world = nullptr;
  g->world_cap = 0;
  cublox_b200::detail::dfree(g->d_image);
  g->d_image = nullptr;
  g->image_cap = 0;
  void **bufs[] = {reinterpret_cast<void **>(&g->d_cloud), reinterpret_cast<void **>(&g->d_bins),
                   reinterpret_cast<void **>(&g->d_work),  reinterpret_cast<void **>(&g->d_segs),
                   reinterpret_cast<void **>(&g->d_rays),  reinterpret_cast<void **>(&g->d_hist),
                   reinterpret_cast<void **>(&g->d_sorted),
                   reinterpret_cast<void **>(&g->d_qout),  reinterpret_cast<void **>(&g->d_qin)};
  for (void **b : bufs) {
    cublox_b200::detail::dfree(*b);
    *b = nullptr;
  }
  g->cloud_cap = g->split_cap = g->bin_cap = g->qcap = 0;
  cublox_b200::detail::free_fetch(&g->fs);
  return CUBLOX_OK;
}

int cublox_b200::detail::acquire_device(cublox_grid *g, const float *occ_host) {
  const size_t n = static_cast<size_t>(g->nalloc);
  cudaError_t e = cudaSuccess;
  if (!g->d_occ) e = cublox_b200::detail::dmalloc(&g->d_occ, n * sizeof(float));
  if (e == cudaSuccess && !g->d_cnt) e = cublox_b200::detail::dmalloc(&g->d_cnt, n * sizeof(uint32_t));
  if (e == cudaSuccess && !g->d_hit) e = cublox_b200::detail::dmalloc(&g->d_hit, n * sizeof(uint32_t));
  if (e != cudaSuccess) {
    cudaGetLastError();
    cublox_b200::detail::dfree(g->d_occ);
    cublox_b200::detail::dfree(g->d_cnt);
    cublox_b200::detail::dfree(g->d_hit);
    g->d_occ = nullptr;
    g->d_cnt = g->d_hit = nullptr;
    return fail(CUBLOX_ERR_NOMEM, "acquire_device: voxel buffers do not fit");
  }
  if ((e = cudaMemsetAsync(g->d_cnt, 0, n * sizeof(uint32_t), g->stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(g->d_hit, 0, n * sizeof(uint32_t), g->stream)) != cudaSuccess)
    return cuda_fail(e, "acquire_device", __LINE__);
  if (occ_host)
    e = cudaMemcpyAsync(g->d_occ, occ_host, n * sizeof(float), cudaMemcpyHostToDevice, g->stream);
  else
    e = cudaMemsetAsync(g->d_occ, 0, n * sizeof(float), g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess) return cuda_fail(e, "acquire_device", __LINE__);
  return CUBLOX_OK;
}

int cublox_b200::detail::detach_voxels(cublox_grid *g, float *occ_host, VoxelBuffers *out) {
  if (!g->d_occ) return fail(CUBLOX_ERR_INVALID, "detach_voxels: grid holds no voxel buffers");
  if (occ_host) {
    const cudaError_t e = cudaMemcpyAsync(occ_host, g->d_occ,
                                          sizeof(float) * static_cast<size_t>(g->nalloc),
                                          cudaMemcpyDeviceToHost, g->stream);
    if (e != cudaSuccess) return cuda_fail(e, "detach_voxels", __LINE__);
  }
  out->nalloc = g->nalloc;
  out->occ = g->d_occ;
  out->cnt = g->d_cnt;
  out->hit = g->d_hit;
  g->d_occ = nullptr;
  g->d_cnt = g->d_hit = nullptr;
  return CUBLOX_OK;
}

int cublox_b200::detail::attach_voxels(cublox_grid *g, VoxelBuffers *in, const float *occ_host) {
  if (g->d_occ || in->nalloc != g->nalloc || !in->occ)
    return fail(CUBLOX_ERR_INVALID, "attach_voxels: buffers of another size, or grid not empty");
  const size_t n = static_cast<size_t>(g->nalloc);
  const cudaError_t e =
      occ_host ? cudaMemcpyAsync(in->occ, occ_host, n * sizeof(float), cudaMemcpyHostToDevice,
                                 g->stream)
               : cudaMemsetAsync(in->occ, 0, n * sizeof(float), g->stream);
  if (e != cudaSuccess) return cuda_fail(e, "attach_voxels", __LINE__);
  g->d_occ = in->occ;
  g->d_cnt = in->cnt;
  g->d_hit = in->hit;
  *in = VoxelBuffers{};
  return CUBLOX_OK;
}

using cublox_b200::detail::snap_first_run;

extern "C" {

static int update_impl(cublox_grid *g, const float *x, const float *y,
                       const float *z, const float *xyz, int layout, int n,
                       const float sensor[3]) {
  if (!g || !sensor) return fail(CUBLOX_ERR_INVALID, "cublox_grid_update: null argument");
  if (g->voxel_num <= 0 || n <= 0) return CUBLOX_OK;  // OccupancyGrid.cpp:183-190
  const void *probe = xyz ? static_cast<const void *>(xyz) : static_cast<const void *>(x);
  if (!probe || (!xyz && (!y || !z)))
    return fail(CUBLOX_ERR_INVALID, "cublox_grid_update: null cloud");
  snap_first_run(g, sensor);
  const int kind = mem_kind(probe);
  const bool dev = kind == 2;
  if (dev && xyz && layout == CUBLOX_LAYOUT_AOS)
    return integrate(g, xyz, xyz + 1, xyz + 2, n, 3, sensor);
  if (dev && xyz)
    return integrate(g, xyz, xyz + n, xyz + 2 * static_cast<size_t>(n), n, 1, sensor);
  if (dev) return integrate(g, x, y, z, n, 1, sensor);
  int rc = ensure_cloud(g, n);
  if (rc) return rc;
  const size_t nbytes = sizeof(float) * static_cast<size_t>(n);
  if (kind == 1 && xyz) {
    // Pinned host cloud: copy straight from it; return once the copy has
    // landed so the caller may reuse its buffer.
    CK(cudaMemcpyAsync(g->d_cloud, xyz, 3 * nbytes, cudaMemcpyHostToDevice, g->stream));
    if (!g->stage_ev[0]) CK(cudaEventCreateWithFlags(&g->stage_ev[0], cudaEventDisableTiming));
    CK(cudaEventRecord(g->stage_ev[0], g->stream));
    rc = layout == CUBLOX_LAYOUT_AOS
             ? integrate(g, g->d_cloud, g->d_cloud + 1, g->d_cloud + 2, n, 3, sensor)
             : integrate(g, g->d_cloud, g->d_cloud + n, g->d_cloud + 2 * static_cast<size_t>(n),
                         n, 1, sensor);
    if (rc) return rc;
    CK(cudaEventSynchronize(g->stage_ev[0]));
    return CUBLOX_OK;
  }
  // Pageable host cloud: stage into pinned memory, one async copy, then
  // integrate.
  rc = ensure_stage(g, n);
  if (rc) return rc;
  const int s = g->stage_idx;
  g->stage_idx ^= 1;
  CK(cudaEventSynchronize(g->stage_ev[s]));
  float *h = g->h_stage[s];
  const size_t nb = sizeof(float) * static_cast<size_t>(n);
  if (xyz && layout == CUBLOX_LAYOUT_AOS) {
    for (int i = 0; i < n; ++i) {
      h[i] = xyz[3 * static_cast<size_t>(i)];
      h[n + i] = xyz[3 * static_cast<size_t>(i) + 1];
      h[2 * static_cast<size_t>(n) + i] = xyz[3 * static_cast<size_t>(i) + 2];
    }
  } else if (xyz) {
    std::memcpy(h, xyz, 3 * nb);
  } else {
    std::memcpy(h, x, nb);
    std::memcpy(h + n, y, nb);
    std::memcpy(h + 2 * static_cast<size_t>(n), z, nb);
  }
  CK(cudaMemcpyAsync(g->d_cloud, h, 3 * nb, cudaMemcpyHostToDevice, g->stream));
  CK(cudaEventRecord(g->stage_ev[s], g->stream));
  return integrate(g, g->d_cloud, g->d_cloud + n, g->d_cloud + 2 * static_cast<size_t>(n), n,
                   1, sensor);
}

int cublox_grid_update(cublox_grid *g, const float *x, const float *y,
                       const float *z, int n, const float sensor_origin[3]) {
  return update_impl(g, x, y, z, nullptr, CUBLOX_LAYOUT_SOA, n, sensor_origin);
}

int cublox_grid_update_xyz(cublox_grid *g, const float *xyz, int layout,
                           int n, const float sensor_origin[3]) {
  if (layout != CUBLOX_LAYOUT_SOA && layout != CUBLOX_LAYOUT_AOS)
    return fail(CUBLOX_ERR_INVALID, "cublox_grid_update_xyz: unknown layout");
  return update_impl(g, nullptr, nullptr, nullptr, xyz, layout, n, sensor_origin);
}

// buildCloudInOdomFrame uses at most the first kMaxCloudPoints points of a
// cloud (src/main.cpp:54, :655-661).
constexpr int kDriverCloudCap = 1000000;

static int ensure_world(cublox_grid *g, int n) {
  if (n <= g->world_cap) return CUBLOX_OK;
  CK(cudaStreamSynchronize(g->stream));
  cublox_b200::detail::dfree(g->d_world);
  g->d_world = nullptr;
  g->world_cap = 0;
  if (cublox_b200::detail::dmalloc(&g->d_world, sizeof(float) * 3 * static_cast<size_t>(n)) != cudaSuccess) {
    cudaGetLastError();
    return fail(CUBLOX_ERR_NOMEM, "sensor-frame update: world buffer allocation failed");
  }
  g->world_cap = n;
  return CUBLOX_OK;
}

// Ingest parameters of a sensor-frame update; on the first run the kept
// points are counted (the driver calls update() only if one survives, and
// the first call snaps the window).
static int world_params(cublox_grid *g, int n, const float rotation[9],
                        const float translation[3], IngestParams *ip) {
  int rc = ensure_world(g, n);
  if (rc) return rc;
  *ip = IngestParams{};
  ip->n = n;
  for (int i = 0; i < 9; ++i) ip->R[i] = rotation[i];
  for (int a = 0; a < 3; ++a) ip->t[a] = translation[a];
  ip->max_r2 = fmul(g->max_range, g->max_range);  // main.cpp:451
  ip->dst = g->d_world;
  ip->count = nullptr;
  if (g->first_run) {
    if (!g->d_kept && cublox_b200::detail::dmalloc(&g->d_kept, sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      return fail(CUBLOX_ERR_NOMEM, "sensor-frame update: allocation failed");
    }
    CK(cudaMemsetAsync(g->d_kept, 0, sizeof(int), g->stream));
    ip->count = g->d_kept;
  }
  return CUBLOX_OK;
}

// After the ingest launch: update(world_cloud, translation), unless nothing
// survived the driver's filters on the first run.
static int world_update(cublox_grid *g, const IngestParams &ip, const float translation[3]) {
  if (ip.count) {
    int kept = 0;
    CK(cudaMemcpyAsync(&kept, ip.count, sizeof(int), cudaMemcpyDeviceToHost, g->stream));
    CK(cudaStreamSynchronize(g->stream));
    if (kept == 0) return CUBLOX_OK;
  }
  snap_first_run(g, translation);
  const int n = ip.n;
  return integrate(g, g->d_world, g->d_world + n, g->d_world + 2 * static_cast<size_t>(n), n, 1,
                   translation);
}

// update() from a sensor-frame cloud and the sensor pose: the reference
// driver's buildCloudInOdomFrame (src/main.cpp:640-693) on the device, then
// update(world_cloud, t) (OccupancyGrid.cpp:181-238).
int cublox_grid_update_pose(cublox_grid *g, const float *xyz, int layout, int n,
                            const float rotation[9], const float translation[3]) {
  if (!g || !rotation || !translation || (n > 0 && !xyz))
    return fail(CUBLOX_ERR_INVALID, "cublox_grid_update_pose: null argument");
  if (layout != CUBLOX_LAYOUT_SOA && layout != CUBLOX_LAYOUT_AOS)
    return fail(CUBLOX_ERR_INVALID, "cublox_grid_update_pose: unknown layout");
  if (g->voxel_num <= 0 || n <= 0) return CUBLOX_OK;  // the driver skips empty clouds
  int rc;
  // the raw cloud on the device, in its own layout
  const float *src = xyz;
  if (mem_kind(xyz) != 2) {
    if ((rc = ensure_cloud(g, n))) return rc;
    const size_t bytes = sizeof(float) * 3 * static_cast<size_t>(n);
    if (mem_kind(xyz) == 1) {
      CK(cudaMemcpyAsync(g->d_cloud, xyz, bytes, cudaMemcpyHostToDevice, g->stream));
      if (!g->stage_ev[0]) CK(cudaEventCreateWithFlags(&g->stage_ev[0], cudaEventDisableTiming));
      CK(cudaEventRecord(g->stage_ev[0], g->stream));
      CK(cudaEventSynchronize(g->stage_ev[0]));  // the caller may reuse its buffer
    } else {
      if ((rc = ensure_stage(g, n))) return rc;
      const int s = g->stage_idx;
      g->stage_idx ^= 1;
      CK(cudaEventSynchronize(g->stage_ev[s]));
      std::memcpy(g->h_stage[s], xyz, bytes);
      CK(cudaMemcpyAsync(g->d_cloud, g->h_stage[s], bytes, cudaMemcpyHostToDevice, g->stream));
      CK(cudaEventRecord(g->stage_ev[s], g->stream));
    }
    src = g->d_cloud;
  }
  IngestParams ip;
  if ((rc = world_params(g, std::min(n, kDriverCloudCap), rotation, translation, &ip))) return rc;
  ip.xyz = src;
  ip.layout = layout;
  ip.col = n;
  launch_ingest(ip, g->stream);
  CK_LAUNCH();
  return world_update(g, ip, translation);
}

// update() from a depth image, as the reference driver's depthCallback
// (src/main.cpp:558-638) turns it into a cloud before the same steps.
int cublox_grid_update_depth(cublox_grid *g, const void *image, int encoding, int width,
                             int height, int64_t step, const float intrinsics[4],
                             const float rotation[9], const float translation[3]) {
  if (!g || !intrinsics || !rotation || !translation)
    return fail(CUBLOX_ERR_INVALID, "cublox_grid_update_depth: null argument");
  if (encoding != CUBLOX_DEPTH_U16_MM && encoding != CUBLOX_DEPTH_F32_M)
    return fail(CUBLOX_ERR_INVALID, "cublox_grid_update_depth: unknown encoding");
  const int64_t px = encoding == CUBLOX_DEPTH_U16_MM ? 2 : 4;
  if (width < 0 || height < 0 || step < px * width ||
      static_cast<int64_t>(width) * height > 0x7fffffff)
    return fail(CUBLOX_ERR_INVALID, "cublox_grid_update_depth: bad image size or step");
  const int n = width * height;
  if (g->voxel_num <= 0 || n == 0) return CUBLOX_OK;  // depthCallback returns on 0 x 0
  if (!image) return fail(CUBLOX_ERR_INVALID, "cublox_grid_update_depth: null image");
  const size_t bytes = static_cast<size_t>(step) * static_cast<size_t>(height);
  const unsigned char *dimg = static_cast<const unsigned char *>(image);
  if (mem_kind(image) != 2) {
    if (bytes > g->image_cap) {
      CK(cudaStreamSynchronize(g->stream));
      cublox_b200::detail::dfree(g->d_image);
      g->d_image = nullptr;
      g->image_cap = 0;
      if (cublox_b200::detail::dmalloc(&g->d_image, bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(CUBLOX_ERR_NOMEM, "cublox_grid_update_depth: image buffer allocation failed");
      }
      g->image_cap = bytes;
    }
    CK(cudaMemcpyAsync(g->d_image, image, bytes, cudaMemcpyHostToDevice, g->stream));
    if (!g->stage_ev[0]) CK(cudaEventCreateWithFlags(&g->stage_ev[0], cudaEventDisableTiming));
    CK(cudaEventRecord(g->stage_ev[0], g->stream));
    CK(cudaEventSynchronize(g->stage_ev[0]));  // the caller may reuse its image
    dimg = g->d_image;
  }
  DepthParams dp{};
  int rc = world_params(g, std::min(n, kDriverCloudCap), rotation, translation, &dp.ingest);
  if (rc) return rc;
  dp.image = dimg;
  dp.encoding = encoding;
  dp.width = width;
  dp.height = height;
  dp.step = step;
  dp.fx = intrinsics[0];
  dp.fy = intrinsics[1];
  dp.cx = intrinsics[2];
  dp.cy = intrinsics[3];
  launch_depth(dp, g->stream);
  CK_LAUNCH();
  return world_update(g, dp.ingest, translation);
}

// ---- recenter ---------------------------------------------------------------
int cublox_grid_set_recenter_mode(cublox_grid *g, int mode) {
  if (!g || (mode != 0 && mode != 1)) return fail(CUBLOX_ERR_INVALID, "bad recenter mode");
  g->recenter_mode = mode;
  return CUBLOX_OK;
}

static int normalize_slice(int x, int half) {
  const int range = 2 * half + 1;
  int y = (x + half) % range;
  if (y < 0) y += range;
  return y - half;
}

int cublox_grid_recenter(cublox_grid *g, const float pos[3], int *action) {
  if (action) *action = 0;
  if (!g || !pos) return fail(CUBLOX_ERR_INVALID, "cublox_grid_recenter: null argument");
  g->last_cleared = 0;
  if (!g->has_thr || g->voxel_num <= 0) return CUBLOX_OK;  // OccupancyGrid.cpp:142-145
  const float dx = pos[0] - g->origin_f[0];
  const float dy = pos[1] - g->origin_f[1];
  const float dz = pos[2] - g->origin_f[2];
  // Host gate (OccupancyGrid.cpp:148): Eigen squaredNorm, no FMA.
  if (sos(dx, dy, dz, kSosPlain) < g->thr_sq) return CUBLOX_OK;
  // planRecenterKernel's own re-check (kernels.cu:326-331), device rounding.
  if (sos(dx, dy, dz, (g->fp >> kFpRecSosShift) & 7u) < g->thr_sq) return CUBLOX_OK;
  int no[3], shift[3];
  int max_shift = 0, max_map = 0;
  for (int a = 0; a < 3; ++a) {
    no[a] = pos_to_global_dev(pos[a], g->res_inv, g->ctr, g->fp);
    shift[a] = no[a] - g->origin_i[a];
    max_shift = std::max(max_shift, std::abs(shift[a]));
    max_map = std::max(max_map, g->map[a]);
  }
  if (max_shift >= max_map) {  // kernels.cu:338-347, :652-662
    CK(cudaMemsetAsync(g->d_occ, 0, sizeof(float) * static_cast<size_t>(g->nalloc),
                       g->stream));
    g->last_cleared = g->voxel_num;
    set_origin(g, no);
    if (action) *action = 2;
    return CUBLOX_OK;
  }
  // Slab plan (kernels.cu:355-397) as a union of marked local slots.
  std::vector<uint32_t> masks(g->mask_words[0] + g->mask_words[1] + g->mask_words[2], 0u);
  uint32_t *m[3] = {masks.data(), masks.data() + g->mask_words[0],
                    masks.data() + g->mask_words[0] + g->mask_words[1]};
  auto mark = [&](int a, int l) {
    const int s = l + g->half[a];
    m[a][s >> 5] |= 1u << (s & 31);
  };
  const bool compat = g->recenter_mode == 0;
  bool any_z = false;
  for (int a = 0; a < 3; ++a) {
    const int sh = shift[a];
    if (sh == 0) continue;
    const int half = g->half[a];
    const int min_l = (-half + g->origin_i[a]) % g->map[a];
    const int n = std::min(std::abs(sh), g->map[a]);
    if (sh > 0) {
      for (int k = 0; k < n; ++k) mark(a, normalize_slice(min_l + k, half));
      if (compat)
        for (int k = 0; k < n; ++k) mark(a, normalize_slice(half - k, half));
    } else {
      for (int k = 1; k <= n; ++k) mark(a, normalize_slice(min_l - k, half));
      if (compat)
        for (int k = 0; k < n; ++k) mark(a, normalize_slice(-half + k, half));
    }
    if (a == 2) any_z = true;
  }
  {
    int64_t keep = 1;  // voxels on no marked slab
    for (int a = 0; a < 3; ++a) {
      int marked = 0;
      for (int w = 0; w < g->mask_words[a]; ++w) marked += __builtin_popcount(m[a][w]);
      keep *= g->map[a] - marked;
    }
    g->last_cleared = g->voxel_num - keep;
  }
  // Brick layouts: the bricks holding a marked slab, as three lists (x
  // brick columns, y brick rows, z brick levels), all cleared by one kernel
  // (a column whose slots are all marked is written as whole lines).
  const bool bricks = g->lay_code != 0;
  std::vector<int> blist;
  int nb[3] = {0, 0, 0};
  std::vector<std::pair<int, int>> x_runs;  // [first, end) brick columns (bricks) or slabs
  auto marked = [&](int a, int sl) { return ((m[a][sl >> 5] >> (sl & 31)) & 1u) != 0; };
  if (bricks) {
    for (int a = 0; a < 3; ++a) {
      const int B = 1 << g->lay.lb[a];
      for (int b = 0; b < g->nbr[a]; ++b) {
        bool any = false;
        for (int sl = b * B; sl < std::min((b + 1) * B, g->map[a]); ++sl) any |= marked(a, sl);
        if (!any) continue;
        blist.push_back(b);
        ++nb[a];
      }
    }
  } else {
    // A marked x slab is one contiguous run of ny*nz values, and
    // neighbouring marked slabs are neighbouring runs.
    for (int x = 0; x < g->map[0];) {
      if (!marked(0, x)) {
        ++x;
        continue;
      }
      int e = x;
      while (e < g->map[0] && marked(0, e)) ++e;
      x_runs.push_back({x, e});
      x = e;
    }
  }
  const size_t mwords = masks.size();
  masks.insert(masks.end(), blist.begin(), blist.end());
  const size_t mb = masks.size() * sizeof(uint32_t);
  // Pinned staging in two halves used in turn: a half is reused once the
  // recenter before last has copied out of it, so the host does not wait
  // for the stream's current work.
  const int half = g->mask_half;
  g->mask_half ^= 1;
  uint32_t *stage = g->h_masks + half * g->mask_stage_words;
  CK(cudaEventSynchronize(g->mask_ev[half]));
  std::memcpy(stage, masks.data(), mb);
  CK(cudaMemcpyAsync(g->d_masks, stage, mb, cudaMemcpyHostToDevice, g->stream));
  CK(cudaEventRecord(g->mask_ev[half], g->stream));
  ClearParams cp{};
  cp.occ = g->d_occ;
  cp.xmask = g->d_masks;
  cp.ymask = g->d_masks + g->mask_words[0];
  cp.zmask = g->d_masks + g->mask_words[0] + g->mask_words[1];
  for (int a = 0; a < 3; ++a) cp.map[a] = g->map[a];
  cp.any_z = any_z ? 1 : 0;
  cp.lay = g->lay;
  tmark(g, 2, 0);
  // x runs: memsets at copy bandwidth
  const size_t run = bricks ? static_cast<size_t>(g->lay.bs[0])
                            : static_cast<size_t>(g->map[1]) * g->map[2];
  for (const auto &r : x_runs)
    CK(cudaMemsetAsync(g->d_occ + static_cast<size_t>(r.first) * run, 0,
                       sizeof(float) * run * static_cast<size_t>(r.second - r.first),
                       g->stream));
  cp.x_done = 1;
  if (bricks) {
    cp.blist = reinterpret_cast<const int *>(g->d_masks + mwords);
    for (int a = 0; a < 3; ++a) {
      cp.nb[a] = nb[a];
      cp.nbr[a] = g->nbr[a];
    }
    if (nb[0] + nb[1] + nb[2] > 0) {
      launch_clear(cp, g->stream);
      CK_LAUNCH();
    }
  } else {
    bool any_y = false;
    for (int w = 0; w < g->mask_words[1]; ++w) any_y = any_y || m[1][w] != 0u;
    if (any_y || any_z) {
      launch_clear(cp, g->stream);
      CK_LAUNCH();
    }
  }
  tmark(g, 2, 1);
  set_origin(g, no);
  if (action) *action = 1;
  return CUBLOX_OK;
}

// ---- fetch -------------------------------------------------------------------
namespace {
struct QueryBox {
  int box[8];
  float r2;
};

// fetchOccupancyAround's host part (OccupancyGrid.cpp:244-293) for one centre:
// the window-clipped candidate box, or an empty box.
QueryBox plan_query(const cublox_grid *g, const float c[3], float radius) {
  QueryBox q{};
  q.box[0] = 0;
  q.box[1] = -1;  // empty
  q.box[2] = 0;
  q.box[3] = -1;
  q.box[4] = 0;
  q.box[5] = -1;
  q.r2 = 0.0f;
  if (g->voxel_num <= 0 || radius <= 0.0f) return q;
  int cg[3];
  for (int a = 0; a < 3; ++a) cg[a] = host_p2g(c[a], g->res_inv, g->ctr);
  float margin = 0.0f;
  {
    const int mx = g->half[0] - std::abs(cg[0] - g->origin_i[0]);
    const int my = g->half[1] - std::abs(cg[1] - g->origin_i[1]);
    if (mx >= 0 && my >= 0) margin = static_cast<float>(std::min(mx, my)) * g->res;
  }
  const float r_eff = std::min(radius, margin);
  if (r_eff <= 0.0f) return q;
  int gmin[3], gmax[3], wmin[3], wmax[3];
  for (int a = 0; a < 3; ++a) {
    wmin[a] = g->origin_i[a] - g->half[a];
    wmax[a] = g->origin_i[a] + g->half[a];
    gmin[a] = std::max(host_p2g(c[a] - r_eff, g->res_inv, g->ctr), wmin[a]);
    gmax[a] = std::min(host_p2g(c[a] + r_eff, g->res_inv, g->ctr), wmax[a]);
    if (gmax[a] < gmin[a]) return q;
  }
  const int disk_r = d2i_x86(std::ceil(static_cast<double>(r_eff * g->res_inv)));
  const int nz = gmax[2] - gmin[2] + 1;
  const int diam = 2 * disk_r + 1;
  const int64_t est = static_cast<int64_t>(diam) * diam * nz;
  if (est <= 0 || est > std::numeric_limits<int>::max() || disk_r < 0) return q;
  // The reference's threads cover x, y in cg +- disk_r (plus a tail that
  // never passes the sphere test) and z in [gmin.z, gmax.z]; its per-voxel
  // window test is applied here as a clip.
  q.box[0] = std::max(cg[0] - disk_r, wmin[0]);
  q.box[1] = std::min(cg[0] + disk_r, wmax[0]);
  q.box[2] = std::max(cg[1] - disk_r, wmin[1]);
  q.box[3] = std::min(cg[1] + disk_r, wmax[1]);
  q.box[4] = gmin[2];
  q.box[5] = gmax[2];
  q.r2 = r_eff * r_eff;
  return q;
}
}  // namespace

// Fetch scratch grows geometrically: a reallocation frees memory, which
// waits for the whole device.
static int ensure_fq(FetchScratch *sc, cudaStream_t st, size_t bytes) {
  if (bytes <= sc->fq_bytes) return CUBLOX_OK;
  bytes = std::max({bytes, 2 * sc->fq_bytes, static_cast<size_t>(4) << 10});
  CK(cudaStreamSynchronize(st));
  cublox_b200::detail::dfree(sc->fq);
  sc->fq = nullptr;
  sc->fq_bytes = 0;
  if (cublox_b200::detail::dmalloc(&sc->fq, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(CUBLOX_ERR_NOMEM, "fetch: query buffer allocation failed");
  }
  sc->fq_bytes = bytes;
  return CUBLOX_OK;
}
static int ensure_fout(FetchScratch *sc, cudaStream_t st, int64_t n) {
  if (n <= sc->fcap) return CUBLOX_OK;
  n = std::max({n, 2 * sc->fcap, static_cast<int64_t>(1) << 12});
  CK(cudaStreamSynchronize(st));
  cublox_b200::detail::dfree(sc->fpos);
  cublox_b200::detail::dfree(sc->fstate);
  sc->fpos = nullptr;
  sc->fstate = nullptr;
  sc->fcap = 0;
  if (cublox_b200::detail::dmalloc(&sc->fpos, sizeof(float) * 3 * static_cast<size_t>(n)) != cudaSuccess ||
      cublox_b200::detail::dmalloc(&sc->fstate, static_cast<size_t>(n)) != cudaSuccess) {
    cudaGetLastError();
    return fail(CUBLOX_ERR_NOMEM, "fetch: output buffer allocation failed");
  }
  sc->fcap = n;
  return CUBLOX_OK;
}

// Bytes of the query block for nq centres cut into nu work units (the
// layout fetch_impl uses).
static size_t fetch_query_bytes(int nq, int nu) {
  auto al = [](size_t v) { return (v + 255) & ~static_cast<size_t>(255); };
  const size_t ll = al(sizeof(long long) * std::max(nu, 1));
  return al(sizeof(float) * 3 * nq) + al(sizeof(int) * 8 * nq) + al(sizeof(float) * nq) +
         al(sizeof(int) * std::max(nu, 1)) + 4 * ll;
}

static int fetch_impl(cublox_grid *g, cudaStream_t st, const float *centers, int nq,
                      float radius, int filter, int max_results, int64_t *kept,
                      int64_t *offsets, float *out_pos, uint8_t *out_state, int64_t capacity,
                      bool write, std::vector<float> *vpos = nullptr,
                      std::vector<uint8_t> *vstate = nullptr, FetchScratch *sc = nullptr) {
  if (!g || (nq > 0 && !centers)) return fail(CUBLOX_ERR_INVALID, "fetch: null argument");
  if (!sc) sc = &g->fs;
  if (filter < -1 || filter > 2) return fail(CUBLOX_ERR_INVALID, "fetch: bad filter");
  if (nq <= 0) {
    if (offsets) offsets[0] = 0;
    return CUBLOX_OK;
  }
  std::vector<int> boxes(8 * static_cast<size_t>(nq));
  std::vector<float> r2(nq);
  std::vector<long long> cand(nq);
  long long all_cand = 0;
  for (int q = 0; q < nq; ++q) {
    const QueryBox b = plan_query(g, centers + 3 * static_cast<size_t>(q), radius);
    std::memcpy(&boxes[8 * static_cast<size_t>(q)], b.box, sizeof(b.box));
    r2[q] = b.r2;
    const long long nx = b.box[1] - b.box[0] + 1, ny = b.box[3] - b.box[2] + 1,
                    nz = b.box[5] - b.box[4] + 1;
    cand[q] = (nx > 0 && ny > 0 && nz > 0) ? nx * ny * nz : 0;
    all_cand += cand[q];
  }
  // about 32 units per SM, never below kFetchMinUnit candidates
  int sms = 148;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device) != cudaSuccess) {
    cudaGetLastError();
    sms = 148;
  }
  const long long unit = std::max<long long>(kFetchMinUnit, all_cand / (32LL * sms) + 1);
  std::vector<int> uq;
  std::vector<long long> ut0;
  for (int q = 0; q < nq; ++q)
    for (long long t = 0; t < cand[q]; t += unit) {
      uq.push_back(q);
      ut0.push_back(t);
    }
  const int nu = static_cast<int>(uq.size());
  const size_t b_cent = sizeof(float) * 3 * nq, b_box = sizeof(int) * 8 * nq,
               b_r2 = sizeof(float) * nq, b_uq = sizeof(int) * std::max(nu, 1),
               b_ll = sizeof(long long) * std::max(nu, 1);
  auto al = [](size_t v) { return (v + 255) & ~static_cast<size_t>(255); };
  const size_t o_box = al(b_cent), o_r2 = o_box + al(b_box), o_uq = o_r2 + al(b_r2),
               o_ut0 = o_uq + al(b_uq), o_cnt = o_ut0 + al(b_ll), o_off = o_cnt + al(b_ll),
               o_lim = o_off + al(b_ll), total = o_lim + al(b_ll);
  int rc = ensure_fq(sc, st, total);
  if (rc) return rc;
  char *base = static_cast<char *>(sc->fq);
  CK(cudaMemcpyAsync(base, centers, b_cent, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(base + o_box, boxes.data(), b_box, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(base + o_r2, r2.data(), b_r2, cudaMemcpyHostToDevice, st));
  if (nu > 0) {
    CK(cudaMemcpyAsync(base + o_uq, uq.data(), sizeof(int) * nu, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(base + o_ut0, ut0.data(), sizeof(long long) * nu, cudaMemcpyHostToDevice,
                       st));
  }
  FetchParams p{};
  p.occ = g->d_occ;
  p.centers = reinterpret_cast<const float *>(base);
  p.qbox = reinterpret_cast<const int *>(base + o_box);
  p.qr2 = reinterpret_cast<const float *>(base + o_r2);
  p.nq = nq;
  p.uq = reinterpret_cast<const int *>(base + o_uq);
  p.ut0 = reinterpret_cast<const long long *>(base + o_ut0);
  p.nu = nu;
  p.unit = unit;
  for (int a = 0; a < 3; ++a) {
    p.win[a] = g->origin_i[a];
    p.half[a] = g->half[a];
    p.map[a] = g->map[a];
  }
  p.res = g->res;
  p.ctr = g->ctr ? 1 : 0;
  p.fp = g->fp;
  p.l_free = g->l_free;
  p.l_occ = g->l_occ;
  p.l_unknown = g->l_unknown;
  p.filter = filter;
  p.lay = g->lay;
  p.counts = reinterpret_cast<long long *>(base + o_cnt);
  p.offsets = reinterpret_cast<const long long *>(base + o_off);
  p.limits = reinterpret_cast<const long long *>(base + o_lim);
  p.err = g->d_err;
  launch_fetch(p, 1, st);
  CK_LAUNCH();
  std::vector<long long> ucnt(std::max(nu, 1)), uoff(std::max(nu, 1)), ulim(std::max(nu, 1));
  if (nu > 0) {
    CK(cudaMemcpyAsync(ucnt.data(), p.counts, sizeof(long long) * nu, cudaMemcpyDeviceToHost,
                       st));
    CK(cudaStreamSynchronize(st));
  }
  // Per query, its units in order: each keeps what fits under the cap, and
  // writes after everything its query kept before it.
  const long long cap_q = max_results > 0 ? max_results : 500000;  // OccupancyGrid.cpp:292
  std::vector<long long> off(nq + 1);
  off[0] = 0;
  for (int u = 0, q = 0; q < nq; ++q) {
    long long running = 0;
    for (; u < nu && uq[u] == q; ++u) {
      uoff[u] = off[q] + std::min(running, cap_q);
      ulim[u] = std::max(0LL, std::min(ucnt[u], cap_q - running));
      running += ucnt[u];
    }
    const long long lim = std::min(running, cap_q);
    off[q + 1] = off[q] + lim;
    if (kept) kept[q] = lim;
  }
  if (offsets)
    for (int q = 0; q <= nq; ++q) offsets[q] = off[q];
  if (!write) return CUBLOX_OK;
  const long long total_s = off[nq];
  if (vpos && vstate) {
    vpos->resize(3 * static_cast<size_t>(total_s));
    vstate->resize(static_cast<size_t>(total_s));
    out_pos = vpos->data();
    out_state = vstate->data();
    capacity = total_s;
  }
  if (total_s > capacity)
    return fail(CUBLOX_ERR_INVALID, "fetch: output capacity " + std::to_string(capacity) +
                                        " < " + std::to_string(total_s) + " samples");
  if (total_s == 0) return CUBLOX_OK;
  rc = ensure_fout(sc, st, total_s);
  if (rc) return rc;
  CK(cudaMemcpyAsync(base + o_off, uoff.data(), sizeof(long long) * nu, cudaMemcpyHostToDevice,
                     st));
  CK(cudaMemcpyAsync(base + o_lim, ulim.data(), sizeof(long long) * nu, cudaMemcpyHostToDevice,
                     st));
  p.out_pos = sc->fpos;
  p.out_state = sc->fstate;
  launch_fetch(p, 2, st);
  CK_LAUNCH();
  if (out_pos)
    CK(cudaMemcpyAsync(out_pos, sc->fpos, sizeof(float) * 3 * static_cast<size_t>(total_s),
                       cudaMemcpyDeviceToHost, st));
  if (out_state)
    CK(cudaMemcpyAsync(out_state, sc->fstate, static_cast<size_t>(total_s),
                       cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return CUBLOX_OK;
}

}  // extern "C"

int cublox_b200::detail::fetch_into(cublox_grid *g, cudaStream_t st, const float *centers,
                                    int nq, float radius, int filter, int max_results,
                                    std::vector<int64_t> &offsets, std::vector<float> &pos,
                                    std::vector<uint8_t> &state, FetchScratch *sc) {
  offsets.assign(static_cast<size_t>(nq) + 1, 0);
  return fetch_impl(g, st, centers, nq, radius, filter, max_results, nullptr, offsets.data(),
                    nullptr, nullptr, 0, true, &pos, &state, sc);
}

int cublox_b200::detail::reserve_fetch(FetchScratch *sc, int centres, int64_t samples,
                                       cudaStream_t st) {
  // work units: at most 32 per SM plus one per centre (fetch_impl's cut)
  int rc = ensure_fq(sc, st, fetch_query_bytes(centres, centres + 32 * 160));
  if (rc) return rc;
  return ensure_fout(sc, st, samples);
}

void cublox_b200::detail::free_fetch(FetchScratch *sc) {
  cublox_b200::detail::dfree(sc->fq);
  cublox_b200::detail::dfree(sc->fpos);
  cublox_b200::detail::dfree(sc->fstate);
  *sc = FetchScratch{};
}

extern "C" {

// The visualisation cloud the reference's driver publishes after its
// OCCUPIED fetch (src/main.cpp:487-491 -> :740-790), built on the device
// from the fetch samples (ascending global index order here).
int cublox_grid_fetch_viz(cublox_grid *g, const float center[3], float radius, int filter,
                          int max_results, int subsample_step, float max_viz_radius,
                          int64_t max_points, const float robot_pos[3], float *out_xyzrgb,
                          int64_t capacity, int64_t *n_out) {
  if (n_out) *n_out = 0;
  if (!g || !center || !robot_pos || !n_out || (capacity > 0 && !out_xyzrgb))
    return fail(CUBLOX_ERR_INVALID, "fetch_viz: null argument");
  if (max_points < 0) return fail(CUBLOX_ERR_INVALID, "fetch_viz: negative max_points");
  int64_t off[2] = {0, 0};
  int rc = fetch_impl(g, g->stream, center, 1, radius, filter, max_results, nullptr, off,
                      nullptr, nullptr, std::numeric_limits<int64_t>::max(), true);
  if (rc) return rc;
  const int64_t total = off[1];
  if (total == 0 || max_points == 0) return CUBLOX_OK;
  const int64_t cap = std::min<int64_t>(max_points, total);
  if (capacity < cap)
    return fail(CUBLOX_ERR_INVALID, "fetch_viz: capacity " + std::to_string(capacity) + " < " +
                                        std::to_string(cap) + " points");
  // output on the device in the query buffers: d_qin (12 B per query slot)
  // takes the 16 B per point, d_qout (1 B per slot) the 8 B count
  const size_t need = sizeof(float) * 4 * static_cast<size_t>(cap);
  if (static_cast<size_t>(g->qcap) * 12 < need || g->qcap < 8) {
    CK(cudaStreamSynchronize(g->stream));
    cublox_b200::detail::dfree(g->d_qin);
    cublox_b200::detail::dfree(g->d_qout);
    g->d_qin = nullptr;
    g->d_qout = nullptr;
    g->qcap = 0;
    const int q = static_cast<int>(std::max<size_t>((need + 11) / 12, 8));
    if (cublox_b200::detail::dmalloc(&g->d_qin, sizeof(float) * 3 * static_cast<size_t>(q)) != cudaSuccess ||
        cublox_b200::detail::dmalloc(&g->d_qout, static_cast<size_t>(q)) != cudaSuccess) {
      cudaGetLastError();
      return fail(CUBLOX_ERR_NOMEM, "fetch_viz: allocation failed");
    }
    g->qcap = q;
  }
  VizParams vp{};
  vp.pos = g->fs.fpos;
  vp.n = total;
  vp.inv = g->res_inv;
  vp.ctr = g->ctr ? 1 : 0;
  vp.step = subsample_step;
  vp.d_max = max_viz_radius;
  for (int a = 0; a < 3; ++a) vp.o[a] = robot_pos[a];
  vp.max_points = cap;
  vp.out = g->d_qin;
  vp.written = reinterpret_cast<long long *>(g->d_qout);
  launch_viz(vp, g->stream);
  CK_LAUNCH();
  long long written = 0;
  CK(cudaMemcpyAsync(&written, vp.written, sizeof(written), cudaMemcpyDeviceToHost, g->stream));
  CK(cudaStreamSynchronize(g->stream));
  if (written > 0)
    CK(cudaMemcpyAsync(out_xyzrgb, g->d_qin, sizeof(float) * 4 * static_cast<size_t>(written),
                       cudaMemcpyDeviceToHost, g->stream));
  CK(cudaStreamSynchronize(g->stream));
  *n_out = written;
  return CUBLOX_OK;
}

int cublox_grid_fetch(cublox_grid *g, const float center[3], float radius,
                      int filter, int max_results, float *out_pos,
                      uint8_t *out_state, int64_t capacity, int64_t *n_out) {
  if (n_out) *n_out = 0;
  if (!g || !center) return fail(CUBLOX_ERR_INVALID, "cublox_grid_fetch: null argument");
  int64_t kept = 0;
  int rc = fetch_impl(g, g->stream, center, 1, radius, filter, max_results, &kept, nullptr,
                      nullptr, nullptr, 0, false);
  if (rc) return rc;
  if (kept > capacity)
    return fail(CUBLOX_ERR_INVALID, "cublox_grid_fetch: capacity " + std::to_string(capacity) +
                                        " < " + std::to_string(kept) + " samples");
  int64_t off[2];
  rc = fetch_impl(g, g->stream, center, 1, radius, filter, max_results, nullptr, off, out_pos,
                  out_state, capacity, true);
  if (rc) return rc;
  if (n_out) *n_out = off[1];
  return CUBLOX_OK;
}

int cublox_grid_fetch_batch(cublox_grid *g, const float *centers,
                            int n_centers, float radius, int filter,
                            int max_results, int64_t *out_offsets,
                            float *out_pos, uint8_t *out_state,
                            int64_t capacity) {
  if (!out_offsets) return fail(CUBLOX_ERR_INVALID, "fetch_batch: null offsets");
  return fetch_impl(g, g ? g->stream : nullptr, centers, n_centers, radius, filter,
                    max_results, nullptr, out_offsets, out_pos, out_state, capacity, true);
}

int cublox_grid_fetch_counts(cublox_grid *g, const float *centers,
                             int n_centers, float radius, int filter,
                             int max_results, int64_t *out_counts) {
  if (!out_counts) return fail(CUBLOX_ERR_INVALID, "fetch_counts: null output");
  return fetch_impl(g, g ? g->stream : nullptr, centers, n_centers, radius, filter,
                    max_results, out_counts, nullptr, nullptr, nullptr, 0, false);
}

// ---- queries / state access ---------------------------------------------------
int cublox_grid_query_states(cublox_grid *g, const float *xyz, int n,
                             uint8_t *out_state) {
  if (!g || (n > 0 && (!xyz || !out_state)))
    return fail(CUBLOX_ERR_INVALID, "query_states: null argument");
  if (n <= 0) return CUBLOX_OK;
  if (n > g->qcap) {
    CK(cudaStreamSynchronize(g->stream));
    cublox_b200::detail::dfree(g->d_qin);
    cublox_b200::detail::dfree(g->d_qout);
    g->d_qin = nullptr;
    g->d_qout = nullptr;
    g->qcap = 0;
    if (cublox_b200::detail::dmalloc(&g->d_qin, sizeof(float) * 3 * static_cast<size_t>(n)) != cudaSuccess ||
        cublox_b200::detail::dmalloc(&g->d_qout, static_cast<size_t>(n)) != cudaSuccess) {
      cudaGetLastError();
      return fail(CUBLOX_ERR_NOMEM, "query_states: allocation failed");
    }
    g->qcap = n;
  }
  CK(cudaMemcpyAsync(g->d_qin, xyz, sizeof(float) * 3 * static_cast<size_t>(n),
                     cudaMemcpyHostToDevice, g->stream));
  QueryParams p{};
  p.occ = g->d_occ;
  p.xyz = g->d_qin;
  p.n = n;
  for (int a = 0; a < 3; ++a) {
    p.win[a] = g->origin_i[a];
    p.half[a] = g->half[a];
    p.map[a] = g->map[a];
  }
  p.inv = g->res_inv;
  p.ctr = g->ctr ? 1 : 0;
  p.l_free = g->l_free;
  p.l_occ = g->l_occ;
  p.l_unknown = g->l_unknown;
  p.out = g->d_qout;
  p.lay = g->lay;
  launch_query(p, g->stream);
  CK_LAUNCH();
  CK(cudaMemcpyAsync(out_state, g->d_qout, static_cast<size_t>(n), cudaMemcpyDeviceToHost,
                     g->stream));
  CK(cudaStreamSynchronize(g->stream));
  return CUBLOX_OK;
}

int cublox_grid_stored_at(cublox_grid *g, int hash_id, float *out) {
  if (!g || !out) return fail(CUBLOX_ERR_INVALID, "stored_at: null argument");
  *out = 0.0f;
  if (hash_id < 0 || hash_id >= g->voxel_num) return CUBLOX_OK;
  CK(cudaMemcpyAsync(out, g->d_occ + hash_addr(g, hash_id), sizeof(float),
                     cudaMemcpyDeviceToHost, g->stream));
  CK(cudaStreamSynchronize(g->stream));
  return CUBLOX_OK;
}

int cublox_grid_origin(const cublox_grid *g, int origin_i[3], float origin_f[3]) {
  if (!g) return fail(CUBLOX_ERR_INVALID, "null grid");
  for (int a = 0; a < 3; ++a) {
    if (origin_i) origin_i[a] = g->origin_i[a];
    if (origin_f) origin_f[a] = g->origin_f[a];
  }
  return CUBLOX_OK;
}

int cublox_grid_geometry(const cublox_grid *g, int map_size[3], int half[3],
                         int *voxel_num, float *resolution,
                         int *origin_at_center) {
  if (!g) return fail(CUBLOX_ERR_INVALID, "null grid");
  for (int a = 0; a < 3; ++a) {
    if (map_size) map_size[a] = g->map[a];
    if (half) half[a] = g->half[a];
  }
  if (voxel_num) *voxel_num = g->voxel_num;
  if (resolution) *resolution = g->res;
  if (origin_at_center) *origin_at_center = g->ctr ? 1 : 0;
  return CUBLOX_OK;
}

int cublox_grid_first_run(const cublox_grid *g, int *first_run) {
  if (!g || !first_run) return fail(CUBLOX_ERR_INVALID, "null argument");
  *first_run = g->first_run ? 1 : 0;
  return CUBLOX_OK;
}

int cublox_grid_set_origin_index(cublox_grid *g, const int origin_i[3]) {
  if (!g || !origin_i) return fail(CUBLOX_ERR_INVALID, "null argument");
  set_origin(g, origin_i);
  g->first_run = false;
  return CUBLOX_OK;
}

// The stored log-odds in the reference's hash order: gathered on the device
// from the grid's layout into the hit array (zero between scans, rezeroed),
// then copied out.  The reference's own order needs no gather.
int cublox_grid_export(cublox_grid *g, float *occ_host) {
  if (!g || !occ_host) return fail(CUBLOX_ERR_INVALID, "export: null argument");
  const float *src = g->d_occ;
  if (g->lay_code != 0) {
    launch_relayout(g->d_occ, reinterpret_cast<float *>(g->d_hit), g->lay, g->map, 1, g->stream);
    CK_LAUNCH();
    src = reinterpret_cast<const float *>(g->d_hit);
  }
  CK(cudaMemcpyAsync(occ_host, src, sizeof(float) * static_cast<size_t>(g->voxel_num),
                     cudaMemcpyDeviceToHost, g->stream));
  if (g->lay_code != 0)
    CK(cudaMemsetAsync(g->d_hit, 0, sizeof(uint32_t) * static_cast<size_t>(g->nalloc),
                       g->stream));
  CK(cudaStreamSynchronize(g->stream));
  return CUBLOX_OK;
}

int cublox_grid_import(cublox_grid *g, const float *occ_host) {
  if (!g || !occ_host) return fail(CUBLOX_ERR_INVALID, "import: null argument");
  float *dst = g->lay_code != 0 ? reinterpret_cast<float *>(g->d_hit) : g->d_occ;
  CK(cudaMemcpyAsync(dst, occ_host, sizeof(float) * static_cast<size_t>(g->voxel_num),
                     cudaMemcpyHostToDevice, g->stream));
  if (g->lay_code != 0) {
    launch_relayout(dst, g->d_occ, g->lay, g->map, 0, g->stream);
    CK_LAUNCH();
    CK(cudaMemsetAsync(g->d_hit, 0, sizeof(uint32_t) * static_cast<size_t>(g->nalloc),
                       g->stream));
  }
  CK(cudaStreamSynchronize(g->stream));
  return CUBLOX_OK;
}

int cublox_grid_stream(const cublox_grid *g, void **stream) {
  if (!g || !stream) return fail(CUBLOX_ERR_INVALID, "null argument");
  *stream = g->stream;
  return CUBLOX_OK;
}

int cublox_grid_synchronize(cublox_grid *g) {
  if (!g) return fail(CUBLOX_ERR_INVALID, "null grid");
  CK(cudaStreamSynchronize(g->stream));
  return CUBLOX_OK;
}

int cublox_grid_enable_stats(cublox_grid *g, int enable) {
  if (!g) return fail(CUBLOX_ERR_INVALID, "null grid");
  g->stats_on = enable != 0;
  return CUBLOX_OK;
}

int cublox_grid_last_stats(cublox_grid *g, cublox_scan_stats *out) {
  if (!g || !out) return fail(CUBLOX_ERR_INVALID, "null argument");
  unsigned long long v[4];
  CK(cudaMemcpyAsync(v, g->d_stats, sizeof(v), cudaMemcpyDeviceToHost, g->stream));
  CK(cudaStreamSynchronize(g->stream));
  out->rays = static_cast<int64_t>(v[0]);
  out->op_incs = static_cast<int64_t>(v[1]);
  out->hit_incs = static_cast<int64_t>(v[2]);
  out->touched = static_cast<int64_t>(v[3]);
  return CUBLOX_OK;
}

int cublox_grid_count_scan(cublox_grid *g, const float *xyz, int n,
                           const float sensor_origin[3], int32_t *op_out,
                           int32_t *hit_out) {
  if (!g || !sensor_origin || !op_out || !hit_out || (n > 0 && !xyz))
    return fail(CUBLOX_ERR_INVALID, "count_scan: null argument");
  const size_t vb = sizeof(uint32_t) * static_cast<size_t>(g->voxel_num);
  if (n > 0) {
    int rc = ensure_cloud(g, n);
    if (rc) return rc;
    std::vector<float> soa(3 * static_cast<size_t>(n));
    for (int i = 0; i < n; ++i)
      for (int a = 0; a < 3; ++a)
        soa[a * static_cast<size_t>(n) + i] = xyz[3 * static_cast<size_t>(i) + a];
    CK(cudaMemcpyAsync(g->d_cloud, soa.data(), soa.size() * sizeof(float),
                       cudaMemcpyHostToDevice, g->stream));
    rc = integrate(g, g->d_cloud, g->d_cloud + n, g->d_cloud + 2 * static_cast<size_t>(n), n,
                   1, sensor_origin, true);
    if (rc) return rc;
    CK(cudaStreamSynchronize(g->stream));
  }
  (void)vb;
  const size_t ab = sizeof(uint32_t) * static_cast<size_t>(g->nalloc);
  std::vector<uint32_t> c(static_cast<size_t>(g->nalloc)), hh(static_cast<size_t>(g->nalloc));
  CK(cudaMemcpyAsync(c.data(), g->d_cnt, ab, cudaMemcpyDeviceToHost, g->stream));
  CK(cudaMemcpyAsync(hh.data(), g->d_hit, ab, cudaMemcpyDeviceToHost, g->stream));
  CK(cudaMemsetAsync(g->d_cnt, 0, ab, g->stream));
  CK(cudaMemsetAsync(g->d_hit, 0, ab, g->stream));
  CK(cudaMemsetAsync(g->d_dirty, 0, static_cast<size_t>(g->nlines), g->stream));
  CK(cudaStreamSynchronize(g->stream));
  for (int h = 0; h < g->voxel_num; ++h) {
    const int a = hash_addr(g, h);
    op_out[h] = static_cast<int32_t>(c[a] & kOpMask);
    hit_out[h] = (c[a] & kHitFlag) ? static_cast<int32_t>(hh[a]) : 0;
  }
  return CUBLOX_OK;
}

int cublox_grid_enable_timing(cublox_grid *g, int enable) {
  if (!g) return fail(CUBLOX_ERR_INVALID, "null grid");
  if (enable)
    for (int i = 0; i < 6; ++i)
      if (!g->tev[i]) CK(cudaEventCreate(&g->tev[i]));
  g->timing_on = enable != 0;
  for (int i = 0; i < 3; ++i) g->tev_used[i] = false;
  return CUBLOX_OK;
}

int cublox_grid_last_clear(const cublox_grid *g, int64_t *voxels) {
  if (!g || !voxels) return fail(CUBLOX_ERR_INVALID, "null argument");
  *voxels = g->last_cleared;
  return CUBLOX_OK;
}

int cublox_grid_last_timing(cublox_grid *g, float ms[3]) {
  if (!g || !ms) return fail(CUBLOX_ERR_INVALID, "null argument");
  CK(cudaStreamSynchronize(g->stream));
  for (int i = 0; i < 3; ++i) {
    ms[i] = -1.0f;
    if (g->timing_on && g->tev_used[i])
      CK(cudaEventElapsedTime(&ms[i], g->tev[2 * i], g->tev[2 * i + 1]));
    g->tev_used[i] = false;
  }
  return CUBLOX_OK;
}

int cublox_grid_reference_steps(cublox_grid *g, const float *xyz, int n,
                                const float sensor_origin[3], int64_t *voxel_steps) {
  if (!g || !sensor_origin || !voxel_steps || (n > 0 && !xyz))
    return fail(CUBLOX_ERR_INVALID, "reference_steps: null argument");
  *voxel_steps = 0;
  if (n <= 0) return CUBLOX_OK;
  int rc = ensure_cloud(g, n);
  if (rc) return rc;
  CK(cudaMemcpyAsync(g->d_cloud, xyz, sizeof(float) * 3 * static_cast<size_t>(n),
                     cudaMemcpyHostToDevice, g->stream));
  CK(cudaMemsetAsync(g->d_stats, 0, 4 * sizeof(unsigned long long), g->stream));
  RayParams p{};
  p.x = g->d_cloud;
  p.y = g->d_cloud + 1;
  p.z = g->d_cloud + 2;
  p.n = n;
  p.stride = 3;
  for (int a = 0; a < 3; ++a) {
    p.o[a] = sensor_origin[a];
    p.win[a] = g->origin_i[a];
    p.half[a] = g->half[a];
    p.map[a] = g->map[a];
  }
  p.res = g->res;
  p.inv = g->res_inv;
  p.max_range = g->max_range;
  p.vnum = g->voxel_num;
  p.ctr = g->ctr ? 1 : 0;
  p.fp = g->fp;
  p.stats = g->d_stats;
  p.err = g->d_err;
  launch_step_count(p, g->stream);
  CK_LAUNCH();
  unsigned long long v[4];
  CK(cudaMemcpyAsync(v, g->d_stats, sizeof(v), cudaMemcpyDeviceToHost, g->stream));
  CK(cudaStreamSynchronize(g->stream));
  *voxel_steps = static_cast<int64_t>(v[0]);
  return CUBLOX_OK;
}

int cublox_grid_check(cublox_grid *g, uint32_t *error_word) {
  if (!g || !error_word) return fail(CUBLOX_ERR_INVALID, "null argument");
  CK(cudaMemcpyAsync(error_word, g->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                     g->stream));
  CK(cudaMemsetAsync(g->d_err, 0, sizeof(uint32_t), g->stream));
  CK(cudaStreamSynchronize(g->stream));
  return CUBLOX_OK;
}

}  // extern "C"

// Allocation-free scan integration (cublox_integrate_noalloc).
//
// For callers that may not allocate device memory once they are running:
// a robot's real-time mapping loop that reserves all GPU memory at start-up
// (a cudaMalloc there can block behind other work and blow the cycle's time
// budget), or code that runs inside a host framework which hands it only a
// stream and buffers it owns (an inference-engine plugin's enqueue step, a
// pooled multi-tenant server).  Such a caller owns the map buffers and the
// points; this entry point owns nothing but a fixed scratch area for
// sorting the rays by direction, which lives in a file-scope __device__
// array (every GPU that loads the library holds it until the process exits).
//
// The scratch is shared by every call on a device and keeps whatever the
// last call left in it.  The direction histogram is cleared at the start of
// each call; every other scratch word is fully overwritten before it is
// read.  Calls whose GPU work overlaps (different streams, or different host
// threads, at the same time) race on the scratch and must not be issued.
//
// The direction-binned walk and the counter sweep used here have no
// device-side check that can fail (every index they form is in range by
// construction), so this entry point reports no device error word: the
// kernels are given none (RayParams::err is null, and neither kernel
// dereferences it).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/cublox_b200.h"
#include "exact_fp.cuh"
#include "kernels.cuh"

using namespace cublox_b200;

namespace {

constexpr int kMaxPoints = CUBLOX_NOALLOC_MAX_POINTS;
constexpr int kBinsWords = 4096;  // direction bins (binned_bins())
// Layout: bins[kMaxPoints] | hist[kBinsWords] | cursor[kBinsWords] |
//         sorted[3 * kMaxPoints] (16-byte aligned)
constexpr size_t kOffHist = sizeof(int) * kMaxPoints;
constexpr size_t kOffCursor = kOffHist + sizeof(int) * kBinsWords;
constexpr size_t kOffSorted = kOffCursor + sizeof(int) * kBinsWords;
static_assert(kOffSorted % 16 == 0, "sorted points must start on a 16-byte boundary");
constexpr size_t kScratchBytes = kOffSorted + sizeof(float) * 3 * kMaxPoints;

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
constexpr int kMaxDevices = 64;
unsigned char *g_scratch_ptr[kMaxDevices] = {};

thread_local std::string g_noalloc_err;

int noalloc_fail(int code, const std::string &msg) {
  g_noalloc_err = msg;
  return code;
}

}  // namespace

extern "C" {

const char *cublox_noalloc_last_error(void) { return g_noalloc_err.c_str(); }

int cublox_integrate_noalloc(const cublox_map_view *map, const float *xyz_soa, int n,
                             const float sensor_origin[3], void *stream) {
  if (!map || !sensor_origin || !map->occ || !map->cnt || !map->hit)
    return noalloc_fail(CUBLOX_ERR_INVALID, "cublox_integrate_noalloc: null argument");
  if (n < 0 || n > kMaxPoints)
    return noalloc_fail(CUBLOX_ERR_INVALID,
                        "cublox_integrate_noalloc: " + std::to_string(n) +
                            " points; this entry point takes at most " +
                            std::to_string(kMaxPoints) + " per call");
  if (n > 0 && !xyz_soa)
    return noalloc_fail(CUBLOX_ERR_INVALID, "cublox_integrate_noalloc: null points");
  if (!(map->resolution > 0.0f))
    return noalloc_fail(CUBLOX_ERR_INVALID, "cublox_integrate_noalloc: resolution must be > 0");
  // 2 * half + 1 per axis and their product, in 64-bit arithmetic: every
  // factor is checked against int32 before the next multiplication, so no
  // intermediate can overflow (Grid.cpp:33, :44-50).
  int64_t vnum = 1;
  int mapsz[3];
  for (int a = 0; a < 3; ++a) {
    if (map->half_map_size[a] < 0)
      return noalloc_fail(CUBLOX_ERR_INVALID, "cublox_integrate_noalloc: negative half size");
    const int64_t ms = 2 * static_cast<int64_t>(map->half_map_size[a]) + 1;
    if (ms > 2147483647 || vnum * ms > 2147483647)
      return noalloc_fail(CUBLOX_ERR_RANGE, "cublox_integrate_noalloc: voxel count above int32");
    mapsz[a] = static_cast<int>(ms);
    vnum *= ms;
  }
  if (n == 0) return CUBLOX_OK;

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return noalloc_fail(CUBLOX_ERR_CUDA, "cublox_integrate_noalloc: no current device");
  unsigned char *base = nullptr;
  {
    // First call on this device: the scratch array's device address.  In
    // host code the array's name is only a host-side stand-in, so the
    // kernels must be given this address instead.
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {
      void *ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess) {
        cudaGetLastError();
        return noalloc_fail(CUBLOX_ERR_CUDA, std::string("cublox_integrate_noalloc: "
                                                         "cudaGetSymbolAddress: ") +
                                                 cudaGetErrorString(e));
      }
      g_scratch_ptr[dev] = static_cast<unsigned char *>(ptr);
    }
    base = g_scratch_ptr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  RayParams p{};
  p.x = xyz_soa;
  p.y = xyz_soa + n;
  p.z = xyz_soa + 2 * static_cast<size_t>(n);
  p.n = n;
  p.stride = 1;
  const float res = map->resolution;
  for (int a = 0; a < 3; ++a) {
    p.o[a] = sensor_origin[a];
    p.win[a] = map->origin_index[a];
    p.half[a] = map->half_map_size[a];
    p.map[a] = mapsz[a];
  }
  p.res = res;
  p.inv = 1.0f / res;
  p.max_range = map->max_range;
  p.vnum = static_cast<int>(vnum);
  p.ctr = map->origin_at_center ? 1 : 0;
  p.fp = kFpPinned;
  p.cnt = map->cnt;
  p.hit = map->hit;
  p.stats = nullptr;
  p.err = nullptr;  // no check on this path can fail (file comment)
  // the caller's arrays are in the reference's hash order, and have no line
  // flags: the fold below sweeps every counter
  p.lay.bs[0] = mapsz[1] * mapsz[2];
  p.lay.bs[1] = mapsz[2];
  p.lay.bs[2] = 1;
  p.dirty = nullptr;

  BinnedScratch b{reinterpret_cast<int *>(base), reinterpret_cast<int *>(base + kOffHist),
                  reinterpret_cast<int *>(base + kOffCursor),
                  reinterpret_cast<float *>(base + kOffSorted)};
  // The direction histogram must start at zero; the sort clears it.
  launch_raycast_binned(p, b, 32, false, true, s);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return noalloc_fail(CUBLOX_ERR_CUDA, std::string("cublox_integrate_noalloc: raycast: ") +
                                             cudaGetErrorString(e));
  ApplyParams a{};
  a.occ = map->occ;
  a.cnt = map->cnt;
  a.hit = map->hit;
  a.vnum = p.vnum;
  a.l_hit = map->l_hit;
  a.l_miss = map->l_miss;
  a.l_min = map->l_min;
  a.l_max = map->l_max;
  a.l_unknown = 0.0f;
  a.fp = kFpPinned;
  a.stats = nullptr;
  a.variant = 1;
  launch_apply(a, s);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return noalloc_fail(CUBLOX_ERR_CUDA, std::string("cublox_integrate_noalloc: fold: ") +
                                             cudaGetErrorString(e));
  return CUBLOX_OK;
}

}  // extern "C"

// Sparse copies of a map's stored log-odds between the device and a pinned
// host snapshot, for the served form's evictions: only the 32-voxel lines
// that hold a non-zero stored value cross the bus (a map that a robot has
// seen part of is mostly unknown, stored as 0).
//
// Snapshot layout (pinned host memory, written and read by the kernels
// through its device-visible address):
//   [0, 16)                  int32 count of packed lines (then padding)
//   [16, 16 + 4 nlines)      int32 line index of each packed line
//   [data, data + 4 nalloc)  128 bytes per packed line, in index order
// with data = 16 + 4 nlines rounded up to 128 bytes.  Lines are packed in
// the order warps find them; the index says where each goes back.
#include <cuda_runtime.h>

#include <cstdint>

#include "grid_internal.hpp"
#include "kernels.cuh"

namespace cublox_b200 {

namespace {

constexpr size_t kSnapIndex = 16;

size_t data_offset(int64_t nlines) {
  return (kSnapIndex + 4 * static_cast<size_t>(nlines) + 127) & ~static_cast<size_t>(127);
}

int swap_grid(int64_t nlines) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (nlines + 7) / 8;  // 8 warps a CTA, a line a warp at least
  const int64_t cap = static_cast<int64_t>(sms > 0 ? sms : 148) * 8;
  return static_cast<int>(want < 1 ? 1 : (want < cap ? want : cap));
}

// Warp per line: a line with any non-zero bit pattern (so -0.0 counts) takes
// the next slot and is written, 128 bytes, to the snapshot.
__global__ void __launch_bounds__(256) pack_lines_kernel(const float *occ, int64_t nlines,
                                                         uint8_t *snap, size_t data_at,
                                                         int *count) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  int *idx = reinterpret_cast<int *>(snap + kSnapIndex);
  float *data = reinterpret_cast<float *>(snap + data_at);
  for (int64_t l = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; l < nlines;
       l += warps) {
    const float v = occ[l * 32 + lane];
    if (!__ballot_sync(0xffffffffu, __float_as_uint(v) != 0u)) continue;
    int slot = 0;
    if (lane == 0) slot = atomicAdd(count, 1);
    slot = __shfl_sync(0xffffffffu, slot, 0);
    data[static_cast<int64_t>(slot) * 32 + lane] = v;
    if (lane == 0) idx[slot] = static_cast<int>(l);
  }
}

// Warp per packed line: back to its place in the (zeroed) array.
__global__ void __launch_bounds__(256) unpack_lines_kernel(const uint8_t *snap, int64_t nlines,
                                                           size_t data_at, float *occ) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  int64_t n = *reinterpret_cast<const volatile int *>(snap);
  if (n > nlines) n = nlines;
  const int *idx = reinterpret_cast<const int *>(snap + kSnapIndex);
  const float *data = reinterpret_cast<const float *>(snap + data_at);
  for (int64_t s = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; s < n;
       s += warps) {
    const int l = idx[s];
    if (l < 0 || l >= nlines) continue;
    occ[static_cast<int64_t>(l) * 32 + lane] = data[s * 32 + lane];
  }
}

}  // namespace

size_t detail::packed_snapshot_bytes(int64_t nalloc) {
  return data_offset(nalloc >> kLineShift) + 4 * static_cast<size_t>(nalloc);
}

cudaError_t detail::launch_pack(const float *occ, int64_t nalloc, void *snap, int *d_count,
                                cudaStream_t s) {
  const int64_t nlines = nalloc >> kLineShift;
  cudaError_t e = cudaMemsetAsync(d_count, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  pack_lines_kernel<<<swap_grid(nlines), 256, 0, s>>>(occ, nlines, static_cast<uint8_t *>(snap),
                                                      data_offset(nlines), d_count);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  return cudaMemcpyAsync(snap, d_count, sizeof(int), cudaMemcpyDeviceToHost, s);
}

cudaError_t detail::launch_unpack(const void *snap, int64_t nalloc, float *occ, cudaStream_t s) {
  const int64_t nlines = nalloc >> kLineShift;
  cudaError_t e = cudaMemsetAsync(occ, 0, sizeof(float) * static_cast<size_t>(nalloc), s);
  if (e != cudaSuccess) return e;
  unpack_lines_kernel<<<swap_grid(nlines), 256, 0, s>>>(static_cast<const uint8_t *>(snap),
                                                        nlines, data_offset(nlines), occ);
  return cudaGetLastError();
}

void detail::unpack_on_host(const void *snap, int64_t nalloc, float *occ) {
  const int64_t nlines = nalloc >> kLineShift;
  const uint8_t *b = static_cast<const uint8_t *>(snap);
  int64_t n = *reinterpret_cast<const int *>(b);
  if (n > nlines) n = nlines;
  const int *idx = reinterpret_cast<const int *>(b + kSnapIndex);
  const float *data = reinterpret_cast<const float *>(b + data_offset(nlines));
  for (int64_t i = 0; i < nalloc; ++i) occ[i] = 0.0f;
  for (int64_t s = 0; s < n; ++s) {
    const int l = idx[s];
    if (l < 0 || l >= nlines) continue;
    for (int k = 0; k < 32; ++k) occ[static_cast<int64_t>(l) * 32 + k] = data[s * 32 + k];
  }
}

}  // namespace cublox_b200

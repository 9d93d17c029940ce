// Peak throughput of the walk's memory operation: 32-bit reductions
// (RED.ADD, an atomicAdd whose result is unused) to distinct addresses.
// It is the denominator of the walk's L2-atomic roofline
// (cublox_probe_red_rate).
//
// Each thread adds 1 to `ops` words of a buffer of `words` words, one
// after another along a pseudo-random walk through the buffer (a 32-bit
// LCG per thread, so addresses are spread over the buffer and, across the
// GPU, distinct), with no dependence between its operations: like the
// walk, a thread never waits for an atomic's result.  A buffer that fits in
// L2 measures the L2's atomic units; a larger one adds the DRAM misses.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/cublox_b200.h"
#include "grid_internal.hpp"

namespace {

__global__ void __launch_bounds__(256) red_probe_kernel(uint32_t *buf, uint32_t mask, int ops) {
  uint32_t x = (blockIdx.x * blockDim.x + threadIdx.x) * 2654435761u + 12345u;
#pragma unroll 8
  for (int k = 0; k < ops; ++k) {
    x = x * 1664525u + 1013904223u;
    atomicAdd(buf + (x & mask), 1u);
  }
}

}  // namespace

extern "C" int cublox_probe_red_rate(int64_t buffer_bytes, int64_t total_ops, void *stream,
                                     double *ops_per_s) {
  using cublox_b200::detail::fail;
  if (!ops_per_s || buffer_bytes < 4096 || total_ops <= 0)
    return fail(CUBLOX_ERR_INVALID, "probe_red_rate: bad argument");
  *ops_per_s = 0.0;
  // a power-of-two number of words, at most buffer_bytes
  int64_t words = 1;
  while (words * 2 * 4 <= buffer_bytes && words < (int64_t(1) << 31)) words *= 2;
  uint32_t *buf = nullptr;
  if (cublox_b200::detail::dmalloc(&buf, static_cast<size_t>(words) * 4) != cudaSuccess) {
    cudaGetLastError();
    return fail(CUBLOX_ERR_NOMEM, "probe_red_rate: buffer allocation failed");
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int block = 256, grid = sms * 8;
  const int64_t threads = static_cast<int64_t>(grid) * block;
  const int ops = static_cast<int>((total_ops + threads - 1) / threads);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  if (e == cudaSuccess) e = cudaMemsetAsync(buf, 0, static_cast<size_t>(words) * 4, s);
  const uint32_t mask = static_cast<uint32_t>(words - 1);
  if (e == cudaSuccess) {
    red_probe_kernel<<<grid, block, 0, s>>>(buf, mask, ops);  // warm-up
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(e0, s);
  if (e == cudaSuccess) {
    red_probe_kernel<<<grid, block, 0, s>>>(buf, mask, ops);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(e1, s);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  float ms = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaStreamSynchronize(s);
  cublox_b200::detail::dfree(buf);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(CUBLOX_ERR_CUDA, std::string("probe_red_rate: ") + cudaGetErrorString(e));
  }
  *ops_per_s = static_cast<double>(threads) * ops / (ms * 1e-3);
  return CUBLOX_OK;
}

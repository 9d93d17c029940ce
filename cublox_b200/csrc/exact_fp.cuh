// Exact FP32 restatement of the reference's per-ray and per-voxel arithmetic.
//
// The library is compiled with -fmad=false, so no multiply-add is fused
// implicitly; the sites where the reference's sm_100a build fuses one are
// spelled out with __fmaf_rn and selected by `fp_mode` (same bit layout as
// the oracle's ORC_FP_* selectors).  Division and square root are the
// correctly rounded forms the reference gets from nvcc's defaults
// (-prec-div=true, -prec-sqrt=true).
#pragma once

#include <cstdint>

namespace cublox_b200 {

// fp_mode bit fields
constexpr unsigned kSosPlain = 0;  // (x*x + y*y) + z*z
constexpr unsigned kSosFyFz = 1;   // fma(z,z, fma(y,y, x*x))
constexpr unsigned kSosFxFz = 2;   // fma(z,z, fma(x,x, y*y))
constexpr unsigned kSosPFz = 3;    // fma(z,z, x*x + y*y)
constexpr unsigned kSosFyP = 4;    // fma(y,y, x*x) + z*z
constexpr unsigned kSosFxP = 5;    // fma(x,x, y*y) + z*z
constexpr unsigned kFpRaySosShift = 0;
constexpr unsigned kFpClipFma = 1u << 3;    // kernels.cu:60-62
constexpr unsigned kFpBoundFma = 1u << 4;   // kernels.cu:89-100
constexpr unsigned kFpCenterFma = 1u << 5;  // utils.cuh:27-29
constexpr unsigned kFpMissFma = 1u << 6;    // kernels.cu:188
constexpr unsigned kFpHitFma = 1u << 7;     // kernels.cu:189
constexpr unsigned kFpRecSosShift = 8;      // kernels.cu:326-331
constexpr unsigned kFpFetchSosShift = 11;   // kernels.cu:532-535
constexpr unsigned kFpFetchDFma = 1u << 14; // kernels.cu:529-534

// The contraction pattern of the reference's own sm_100a release build,
// pinned black-box: sums of squares fma(z,z, fma(x,x, y*y)); apply terms
// fused; clip point, boundary distance and fetch offset not fused.  Centre
// binning reads the same fused or not except at exact ties of p*inv.
constexpr unsigned kFpPinned =
    (kSosFxFz << kFpRaySosShift) | kFpCenterFma | kFpMissFma | kFpHitFma |
    (kSosFxFz << kFpRecSosShift) | (kSosFxFz << kFpFetchSosShift);

#if defined(__CUDACC__)
#define CBX_HD __host__ __device__ __forceinline__
#else
#define CBX_HD inline
#endif

#if defined(__CUDA_ARCH__)
CBX_HD float fmul(float a, float b) { return __fmul_rn(a, b); }
CBX_HD float fadd(float a, float b) { return __fadd_rn(a, b); }
CBX_HD float fsub(float a, float b) { return __fsub_rn(a, b); }
CBX_HD float ffma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
CBX_HD float fdiv(float a, float b) { return __fdiv_rn(a, b); }
CBX_HD float fsqrt(float a) { return __fsqrt_rn(a); }
CBX_HD float ffloor(float a) { return floorf(a); }
// static_cast<int>(float): cvt.rzi.s32.f32 (truncating, saturating, NaN -> 0)
CBX_HD int f2i(float v) { return static_cast<int>(v); }
#else
// Host twins (compiled with -ffp-contract=off).
CBX_HD float fmul(float a, float b) { return a * b; }
CBX_HD float fadd(float a, float b) { return a + b; }
CBX_HD float fsub(float a, float b) { return a - b; }
CBX_HD float ffma(float a, float b, float c) { return __builtin_fmaf(a, b, c); }
CBX_HD float fdiv(float a, float b) { return a / b; }
CBX_HD float fsqrt(float a) { return __builtin_sqrtf(a); }
CBX_HD float ffloor(float a) { return __builtin_floorf(a); }
CBX_HD int f2i(float v) {
  if (v != v) return 0;
  if (v >= 2147483648.0f) return 2147483647;
  if (v < -2147483648.0f) return (-2147483647 - 1);
  return static_cast<int>(v);
}
#endif

CBX_HD float sos(float x, float y, float z, unsigned shape) {
  switch (shape) {
  case kSosFyFz:
    return ffma(z, z, ffma(y, y, fmul(x, x)));
  case kSosFxFz:
    return ffma(z, z, ffma(x, x, fmul(y, y)));
  case kSosPFz:
    return ffma(z, z, fadd(fmul(x, x), fmul(y, y)));
  case kSosFyP:
    return fadd(ffma(y, y, fmul(x, x)), fmul(z, z));
  case kSosFxP:
    return fadd(ffma(x, x, fmul(y, y)), fmul(z, z));
  default:
    return fadd(fadd(fmul(x, x), fmul(y, y)), fmul(z, z));
  }
}

// posToGlobalIndex as the device computes it (utils.cuh:24-32).
CBX_HD int pos_to_global_dev(float p, float inv, bool ctr, unsigned fp) {
  if (ctr) {
    const float half = p < 0.0f ? -0.5f : 0.5f;
    const float v =
        (fp & kFpCenterFma) ? ffma(p, inv, half) : fadd(fmul(p, inv), half);
    return f2i(v);
  }
  return f2i(ffloor(fmul(p, inv)));
}

// globalIndexToLocalIndex (utils.cuh:60-70): C remainder wrapped to [-h, h].
CBX_HD int global_to_local(int g, int map, int half) {
  int l = g % map;
  if (l > half) {
    l -= map;
  } else if (l < -half) {
    l += map;
  }
  return l;
}

}  // namespace cublox_b200

// Exact jump-ahead through a rounded running sum s_{j+1} = fl(s_j + d).
//
// The Amanatides–Woo walk keeps, per axis, tM <- fl(tM + tD) (kernels.cu:
// 123-135).  Splitting one ray between several lanes needs the walk state
// at an arbitrary point, i.e. s_j for large j, bit for bit.  Summing j times
// is what the split avoids; instead:
//
// Within one binade [2^e, 2^(e+1)) every float is a multiple of the ulp u,
// so for s_j in the binade with s_j + d < 2^(e+1):
//   fl(s_j + d) = s_j + (d rounded to a multiple of u),
// with ties to even.  The increment is therefore the same for every step
// after the first one in a binade (a tie can flip it once, after which the
// sum's parity is fixed), and the whole stretch is an arithmetic progression
// whose terms are exact in FP32.  Only the step that leaves the binade (or
// one starting at or below zero) needs a real rounded add.  A query costs
// O(number of binades crossed) adds and two integer divisions per binade.
//
// Everything here is __host__ __device__ and plain IEEE arithmetic, so the
// CPU test (tests/cpp/test_dda_jump.cpp) checks the same code the kernels run.
#pragma once

#include <cstdint>

#include "exact_fp.cuh"

namespace cublox_b200 {

struct JumpResult {
  int64_t j;  // index reached
  float s;    // s_j
  bool ok;    // false: the sum stalls (d below half an ulp) before the target
};

CBX_HD int f32_exponent(float v) {  // unbiased exponent of a positive normal
#if defined(__CUDA_ARCH__)
  return ((__float_as_uint(v) >> 23) & 0xff) - 127;
#else
  uint32_t b;
  __builtin_memcpy(&b, &v, 4);
  return static_cast<int>((b >> 23) & 0xff) - 127;
#endif
}

CBX_HD bool f32_is_normal_pos(float v) {
  return v >= 1.17549435e-38f && v < 3.4028234e38f;
}

// Exact 2^k as float for k in [-126, 127].
CBX_HD float f32_pow2(int k) {
  const uint32_t b = static_cast<uint32_t>(k + 127) << 23;
#if defined(__CUDA_ARCH__)
  return __uint_as_float(b);
#else
  float v;
  __builtin_memcpy(&v, &b, 4);
  return v;
#endif
}

// Integer helpers: floor/ceil of an exact float that holds an integer or a
// value with few fractional bits, and floor division with a positive divisor.
// floor(a / b) for b > 0 and |a| < 2^27: a rounded float quotient, then an
// exact integer correction (the estimate is off by a few units at most).
CBX_HD int32_t floor_div_pos(int32_t a, int32_t b) {
  int32_t q = static_cast<int32_t>(ffloor(fdiv(static_cast<float>(a), static_cast<float>(b))));
  while (static_cast<int64_t>(q) * b > a) --q;
  while (static_cast<int64_t>(q + 1) * b <= a) ++q;
  return q;
}

CBX_HD float f32_scale(float v, int k) {  // v * 2^k, exact while normal
  return fmul(v, f32_pow2(k));
}

// Smallest j >= 0 with s_j >= tau (the sequence starts at s_0 = s0), and s_j.
// Also stops at j == jmax (returning s_jmax) so callers can bound work.
// d must be > 0 and finite; s0 may be any non-NaN value.
//
// Inside a binade of ulp u every quantity is an exact integer multiple of u
// except d; with F = floor(d/u), a step from v = V*u stays on the grid iff
//   v > 0:  V + F <= 2^24 - 1         (the sum stays below 2^(e+1))
//   v < 0:  V + F <= -2^23 - [d/u not an integer]   (magnitude >= 2^e)
// so the number of on-grid steps and the first term >= tau are integer
// divisions.
// The on-grid run of the sum inside one binade that a query ended in:
// positions S + k*D (in ulps u = 2^(e-23)) for k = 0..m, the value at
// position S being s at index j, each step adding delta = D*u exactly.  A
// later query with a larger tau that lands in the same run needs one
// integer division (stretch_query), not a walk.
struct JumpStretch {
  int64_t j;
  float s, delta;
  int32_t S, D, m;
  int e;
  bool valid;
};

CBX_HD JumpResult first_at_or_above(float s0, float d, float tau, int64_t jmax,
                                    JumpStretch *stretch = nullptr) {
  JumpResult r{0, s0, true};
  for (int guard = 0; guard < 4096; ++guard) {
    if (r.s >= tau || r.j >= jmax) return r;
    const float s1 = fadd(r.s, d);
    if (s1 == r.s) {  // stalled: never reaches tau
      r.ok = false;
      return r;
    }
    r.j += 1;
    r.s = s1;
    if (r.s >= tau || r.j >= jmax) return r;
    const float mag = r.s < 0.0f ? -r.s : r.s;
    if (!f32_is_normal_pos(mag)) continue;  // zero, subnormal or infinite
    const bool neg = r.s < 0.0f;
    const int e = f32_exponent(mag);
    if (e > 100 || e < -100) continue;
    const float Ddf = f32_scale(d, 23 - e);  // d/u, exact
    if (!(Ddf < 16777216.0f)) continue;     // d spans the binade: real steps
    const float Ff = ffloor(Ddf);
    const int32_t F = static_cast<int32_t>(Ff);
    const int32_t frac = (Ddf != Ff) ? 1 : 0;
    const int32_t lim = neg ? (-8388608 - frac - F) : (16777215 - F);
    // A second on-grid step: if d sits exactly halfway between two ulp
    // multiples, it rounds the sum to an even multiple, after which every
    // on-grid step rounds the same way.
    int32_t S = static_cast<int32_t>(f32_scale(r.s, 23 - e));
    if (S > lim) continue;
    const float s2 = fadd(r.s, d);
    r.j += 1;
    r.s = s2;
    if (r.s >= tau || r.j >= jmax) return r;
    S = static_cast<int32_t>(f32_scale(r.s, 23 - e));
    if (S > lim) continue;
    const float s3 = fadd(r.s, d);
    const float delta = fsub(s3, r.s);  // exact: both on the ulp grid
    if (!(delta > 0.0f)) continue;
    const int32_t D = static_cast<int32_t>(f32_scale(delta, 23 - e));
    // m = number of on-grid steps from here = #{k >= 0 : S + k D <= lim}
    const int32_t m = floor_div_pos(lim - S, D) + 1;
    if (m <= 0) continue;
    // First k with S + k D >= ceil(tau/u); anything past the stretch is m+1.
    int32_t kt = m + 1;
    if (tau < 3.4028234e38f) {
      const float Tf = f32_scale(tau, 23 - e);
      const float hi = static_cast<float>(S) + static_cast<float>(m) * static_cast<float>(D);
      if (Tf <= static_cast<float>(S)) {
        kt = 0;
      } else if (Tf <= hi) {
        const int32_t T = static_cast<int32_t>(ceilf(Tf));
        kt = -floor_div_pos(-(T - S), D);  // ceil((T - S) / D)
      }
    }
    if (stretch && kt <= m) *stretch = JumpStretch{r.j, r.s, delta, S, D, m, e, true};
    int64_t k = kt < m ? kt : m;
    if (jmax - r.j < k) k = jmax - r.j;
    r.s = fadd(r.s, fmul(static_cast<float>(k), delta));  // exact
    r.j += k;
  }
  r.ok = false;
  return r;
}

// The first j >= the stretch's own index with s_j >= tau, capped at jmax,
// if tau lies inside the stretch (the same arithmetic as the jump in
// first_at_or_above); false if it lies beyond, or no stretch is known.
// The caller has checked that its current s_j is still below tau.
CBX_HD bool stretch_query(const JumpStretch &st, float tau, int64_t jmax, JumpResult &out) {
  if (!st.valid || !(tau < 3.4028234e38f)) return false;
  const float Tf = f32_scale(tau, 23 - st.e);
  const float hi = static_cast<float>(st.S) + static_cast<float>(st.m) * static_cast<float>(st.D);
  if (!(Tf <= hi)) return false;
  int32_t kt = 0;
  if (Tf > static_cast<float>(st.S)) {
    const int32_t T = static_cast<int32_t>(ceilf(Tf));
    kt = -floor_div_pos(-(T - st.S), st.D);  // ceil((T - S) / D)
  }
  if (kt > st.m) return false;  // hi rounded past the run's end
  int64_t k = kt;
  if (jmax - st.j < k) k = jmax - st.j;
  out.j = st.j + k;
  out.s = fadd(st.s, fmul(static_cast<float>(k), st.delta));  // exact
  out.ok = true;
  return true;
}

// Advance a position (j, s = s_j) of the sequence to the first index with
// s_j >= tau, capped at jmax, for queries with growing tau: a query that
// lands in the stretch the previous one ended in costs one division, any
// other walks on with first_at_or_above and records its stretch in st.
CBX_HD JumpResult advance_to(int64_t j, float s, float d, float tau, int64_t jmax,
                             JumpStretch &st) {
  JumpResult r{j, s, true};
  if (s >= tau || j >= jmax) return r;
  if (st.valid) {
    if (stretch_query(st, tau, jmax, r)) return r;
    // tau lies past the run (its end S + m*D is exact in FP32: |S + m*D| <=
    // 2^24): continue from the run's last on-grid position.
    int64_t k = st.m;
    if (jmax - st.j < k) k = jmax - st.j;
    if (st.j + k > j) {
      r.j = st.j + k;
      r.s = fadd(st.s, fmul(static_cast<float>(k), st.delta));  // exact
      if (r.s >= tau || r.j >= jmax) return r;
      j = r.j;
      s = r.s;
    }
  }
  st.valid = false;
  r = first_at_or_above(s, d, tau, jmax - j, &st);
  r.j += j;
  if (st.valid) st.j += j;
  return r;
}

// s_j for a given j (jump by index).
CBX_HD JumpResult value_at(float s0, float d, int64_t j) {
  return first_at_or_above(s0, d, 3.4028235e38f * 2.0f, j);
}

}  // namespace cublox_b200

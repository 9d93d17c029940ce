// CPU check of the exact jump-ahead (cublox_b200/csrc/dda_jump.cuh) against
// step-by-step rounded summation.  Built with -ffp-contract=off.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <random>

#include "../../cublox_b200/csrc/dda_jump.cuh"

using namespace cublox_b200;

int main(int argc, char **argv) {
  const int cases = argc > 1 ? std::atoi(argv[1]) : 20000;
  std::mt19937_64 rng(7);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  long fails = 0, checks = 0;
  for (int c = 0; c < cases; ++c) {
    // tM starts near the sensor (possibly slightly negative); tD = res/|u|.
    float s0;
    switch (c % 4) {
      case 0: s0 = static_cast<float>(U(rng) * 0.2 - 0.01); break;
      case 1: s0 = static_cast<float>(U(rng) * 1e-6 - 5e-7); break;
      case 2: s0 = static_cast<float>(U(rng) * 5.0); break;
      default: s0 = 0.0f; break;
    }
    float d = static_cast<float>(0.05 / std::max(1e-4, U(rng)));
    if (c % 7 == 0) {  // d exactly halfway between ulp multiples of a binade
      const int e = static_cast<int>(U(rng) * 6) - 3;
      d = std::ldexp(static_cast<float>(1 + 2 * static_cast<int>(U(rng) * 1000)), e - 24);
    }
    if (c % 11 == 0) d = static_cast<float>(U(rng) * 1e-3 + 1e-5);
    const int n = 1 + static_cast<int>(U(rng) * 20000);
    float s = s0;
    float *seq = new float[n + 1];
    seq[0] = s;
    for (int j = 1; j <= n; ++j) {
      s = s + d;
      seq[j] = s;
    }
    for (int q = 0; q < 8; ++q) {
      const int j = static_cast<int>(U(rng) * n);
      const JumpResult r = value_at(s0, d, j);
      ++checks;
      // A stalled sum is reported (ok = false) for the caller to walk it
      // step by step; that is only allowed where it genuinely stalls.
      if (!r.ok && (r.s + d) == r.s && seq[j] == r.s) continue;
      if (!r.ok || r.j != j || r.s != seq[j]) {
        if (fails < 10)
          std::printf("value_at s0=%a d=%a j=%d got j=%lld s=%a want %a ok=%d\n", s0, d, j,
                      static_cast<long long>(r.j), r.s, seq[j], r.ok);
        ++fails;
      }
      // tau between / at sequence values
      const float tau = (q & 1) ? seq[j] : std::nextafter(seq[j], -INFINITY);
      const JumpResult t = first_at_or_above(s0, d, tau, n);
      if (!t.ok && (t.s + d) == t.s) continue;
      int want = 0;
      while (want <= n && seq[want] < tau) ++want;
      ++checks;
      if (want <= n && (t.j != want || t.s != seq[want])) {
        if (fails < 10)
          std::printf("first_at_or_above s0=%a d=%a tau=%a got %lld want %d\n", s0, d, tau,
                      static_cast<long long>(t.j), want);
        ++fails;
      }
    }
    // growing taus through one position, as the split-walk planner asks
    // them (advance_to and its stretch cache)
    {
      float taus[16];
      for (int q = 0; q < 16; ++q) {
        const int j = static_cast<int>(U(rng) * n);
        taus[q] = (q % 3 == 0) ? seq[j]
                : (q % 3 == 1) ? std::nextafter(seq[j], -INFINITY)
                               : static_cast<float>(seq[0] + U(rng) * (seq[n] - seq[0]));
      }
      std::sort(taus, taus + 16);
      const int64_t jmax = (c % 5 == 0) ? n / 2 : n;
      int64_t jc = 0;
      float sc = s0;
      JumpStretch st{};
      st.valid = false;
      for (int q = 0; q < 16; ++q) {
        const JumpResult a = advance_to(jc, sc, d, taus[q], jmax, st);
        if (!a.ok && (a.s + d) == a.s) break;  // stalled sum: left to the caller
        int want = 0;
        while (want < jmax && seq[want] < taus[q]) ++want;
        ++checks;
        if (!a.ok || a.j != want || a.s != seq[want]) {
          if (fails < 10)
            std::printf("advance_to s0=%a d=%a tau=%a got %lld %a want %d %a\n", s0, d,
                        taus[q], static_cast<long long>(a.j), a.s, want, seq[want]);
          ++fails;
        }
        jc = a.j;
        sc = a.s;
      }
    }
    delete[] seq;
  }
  std::printf("dda_jump: %ld checks, %ld failures\n", checks, fails);
  return fails ? 1 : 0;
}

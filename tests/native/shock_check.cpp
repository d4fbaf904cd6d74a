// Host check of quotient_exceeds (fluid_physics.cuh): the screened test
// RN(a / m) > t against the plain IEEE division, compiled with g++ without
// contraction.  Cases: random magnitudes; a = t m (1 + k 2^-52) for small k;
// the doubles next to both screen bounds RN(RN(t m) (1 +- 2^-50)); extreme
// exponents; zeros, infinities and NaNs.  Prints "cases mismatches".
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <random>

#define __device__
#define __host__
#define __forceinline__ inline
#define __noinline__
static inline double __fma_rn(double a, double b, double c) { return std::fma(a, b, c); }
template <class T>
static inline T __ldg(const T* p) {
  return *p;
}
static inline long long __double_as_longlong(double x) {
  long long u;
  std::memcpy(&u, &x, 8);
  return u;
}
static inline double __longlong_as_double(long long u) {
  double x;
  std::memcpy(&x, &u, 8);
  return x;
}
using std::copysign;
using std::fabs;
using std::fmin;
using std::log;
using std::pow;
using std::sqrt;

#include "fluid_physics.cuh"

static long long n_cases = 0, n_bad = 0;

static void check(double a, double m, double t) {
  volatile double q = a / m;
  const bool want = q > t;
  const bool got = gfx::quotient_exceeds(a, m, t);
  ++n_cases;
  if (want != got) {
    ++n_bad;
    if (n_bad <= 10) std::printf("# mismatch a=%a m=%a t=%a\n", a, m, t);
  }
}

// a and its neighbours within k ulps
static void around(double a, double m, double t, int k) {
  double lo = a, hi = a;
  check(a, m, t);
  for (int i = 0; i < k; ++i) {
    lo = std::nextafter(lo, 0.0);
    hi = std::nextafter(hi, std::numeric_limits<double>::infinity());
    check(lo, m, t);
    check(hi, m, t);
  }
}

int main() {
  std::mt19937_64 rng(20261203);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  const double ts[] = {0.1, 1.0 / 3.0, 0.5, 1.0, 1e-3, 7.25, 1e-300, 1e300, 0x1p-1000, 0x1p-1022,
                       4.9e-324};
  for (double t : ts) {
    for (int s = 0; s < 20000; ++s) {
      // m over many binades; a near t m
      const double m = std::ldexp(0.5 + u(rng), (int)(u(rng) * 600.0) - 300);
      const double p = t * m;
      const int k = (int)(u(rng) * 64.0) - 32;
      around(p * (1.0 + k * 0x1p-52), m, t, 3);
      around(p * (1.0 + 0x1p-50), m, t, 4);
      around(p * (1.0 - 0x1p-50), m, t, 4);
      check(p * std::ldexp(0.5 + u(rng), (int)(u(rng) * 8.0) - 4), m, t);
    }
    // pressures as the shock test forms them
    for (int s = 0; s < 20000; ++s) {
      const double P0 = std::ldexp(0.5 + u(rng), (int)(u(rng) * 40.0) - 20);
      const double P1 = P0 * (1.0 + t * (1.0 + ((int)(u(rng) * 64.0) - 32) * 0x1p-52));
      const double dP = std::fabs(P0 - P1);
      const double pmin = (P0 < P1) ? P0 : P1;
      around(dP, gfx::fmax2(pmin, gfx::kSqrtTiny), t, 2);
    }
  }
  const double inf = std::numeric_limits<double>::infinity();
  const double nan = std::numeric_limits<double>::quiet_NaN();
  const double ms[] = {gfx::kSqrtTiny, 1e-200, 1.0, 1e200, 1.7e308, 0x1p-960, 0x1p960};
  for (double t : ts)
    for (double m : ms) {
      check(0.0, m, t);
      check(inf, m, t);
      check(nan, m, t);
      check(1.7e308, m, t);
      check(4.9e-324, m, t);
      around(t * m, m, t, 8);
    }
  check(1.0, nan, 0.1);
  check(1.0, inf, 0.1);
  std::printf("%lld %lld\n", n_cases, n_bad);
  return 0;
}

// Host check of the pointwise adjoints in adjoint_physics.cuh against central
// finite differences of the forward functions of fluid_physics.cuh, compiled
// with g++ through the shims below (the device intrinsics the forward uses,
// restated on the host).  Prints one line per piece: name, samples, passed,
// worst relative error of the directional derivative.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
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

#include "adjoint_physics.cuh"

using namespace gfx;

static std::mt19937_64 rng(20261207);
static double uni(double a, double b) { return std::uniform_real_distribution<double>(a, b)(rng); }

struct Tally {
  const char* name;
  int n = 0, ok = 0;
  double worst = 0.0;
  void add(double fd, double ad) {
    const double scale = std::fmax(std::fabs(fd), std::fabs(ad)) + 1e-12;
    const double e = std::fabs(fd - ad) / scale;
    ++n;
    if (e < 1e-5) ++ok;
    if (e > worst) worst = e;
  }
  void print() const { std::printf("%s %d %d %.3e\n", name, n, ok, worst); }
};

static Phys phys() {
  Phys ph{};
  ph.gamma = 1.4;
  ph.gm1 = 0.4;
  ph.c_v = 1.0 / (1.0 * 0.4);
  ph.theta = 1.4;
  ph.nmin = 0.0;
  ph.use_limiter = 1;
  return ph;
}

static void random_prim(double* w) {
  w[0] = uni(0.3, 3.0);
  w[1] = uni(-1.5, 1.5);
  w[2] = uni(-1.5, 1.5);
  w[3] = uni(-1.5, 1.5);
  w[4] = uni(0.2, 5.0);
}

template <int D, bool HLLC>
static void check_flux(Tally& t, bool diffusive) {
  const Phys ph = phys();
  double l[5], r[5], dl[5], dr[5], lF[5];
  random_prim(l);
  random_prim(r);
  if (uni(0, 1) < 0.5)  // nearby states: weak waves, both HLLC sides
    for (int q = 0; q < 5; ++q) r[q] = l[q] * (1.0 + uni(-0.2, 0.2));
  for (int q = 0; q < 5; ++q) {
    dl[q] = uni(-1, 1);
    dr[q] = uni(-1, 1);
    lF[q] = uni(-1, 1);
  }
  auto J = [&](double e) {
    double a[5], b[5], F[5];
    for (int q = 0; q < 5; ++q) {
      a[q] = l[q] + e * dl[q];
      b[q] = r[q] + e * dr[q];
    }
    FaceState L, R;
    face_state<5>(a[0], a[1], a[2], a[3], a[4], ph, L);
    face_state<5>(b[0], b[1], b[2], b[3], b[4], ph, R);
    riemann_flux<D, HLLC, 5>(L, R, diffusive, F);
    double s = 0.0;
    for (int u = 0; u < 5; ++u) s += lF[u] * F[u];
    return s;
  };
  const double h = 1e-6;
  const double fd = (J(h) - J(-h)) / (2 * h);
  double ll[5] = {0}, lr[5] = {0};
  flux_adjoint<D, HLLC>(l, r, diffusive, lF, ph, ll, lr);
  double ad = 0.0;
  for (int q = 0; q < 5; ++q) ad += ll[q] * dl[q] + lr[q] * dr[q];
  t.add(fd, ad);
}

static void check_slope(Tally& t, int use_limiter) {
  const double dxl = uni(0.5, 2.0) * 0.01, dxr = uni(0.5, 2.0) * 0.01;
  const double sql = dxl * dxl, sqr = dxr * dxr, cden = dxl * dxr * (dxl + dxr);
  const double rdxl = 1.0 / dxl, rdxr = 1.0 / dxr, rcden = 1.0 / cden;
  double v[3], dv[3];
  for (int i = 0; i < 3; ++i) {
    v[i] = uni(-1, 1);
    dv[i] = uni(-1, 1);
  }
  auto S = [&](double e) {
    return limited_slope(v[0] + e * dv[0], v[1] + e * dv[1], v[2] + e * dv[2], dxl, dxr, sql,
                         sqr, cden, rdxl, rdxr, rcden, 1.4, use_limiter);
  };
  const double h = 1e-7;
  const double fd = (S(h) - S(-h)) / (2 * h);
  int branch;
  const double s0 = limited_slope_branch(v[0], v[1], v[2], dxl, dxr, sql, sqr, cden, rdxl,
                                         rdxr, rcden, 1.4, use_limiter, branch);
  if (s0 != S(0.0)) {  // the branch-recording slope must be the forward's, bit for bit
    t.add(1.0, 0.0);
    return;
  }
  double gl, gr;
  slope_coeffs(branch, sql, sqr, rdxl, rdxr, rcden, 1.4, gl, gr);
  t.add(fd, -gl * dv[0] + (gl - gr) * dv[1] + gr * dv[2]);
}

static void check_c2p(Tally& t) {
  const Phys ph = phys();
  double w[5];
  random_prim(w);
  const double U[5] = {w[0], w[0] * w[1], w[0] * w[2], w[0] * w[3],
                       w[4] + 0.5 * w[0] * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3])};
  double du[5], lw[5];
  for (int q = 0; q < 5; ++q) {
    du[q] = uni(-1, 1);
    lw[q] = uni(-1, 1);
  }
  auto J = [&](double e) {
    Cons c{U[0] + e * du[0], U[1] + e * du[1], U[2] + e * du[2], U[3] + e * du[3],
           U[4] + e * du[4]};
    Prim p;
    cons_to_prim(c, p, ph.nmin);
    return lw[0] * p.N + lw[1] * p.V1 + lw[2] * p.V2 + lw[3] * p.V3 + lw[4] * p.E;
  };
  const double h = 1e-7;
  const double fd = (J(h) - J(-h)) / (2 * h);
  Cons c{U[0], U[1], U[2], U[3], U[4]};
  Prim p;
  cons_to_prim(c, p, ph.nmin);
  const double wp[5] = {p.N, p.V1, p.V2, p.V3, p.E};
  double lu[5];
  c2p_adjoint(wp, lw, ph.nmin, lu);
  double ad = 0.0;
  for (int q = 0; q < 5; ++q) ad += lu[q] * du[q];
  t.add(fd, ad);
}

static void check_final(Tally& t) {
  const Phys ph = phys();
  double w[5];
  random_prim(w);
  const double U[5] = {w[0], w[0] * w[1], w[0] * w[2], w[0] * w[3],
                       w[4] + 0.5 * w[0] * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3])};
  double du[5], lU[6];
  for (int q = 0; q < 5; ++q) du[q] = uni(-1, 1);
  for (int q = 0; q < 6; ++q) lU[q] = uni(-1, 1);
  // J = lU . (D', S', G', DS) with DS = N SB(N, E) of the recovered state
  auto J = [&](double e) {
    Cons c{U[0] + e * du[0], U[1] + e * du[1], U[2] + e * du[2], U[3] + e * du[3],
           U[4] + e * du[4]};
    Prim p;
    cons_to_prim(c, p, ph.nmin);
    double P, CS, SB;
    eos_cell(p.N, p.E, ph, P, CS, &SB);
    return lU[0] * c.D + lU[1] * c.S1 + lU[2] * c.S2 + lU[3] * c.S3 + lU[4] * c.G +
           lU[5] * SB * p.N;
  };
  const double h = 1e-7;
  const double fd = (J(h) - J(-h)) / (2 * h);
  Cons c{U[0], U[1], U[2], U[3], U[4]};
  Prim p;
  cons_to_prim(c, p, ph.nmin);
  const double wp[5] = {p.N, p.V1, p.V2, p.V3, p.E};
  double lz[5];
  final_adjoint(wp, lU, ph, lz);
  double ad = 0.0;
  for (int q = 0; q < 5; ++q) ad += lz[q] * du[q];
  t.add(fd, ad);
}

int main() {
  const int n = 4000;
  Tally hll[3] = {{"flux_hll_x"}, {"flux_hll_y"}, {"flux_hll_z"}};
  Tally hllc[3] = {{"flux_hllc_x"}, {"flux_hllc_y"}, {"flux_hllc_z"}};
  Tally hllcd{"flux_hllc_diffusive_z"};
  Tally sl{"slope_limited"}, su{"slope_unlimited"}, c2p{"c2p"}, fin{"final"};
  for (int i = 0; i < n; ++i) {
    check_flux<0, false>(hll[0], false);
    check_flux<1, false>(hll[1], false);
    check_flux<2, false>(hll[2], false);
    check_flux<0, true>(hllc[0], false);
    check_flux<1, true>(hllc[1], false);
    check_flux<2, true>(hllc[2], false);
    check_flux<2, true>(hllcd, true);
    check_slope(sl, 1);
    check_slope(su, 0);
    check_c2p(c2p);
    check_final(fin);
  }
  for (auto& t : hll) t.print();
  for (auto& t : hllc) t.print();
  hllcd.print();
  sl.print();
  su.print();
  c2p.print();
  fin.print();
  return 0;
}

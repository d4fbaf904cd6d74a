// fluid_physics.cuh -- pointwise FP64 arithmetic of the Fluid_P_I step.
//
// Every expression keeps the operand order of the reference's Fortran so that
// each rounding matches (the library is compiled with --fmad=false).  The
// baryon mass M and every metric entry are exactly 1 on the rectangular chart,
// so the products with them that the reference performs are exact and are
// left out here.
//
// GFX_FAST_MATH = 1 builds the speed variant of the same kernels (compiled
// with --fmad=true): multiplies and adds may fuse, a division by a value with
// a known rounded reciprocal r is the product a r (within 1.5 ulp of the
// quotient, where the exact variant corrects it to the rounded quotient), the
// limiter takes the smallest of those products, and the entropy per baryon is
// c_v (log P - gamma log N) instead of c_v log(P (1/N)^gamma).  Each changes a
// result by a few units in the last place of that operation, far inside the
// 1e-12 per-step bar.  The shock threshold test stays exact in both variants.
#pragma once

#ifndef GFX_FAST_MATH
#define GFX_FAST_MATH 0
#endif

#include <cfloat>
#include <cstdint>
#include <cstring>

namespace gfx {

constexpr double kTiny = DBL_MIN;                      // tiny(0._KDR)
constexpr double kSqrtTiny = 1.4916681462400413e-154;  // sqrt(tiny(0._KDR))
constexpr double kSqrtHuge = 1.3407807929942596e+154;  // sqrt(huge(1._KDR))

struct Phys {
  double gamma;  // AdiabaticIndex
  double gm1;    // AdiabaticIndex - 1
  double c_v;    // SpecificHeatVolume = 1 / (1 * (gamma - 1))
  double theta;  // LimiterParameter
  double nmin;   // BaryonDensityMin
  double accel;  // UniformAcceleration (z)
  double shock_threshold;
  double courant;
  int use_limiter;
  int n_ramp;
  int parabolic;  // ReconstructionType PARABOLIC
};

// Fortran MAX / MIN with gfortran's argument order: the first argument wins ties.
__device__ __forceinline__ double fmax2(double a, double b) { return (b > a) ? b : a; }
__device__ __forceinline__ double fmax3(double a, double b, double c) {
  double r = a;
  if (b > r) r = b;
  if (c > r) r = c;
  return r;
}
__device__ __forceinline__ double fmin3(double a, double b, double c) {
  double r = a;
  if (b < r) r = b;
  if (c < r) r = c;
  return r;
}

// Correctly rounded a / b from r = RN(1 / b), by two Markstein corrections
// (P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Dev. 34(1), 1990): the first correction
// makes the quotient faithful, the second rounds it correctly, each remainder
// a - b q being exact through the fused multiply-add as long as nothing
// underflows or overflows.  markstein() is that straight-line sequence;
// quotient_in_range() tells whether a and the first approximation a r lie in
// the exponent range where it is exact (zero included, whose sign may come out
// flipped: no branch of the step distinguishes the zeros).  Callers evaluate a
// group of independent quotients branch-free and redo the group with the IEEE
// division in the rare case that one of them is out of range.
__device__ __noinline__ double div_ieee(double a, double b) { return a / b; }

__device__ __forceinline__ double markstein(double a, double b, double r) {
#if GFX_FAST_MATH
  (void)b;
  return a * r;
#endif
  const double q0 = a * r;
  const double e0 = __fma_rn(-b, q0, a);
  const double q1 = __fma_rn(e0, r, q0);
  const double e1 = __fma_rn(-b, q1, a);
  return __fma_rn(e1, r, q1);
}

// 1 / b for a normal b: correctly rounded in the exact build; in the speed
// build the hardware's approximate reciprocal (PTX rcp.approx.ftz.f64)
// refined by two Newton-Raphson steps y <- y + y (1 - b y), each a pair of
// fused multiply-adds, which leaves it within about an ulp.
__device__ __forceinline__ double recip(double b) {
#if GFX_FAST_MATH
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  double e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  e = __fma_rn(-b, y, 1.0);
  return __fma_rn(y, e, y);
#else
  return 1.0 / b;
#endif
}

// The sound speed sqrt(gamma P / N) for N > 0 and P > 0 (Apply_EOS_I_E_Kernel,
// Fluid_P_I__Kernel.f90:244-267): as written in the exact build; in the speed
// build a rsqrt(a N) with a = gamma P, one reciprocal square root (CUDA's
// rsqrt, within an ulp) instead of a division and a square root.
__device__ __forceinline__ double sound_speed(double P, double N, const Phys& ph) {
#if GFX_FAST_MATH
  const double a = ph.gamma * P;
  return a * rsqrt(a * N);
#else
  return sqrt(ph.gamma * P / N);
#endif
}

// |x| == 0 or 2^-900 <= |x| < 2^1001 (NaN and infinities fail).
__device__ __forceinline__ bool exp_in_range(double x) {
  const double ax = fabs(x);
  return (ax >= 0x1p-900 && ax < 0x1p1001) || x == 0.0;
}

__device__ __forceinline__ bool quotient_in_range(double a, double r) {
#if GFX_FAST_MATH
  (void)a, (void)r;
  return true;  // the product a r needs no exponent window
#else
  return exp_in_range(a) & exp_in_range(a * r);
#endif
}

// The same window for a divisor of the chart geometry (a width, a centre
// difference, the limiter's central denominator or a cell volume), whose
// rounded reciprocal r lies in [2^-300, 2^300] because every cell width lies
// in [2^-98, 2^98] (checked when a brick is created): then 2^-600 <= |a| <
// 2^700, or a == 0, puts both a and a r inside the window, and one test on
// a suffices.
__device__ __forceinline__ bool geo_quotient_in_range(double a) {
#if GFX_FAST_MATH
  (void)a;
  return true;
#else
  const double ax = fabs(a);
  return (ax >= 0x1p-600 && ax < 0x1p700) || a == 0.0;
#endif
}

__device__ __forceinline__ double div_geo(double a, double b, double r) {
  const double q = markstein(a, b, r);
  return geo_quotient_in_range(a) ? q : div_ieee(a, b);
}

__device__ __forceinline__ double div_rn(double a, double b, double r) {
  const double q = markstein(a, b, r);
  return quotient_in_range(a, r) ? q : div_ieee(a, b);
}

// The limiter exactly as Gradient_Kernel.f90:176-180 writes it, with IEEE
// divisions: the slow path of limited_slope.
__device__ __noinline__ double limited_slope_ieee(double dvl, double dvr, double dxl, double dxr,
                                                  double sql, double sqr, double cden,
                                                  double theta) {
  const double central = (sqr * dvl + sql * dvr) / cden;
  const double s = copysign(0.5, dvl) + copysign(0.5, dvr);
  return s * fmin3(fabs(theta * dvl / dxl), fabs(theta * dvr / dxr), fabs(central));
}

// Generalized-minmod limited slope of one cell, Gradient_Kernel.f90:166-190.
// vm, v0, vp: values at i-1, i, i+1; dxl = X(i) - X(i-1), dxr = X(i+1) - X(i);
// sql = dxl*dxl, sqr = dxr*dxr, cden = (dxl*dxr)*(dxl+dxr) and the rounded
// reciprocals come from the per-axis geometry tables (same operations,
// evaluated once on the host).
//   slope = (sign(1/2, dV_L) + sign(1/2, dV_R))
//           * min(|theta dV_L / dX_L|, |theta dV_R / dX_R|, |num / cden|)
// The correctly rounded quotients are monotone in the exact ones, so the
// minimum is the rounded quotient of the smallest exact one: approximate
// quotients (within 2^-52 relative) pick it, and only that one is divided
// exactly.  When two non-zero candidates are too close to separate, or a
// quotient is outside the Markstein range, the whole slope is redone the
// reference's way.
// When the signs differ the factor is +0 and so is the slope.
__device__ __forceinline__ double limited_slope(double vm, double v0, double vp, double dxl,
                                                double dxr, double sql, double sqr,
                                                double cden, double rdxl, double rdxr,
                                                double rcden, double theta, int use_limiter) {
  const double dvl = v0 - vm;
  const double dvr = vp - v0;
  const double num = sqr * dvl + sql * dvr;
  if (!use_limiter) return div_rn(num, cden, rcden);
  const double s = copysign(0.5, dvl) + copysign(0.5, dvr);
  const double a1 = fabs(theta * dvl), a2 = fabs(theta * dvr), a3 = fabs(num);
  const double t1 = a1 * rdxl, t2 = a2 * rdxr, t3 = a3 * rcden;
#if GFX_FAST_MATH
  // the smallest of the products with the reciprocals is the slope's size
  (void)dxl, (void)dxr, (void)sql, (void)cden;
  return s * fmin3(t1, t2, t3);
#endif
  // branch-free argmin of the approximations and the runner-up
  const bool p12 = t1 <= t2;
  double tm = p12 ? t1 : t2, tr = p12 ? t2 : t1;
  double am = p12 ? a1 : a2, bm = p12 ? dxl : dxr, rm = p12 ? rdxl : rdxr;
  const bool p3 = t3 < tm;
  tr = p3 ? tm : fmin(tr, t3);
  tm = p3 ? t3 : tm;
  am = p3 ? a3 : am;
  bm = p3 ? cden : bm;
  rm = p3 ? rcden : rm;
  const double q = markstein(am, bm, rm);
  // a zero candidate is the minimum whatever the ties
  const bool fast = (am == 0.0 || tr > tm * (1.0 + 0x1p-50)) && geo_quotient_in_range(am);
  if (s == 0.0) return 0.0;
  return fast ? s * q : limited_slope_ieee(dvl, dvr, dxl, dxr, sql, sqr, cden, theta);
}

// PARABOLIC reconstruction of one cell (IncrementDivergence_FV__Kernel.f90:
// 296-596) with the cell averages XA = X and X2A = X**2 its caller passes
// (IncrementDivergence_FV__Form.f90:850-927).  g holds per-axis tables over
// the ghost-inclusive index (entry t of table q at g[q L + t]): the centre, its
// square, the inner and outer edges, and each denominator of the scheme that
// depends on the geometry only, with its correctly rounded reciprocal; every
// division by them is exact (div_rn).  The extremum position divides by a
// value-dependent quantity and uses the IEEE division.  SqrtTiny is
// tiny(0.0), as the reference sets it.
enum {
  PG_XC, PG_X2, PG_XI, PG_XO,
  PG_D1, PG_R1, PG_DA, PG_RA, PG_DB, PG_RB,
  PG_D3, PG_R3, PG_D4A, PG_R4A, PG_D4B, PG_R4B,
  PG_N
};

struct FaceVals {
  double vI, vO;  // inner and outer face values of the cell
};

__device__ __noinline__ FaceVals parabolic_cell(double vM, double vC, double vP,
                                                const double* __restrict__ g, int L, int t) {
  const double SqrtTiny = kTiny;
  const double xAM = __ldg(g + PG_XC * L + t - 1), xAC = __ldg(g + PG_XC * L + t),
               xAP = __ldg(g + PG_XC * L + t + 1);
  const double x2AM = __ldg(g + PG_X2 * L + t - 1), x2AC = __ldg(g + PG_X2 * L + t),
               x2AP = __ldg(g + PG_X2 * L + t + 1);
  const double xI = __ldg(g + PG_XI * L + t), xO = __ldg(g + PG_XO * L + t);
  FaceVals r;
  if ((vC - vM) * (vP - vC) <= 0.0) {
    r.vI = vC;
    r.vO = vC;
    return r;
  }
  double D = __ldg(g + PG_D1 * L + t), R = __ldg(g + PG_R1 * L + t);
  double c0 = div_rn(vP * (x2AM * xAC - x2AC * xAM) + vM * (x2AC * xAP - x2AP * xAC) +
                         vC * (x2AP * xAM - x2AM * xAP),
                     D, R);
  double c1 = div_rn(vP * (x2AC - x2AM) + vC * (x2AM - x2AP) + vM * (x2AP - x2AC), D, R);
  double c2 = div_rn(vP * (xAM - xAC) + vM * (xAC - xAP) + vC * (xAP - xAM), D, R);
  double c2s = copysign(fmax2(fabs(c2), SqrtTiny), c2);
  double xE = -div_ieee(c1, 2.0 * c2s);
  double vI = c0 + c1 * xI + c2 * (xI * xI);
  double vO = c0 + c1 * xO + c2 * (xO * xO);
  if (xE > xAM && xE <= xAC) {
    D = __ldg(g + PG_DA * L + t);
    R = __ldg(g + PG_RA * L + t);
    c0 = div_rn((vM * x2AC - vC * x2AM) + 2.0 * (vC * xAM - vM * xAC) * xAM, D, R);
    c1 = -div_rn(2.0 * (vC - vM) * xAM, D, R);
    c2 = div_rn(vC - vM, D, R);
    vI = c0 + c1 * xI + c2 * (xI * xI);
  } else if (xE > xAC && xE < xAP) {
    D = __ldg(g + PG_DB * L + t);
    R = __ldg(g + PG_RB * L + t);
    c0 = div_rn((vP * x2AC - vC * x2AP) + 2.0 * (vC * xAP - vP * xAC) * xAP, D, R);
    c1 = -div_rn(2.0 * (vC - vP) * xAP, D, R);
    c2 = div_rn(vC - vP, D, R);
    vO = c0 + c1 * xO + c2 * (xO * xO);
  }
  D = __ldg(g + PG_D3 * L + t);
  R = __ldg(g + PG_R3 * L + t);
  c0 = div_rn(vO * xI * (x2AC - xAC * xI) + vC * xI * xO * (xI - xO) +
                  vI * xO * (xAC * xO - x2AC),
              D, R);
  c1 = div_rn(vO * (xI * xI - x2AC) + vI * (x2AC - xO * xO) + vC * (xO * xO - xI * xI), D, R);
  c2 = div_rn(vO * (xAC - xI) + vC * (xI - xO) + vI * (xO - xAC), D, R);
  c2s = copysign(fmax2(fabs(c2), SqrtTiny), c2);
  xE = -div_ieee(c1, 2.0 * c2s);
  const double vI2 = c0 + c1 * xI + c2 * (xI * xI);
  const double vO2 = c0 + c1 * xO + c2 * (xO * xO);
  vI = vI2;
  vO = vO2;
  if (xE > xI && xE <= xAC) {
    D = __ldg(g + PG_D4A * L + t);
    R = __ldg(g + PG_R4A * L + t);
    c0 = div_rn((vO * x2AC - vC * (xO * xO)) + 2.0 * xI * (vC * xO - vO * xAC), D, R);
    c1 = -div_rn(2.0 * (vC - vO) * xI, D, R);
    c2 = div_rn(vC - vO, D, R);
    vI = c0 + c1 * xI + c2 * (xI * xI);
  } else if (xE > xAC && xE < xO) {
    D = __ldg(g + PG_D4B * L + t);
    R = __ldg(g + PG_R4B * L + t);
    c0 = div_rn((vI * x2AC - vC * (xI * xI)) + 2.0 * xO * (vC * xI - vI * xAC), D, R);
    c1 = -div_rn(2.0 * (vC - vI) * xO, D, R);
    c2 = div_rn(vC - vI, D, R);
    vO = c0 + c1 * xO + c2 * (xO * xO);
  }
  r.vI = vI;
  r.vO = vO;
  return r;
}

// Entropy per baryon of Apply_EOS_I_E_Kernel (Fluid_P_I__Kernel.f90:244-267)
// with N0 = P0 = 1, for N > 0 and P > 0: c_v log(P (N0/N)^gamma) as written,
// or c_v (log P - gamma log N) in the speed variant (two logarithms instead of
// a logarithm and a power).
__device__ __forceinline__ double entropy_per_baryon(double P, double N, const Phys& ph) {
#if GFX_FAST_MATH
  return ph.c_v * (log(P) - ph.gamma * log(N));
#else
  return ph.c_v * log(P * pow(1.0 / N, ph.gamma));
#endif
}

// State at one face after ComputeFromPrimitiveCommon (Fluid_P_I__Form.f90:509-601):
// Apply_EOS_I_E (Fluid_P_I__Kernel.f90:244-267), Compute_D_S_G
// (Fluid_D__Kernel.f90:47-101), Compute_G_G (Fluid_P__Kernel.f90:12-52),
// Compute_DS_G (:55-91), Compute_FE_P_G (:242-316).
struct FaceState {
  double N, V1, V2, V3, E;
  double D, S1, S2, S3, G;
  double P, CS, DS;
};

template <int NF>
__device__ __forceinline__ void face_state(double N, double V1, double V2, double V3, double E,
                                           const Phys& ph, FaceState& s) {
  const double P = ph.gm1 * E;
  double CS = 0.0, SB = -kSqrtHuge;
  if (N > 0.0 && P > 0.0) {
    CS = sound_speed(P, N, ph);
    if (NF == 6) SB = entropy_per_baryon(P, N, ph);
  }
  if (N < 0.0) N = 0.0;
  s.N = N;
  s.V1 = V1;
  s.V2 = V2;
  s.V3 = V3;
  s.E = E;
  s.D = N;
  s.S1 = N * V1;
  s.S2 = N * V2;
  s.S3 = N * V3;
  s.G = E + 0.5 * (s.S1 * V1 + s.S2 * V2 + s.S3 * V3);
  s.P = P;
  s.CS = CS;
  s.DS = (NF == 6) ? SB * N : 0.0;
}

template <int D>
__device__ __forceinline__ double vel(const FaceState& s) {
  return D == 0 ? s.V1 : (D == 1 ? s.V2 : s.V3);
}
template <int D>
__device__ __forceinline__ double mom(const FaceState& s) {
  return D == 0 ? s.S1 : (D == 1 ? s.S2 : s.S3);
}

// Riemann flux through one face along direction D: HLL (Current_Kernel.f90:
// 50-137 with the unit diffusion factor) and, for HLLC, the centre states of
// Fluid_P__Kernel.f90:319-668.  The HLLC selection is evaluated first; the HLL
// flux is only formed when the reference would keep it (diffusive-flux flag
// set, or a vanishing outer wave speed), which leaves every value unchanged.
// F holds D, S1, S2, S3, G and, for NF == 6, DS.
template <int D, bool HLLC, int NF>
__device__ __forceinline__ void riemann_flux(const FaceState& L, const FaceState& R,
                                             bool diffusive, double* F) {
  const double vl = vel<D>(L), vr = vel<D>(R);
  const double AP = fmax3(0.0, vl + L.CS, vr + R.CS);
  const double AM = fmax3(0.0, -(vl - L.CS), -(vr - R.CS));
  if (HLLC) {
    const double fdl = L.D * vl, fdr = R.D * vr;
    const double fsl = mom<D>(L) * vl + L.P, fsr = mom<D>(R) * vr + R.P;
    const double MD = AP * R.D + AM * L.D - fdr + fdl;
    const double SN = AP * mom<D>(R) + AM * mom<D>(L) - fsr + fsl;
#if GFX_FAST_MATH
    const double MDinv = fmax2(MD, 0.0) * recip(fmax2(MD * MD, kTiny));
#else
    const double MDinv = fmax2(MD, 0.0) / fmax2(MD * MD, kTiny);
#endif
    const double AC = SN * MDinv;
    if (!diffusive && AP != 0.0 && AM != 0.0) {
      const FaceState& S = (AC >= 0.0) ? L : R;
      const double vs = vel<D>(S);
      double A_V, A_AC;
      if (AC >= 0.0) {
        A_V = AM + vs;
        A_AC = AM + AC;
      } else {
        A_V = AP - vs;
        A_AC = AP - AC;
      }
      const double inv = recip(fmax2(fabs(A_AC), kSqrtTiny));
      const double Dc = S.D * A_V * inv;
      const double v1 = (D == 0) ? AC : S.V1;
      const double v2 = (D == 1) ? AC : S.V2;
      const double v3 = (D == 2) ? AC : S.V3;
      const double s1 = Dc * v1, s2 = Dc * v2, s3 = Dc * v3;
      const double sd = (D == 0) ? s1 : (D == 1 ? s2 : s3);
      double Pc, Gc;
      if (AC >= 0.0) {
        Pc = S.P + mom<D>(S) * A_V - sd * A_AC;
        Gc = (S.G * A_V + vs * S.P - AC * Pc) * inv;
      } else {
        Pc = S.P - mom<D>(S) * A_V + sd * A_AC;
        Gc = (S.G * A_V - vs * S.P + AC * Pc) * inv;
      }
      F[0] = Dc * AC;
      F[1] = s1 * AC;
      F[2] = s2 * AC;
      F[3] = s3 * AC;
      F[1 + D] = F[1 + D] + Pc;
      F[4] = (Gc + Pc) * AC;
      if (NF == 6) F[5] = S.DS * A_V * inv * AC;
      return;
    }
  }
  // HLL
  double FL[NF], FR[NF];
  FL[0] = L.D * vl;  FR[0] = R.D * vr;
  FL[1] = L.S1 * vl; FR[1] = R.S1 * vr;
  FL[2] = L.S2 * vl; FR[2] = R.S2 * vr;
  FL[3] = L.S3 * vl; FR[3] = R.S3 * vr;
  FL[1 + D] = FL[1 + D] + L.P;
  FR[1 + D] = FR[1 + D] + R.P;
  FL[4] = (L.G + L.P) * vl;
  FR[4] = (R.G + R.P) * vr;
  if (NF == 6) {
    FL[5] = L.DS * vl;
    FR[5] = R.DS * vr;
  }
  const double UL[6] = {L.D, L.S1, L.S2, L.S3, L.G, L.DS};
  const double UR[6] = {R.D, R.S1, R.S2, R.S3, R.G, R.DS};
  const double den = fmax2(AP + AM, kTiny);
  const double rden = recip(den);
  const double apam = AP * AM;
  double num[NF];
  bool ok = true;
#pragma unroll
  for (int u = 0; u < NF; ++u) {
    num[u] = AP * FL[u] + AM * FR[u] - apam * (UR[u] - UL[u]);
    F[u] = markstein(num[u], den, rden);
    ok &= quotient_in_range(num[u], rden);
  }
  if (!ok) {
#pragma unroll
    for (int u = 0; u < NF; ++u) F[u] = div_ieee(num[u], den);
  }
}

// Compute_N_V_E_G_Kernel (Fluid_P__Kernel.f90:94-192, both loops): the floored
// conserved values and the primitives of one value.
struct Prim {
  double N, V1, V2, V3, E;
};
struct Cons {
  double D, S1, S2, S3, G;
};

__device__ __forceinline__ void cons_to_prim(Cons& u, Prim& w, double nmin) {
  if (u.D > nmin) {
    w.N = u.D;
    const double rd = 1.0 / u.D;
    w.V1 = markstein(u.S1, u.D, rd);
    w.V2 = markstein(u.S2, u.D, rd);
    w.V3 = markstein(u.S3, u.D, rd);
    if (!(quotient_in_range(u.S1, rd) & quotient_in_range(u.S2, rd) &
          quotient_in_range(u.S3, rd))) {
      w.V1 = div_ieee(u.S1, u.D);
      w.V2 = div_ieee(u.S2, u.D);
      w.V3 = div_ieee(u.S3, u.D);
    }
    w.E = u.G - 0.5 * (u.S1 * w.V1 + u.S2 * w.V2 + u.S3 * w.V3);
  } else {
    w.N = nmin;
    w.V1 = 0.0;
    w.V2 = 0.0;
    w.V3 = 0.0;
    w.E = 0.0;
    u.D = nmin;
    u.S1 = 0.0;
    u.S2 = 0.0;
    u.S3 = 0.0;
    u.G = 0.0;
  }
  if (w.E < 0.0) {
    w.E = 0.0;
    u.G = w.E + 0.5 * (u.S1 * w.V1 + u.S2 * w.V2 + u.S3 * w.V3);
  }
}

// The recovery as the shock test needs it: the pressure and velocities of the
// reference's arithmetic, every operation rounded on its own, in both builds.
// The test's flags switch the flux discontinuously, so a pressure or a
// velocity difference one unit in the last place off can flip a flag where
// the jump sits at the threshold or the velocities are equal.  The exact
// build's cons_to_prim already rounds so; the speed build spells the
// operations out as intrinsics, which are never fused.
__device__ __forceinline__ void cons_to_prim_exact(Cons& u, Prim& w, double nmin) {
#if GFX_FAST_MATH
  if (u.D > nmin) {
    w.N = u.D;
    w.V1 = __ddiv_rn(u.S1, u.D);
    w.V2 = __ddiv_rn(u.S2, u.D);
    w.V3 = __ddiv_rn(u.S3, u.D);
    const double ke = __dadd_rn(__dadd_rn(__dmul_rn(u.S1, w.V1), __dmul_rn(u.S2, w.V2)),
                                __dmul_rn(u.S3, w.V3));
    w.E = __dsub_rn(u.G, __dmul_rn(0.5, ke));
  } else {
    w.N = nmin;
    w.V1 = 0.0;
    w.V2 = 0.0;
    w.V3 = 0.0;
    w.E = 0.0;
    u.D = nmin;
    u.S1 = 0.0;
    u.S2 = 0.0;
    u.S3 = 0.0;
    u.G = 0.0;
  }
  if (w.E < 0.0) {
    w.E = 0.0;
    u.G = __dmul_rn(0.5, __dadd_rn(__dadd_rn(__dmul_rn(u.S1, w.V1), __dmul_rn(u.S2, w.V2)),
                                   __dmul_rn(u.S3, w.V3)));
  }
#else
  cons_to_prim(u, w, nmin);
#endif
}

// The floored conserved values that cons_to_prim would have produced, rebuilt
// from the original conserved values and the primitives without divisions:
// D' = N; S' = S unless D <= nmin; G' = 0.5 (S'.V) exactly when the recovered
// E is zero (E < 0 floored, or G - 0.5 (S.V) == 0, where G already equals it).
__device__ __forceinline__ Cons floored_cons(const Cons& u, const Prim& w, double nmin) {
  Cons f;
  const bool live = u.D > nmin;
  f.D = w.N;
  f.S1 = live ? u.S1 : 0.0;
  f.S2 = live ? u.S2 : 0.0;
  f.S3 = live ? u.S3 : 0.0;
  f.G = live ? u.G : 0.0;
  if (w.E == 0.0) f.G = w.E + 0.5 * (f.S1 * w.V1 + f.S2 * w.V2 + f.S3 * w.V3);
  return f;
}

// RN(a / m) > t, exactly, for a >= 0 (or NaN) and m > 0.  The product
// p = RN(t m) carries a relative error of at most 2^-53 when it is normal, so
// a > RN(p (1 + 2^-50)) implies a / m > t (1 + 2^-51) >= t + ulp(t), and
// a < RN(p (1 - 2^-50)) implies a / m < t (1 - 2^-51) <= pred(t): the
// rounded quotient is then above t, resp. not above it.  Only between the two
// bounds (or out of the exponent window) is the division carried out.
__device__ __forceinline__ bool quotient_exceeds(double a, double m, double t) {
  const double p = t * m;
  if (t >= 0x1p-1000 && t <= 0x1p1000 && p >= 0x1p-960 && p <= 0x1p960) {
    if (a > p * (1.0 + 0x1p-50)) return true;
    if (a < p * (1.0 - 0x1p-50)) return false;
  }
  return a / m > t;
}

// The shock test of DetectShocks_CSL_Kernel (FluidFeatures_P__Kernel.f90:
// 12-186) between a cell (pressure P0) and its lower neighbour along one
// axis (P1), dV the difference of their normal velocities.
__device__ __forceinline__ bool shock_between(double P0, double P1, double dV, double thr) {
  const double dP = fabs(P0 - P1);
  const double pmin = (P0 < P1) ? P0 : P1;  // Fortran MIN: ties give either
  return quotient_exceeds(dP, fmax2(pmin, kSqrtTiny), thr) && dV <= 0.0;
}

// Apply_EOS_I_E_Kernel for a cell value: pressure, sound speed and (when
// asked) the entropy per baryon.
__device__ __forceinline__ void eos_cell(double N, double E, const Phys& ph, double& P,
                                         double& CS, double* SB) {
  P = ph.gm1 * E;
  if (N > 0.0 && P > 0.0) {
    CS = sound_speed(P, N, ph);
    if (SB) *SB = entropy_per_baryon(P, N, ph);
  } else {
    CS = 0.0;
    if (SB) *SB = -kSqrtHuge;
  }
}

// Inverse CFL time of one cell, Integrator_C_PS__Kernel.f90:122-137
// (coarsening factors are 1 on this chart).
__device__ __forceinline__ double inverse_cfl_time(const Prim& w, double CS, double w0,
                                                   double w1, double w2, double r0, double r1,
                                                   double r2) {
  return div_geo(fmax2(w.V1 + CS, -(w.V1 - CS)), w0, r0) +
         div_geo(fmax2(w.V2 + CS, -(w.V2 - CS)), w1, r1) +
         div_geo(fmax2(w.V3 + CS, -(w.V3 - CS)), w2, r2);
}

// Total order of doubles as unsigned integers, for atomicMax reductions.
__device__ __forceinline__ unsigned long long ordered_bits(double x) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double from_ordered_bits_dev(unsigned long long u) {
  const unsigned long long b = (u & 0x8000000000000000ull) ? (u & 0x7fffffffffffffffull) : ~u;
  return __longlong_as_double((long long)b);
}
inline double from_ordered_bits(unsigned long long u) {
  const unsigned long long b = (u & 0x8000000000000000ull) ? (u & 0x7fffffffffffffffull) : ~u;
  double x;
  memcpy(&x, &b, sizeof(x));
  return x;
}

}  // namespace gfx

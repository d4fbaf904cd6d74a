// adjoint_physics.cuh -- pointwise reverse-mode derivatives of the Fluid_P_I
// step: the limiter, the face equation of state, the HLL / HLLC fluxes, the
// conserved-to-primitive recovery, the uniform-gravity source and the final
// ComputeFromConserved with its entropy field.
//
// Each function recomputes the forward values it needs and returns the
// transposed Jacobian applied to an adjoint vector, differentiating the branch
// that the forward takes (limiter argument, wave-speed maxima, HLLC side,
// floors).  Forward quotients use IEEE division here: they are correctly
// rounded like the exact divisions of the stage kernels, so every branch
// decision matches the forward step.
#pragma once

#include "fluid_physics.cuh"

namespace gfx {

// limited_slope (the same value, bit for bit) together with the branch it
// took: 0 = zero slope (signs differ, or s == 0), 1 = |theta dV_L| / dX_L,
// 2 = |theta dV_R| / dX_R, 3 = the centred difference.  On that branch the
// slope is linear in (dV_L, dV_R) with the coefficients of slope_coeffs:
// s sign(dV_L) = s sign(dV_R) = s sign(num) = 1 whenever s != 0.
__device__ __forceinline__ double limited_slope_branch(double vm, double v0, double vp,
                                                       double dxl, double dxr, double sql,
                                                       double sqr, double cden, double rdxl,
                                                       double rdxr, double rcden, double theta,
                                                       int use_limiter, int& branch) {
  const double dvl = v0 - vm;
  const double dvr = vp - v0;
  const double num = sqr * dvl + sql * dvr;
  if (!use_limiter) {
    branch = 3;
    return div_rn(num, cden, rcden);
  }
  const double s = copysign(0.5, dvl) + copysign(0.5, dvr);
  const double a1 = fabs(theta * dvl), a2 = fabs(theta * dvr), a3 = fabs(num);
  const double t1 = a1 * rdxl, t2 = a2 * rdxr, t3 = a3 * rcden;
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
  const bool fast = (am == 0.0 || tr > tm * (1.0 + 0x1p-50)) && geo_quotient_in_range(am);
  branch = (s == 0.0) ? 0 : (p3 ? 3 : (p12 ? 1 : 2));
  if (s == 0.0) return 0.0;
  return fast ? s * q : limited_slope_ieee(dvl, dvr, dxl, dxr, sql, sqr, cden, theta);
}

// d slope / d dV_L (gl) and d slope / d dV_R (gr) on a branch.
__device__ __forceinline__ void slope_coeffs(int branch, double sql, double sqr, double rdxl,
                                             double rdxr, double rcden, double theta,
                                             double& gl, double& gr) {
  gl = 0.0;
  gr = 0.0;
  if (branch == 1) {
    gl = theta * rdxl;
  } else if (branch == 2) {
    gr = theta * rdxr;
  } else if (branch == 3) {
    gl = sqr * rcden;
    gr = sql * rcden;
  }
}

// Adjoint of one face state (face_state<5>): given the adjoints of D, S1..3,
// G, P, CS and direct adjoints of the velocities (lv), returns the adjoints
// of the reconstructed primitives N, V1, V2, V3, E.
struct FaceStateAdj {
  double D, S[3], G, P, CS, V[3];
};

__device__ __forceinline__ void face_state_adjoint(const double* w, const FaceState& s,
                                                   const Phys& ph, const FaceStateAdj& a,
                                                   double* lw) {
  const double N = w[0];
  const double Np = s.N;  // max(N, 0)
  const double V[3] = {w[1], w[2], w[3]};
  // G = E + 0.5 (N' V1 V1 + N' V2 V2 + N' V3 V3); S_i = N' V_i; D = N'
  double lN = 0.0;
  if (N > 0.0) {
    lN = a.D + a.S[0] * V[0] + a.S[1] * V[1] + a.S[2] * V[2] +
         a.G * 0.5 * (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
  }
  double lE = a.G + ph.gm1 * a.P;
  if (s.CS > 0.0 && a.CS != 0.0) {
    // CS = sqrt(gamma (gamma - 1) E / N): dCS/dE = CS / (2 E), dCS/dN = -CS / (2 N)
    const double r = 0.5 * s.CS * recip(N * w[4]);
    lE += a.CS * r * N;
    lN += -a.CS * r * w[4];
  }
  lw[0] = lN;
#pragma unroll
  for (int i = 0; i < 3; ++i) lw[1 + i] = a.V[i] + a.S[i] * Np + a.G * Np * V[i];
  lw[4] = lE;
}

template <int D>
__device__ __forceinline__ double mom_of(const FaceState& s) {
  return D == 0 ? s.S1 : (D == 1 ? s.S2 : s.S3);
}
template <int D>
__device__ __forceinline__ double vel_of(const FaceState& s) {
  return D == 0 ? s.V1 : (D == 1 ? s.V2 : s.V3);
}

// Adjoint of the wave speeds AP = max(0, vl + CSl, vr + CSr) and
// AM = max(0, -(vl - CSl), -(vr - CSr)) (fmax3: the first of equal values wins).
template <int D>
__device__ __forceinline__ void wave_speed_adjoint(const FaceState& L, const FaceState& R,
                                                   double lAP, double lAM, FaceStateAdj& aL,
                                                   FaceStateAdj& aR) {
  const double vl = vel_of<D>(L), vr = vel_of<D>(R);
  {
    const double b = vl + L.CS, c = vr + R.CS;
    double r = 0.0;
    int arg = 0;
    if (b > r) {
      r = b;
      arg = 1;
    }
    if (c > r) arg = 2;
    if (arg == 1) {
      aL.V[D] += lAP;
      aL.CS += lAP;
    } else if (arg == 2) {
      aR.V[D] += lAP;
      aR.CS += lAP;
    }
  }
  {
    const double b = -(vl - L.CS), c = -(vr - R.CS);
    double r = 0.0;
    int arg = 0;
    if (b > r) {
      r = b;
      arg = 1;
    }
    if (c > r) arg = 2;
    if (arg == 1) {
      aL.V[D] -= lAM;
      aL.CS += lAM;
    } else if (arg == 2) {
      aR.V[D] -= lAM;
      aR.CS += lAM;
    }
  }
}

// Adjoint of riemann_flux<D, HLLC, 5> (Current_Kernel.f90:50-137;
// Fluid_P__Kernel.f90:319-668) for one face: lF holds the adjoints of the five
// fluxes; the adjoints of the reconstructed primitives of the left and right
// states are added to ll and lr.  The branch (HLLC centre state of the side
// selected by AC, or HLL) is the forward's.
template <int D, bool HLLC>
__device__ __forceinline__ void flux_adjoint(const double* l, const double* r, bool diffusive,
                                             const double* lF, const Phys& ph, double* ll,
                                             double* lr) {
  FaceState L, R;
  face_state<5>(l[0], l[1], l[2], l[3], l[4], ph, L);
  face_state<5>(r[0], r[1], r[2], r[3], r[4], ph, R);
  FaceStateAdj aL{}, aR{};
  const double vl = vel_of<D>(L), vr = vel_of<D>(R);
  const double AP = fmax3(0.0, vl + L.CS, vr + R.CS);
  const double AM = fmax3(0.0, -(vl - L.CS), -(vr - R.CS));
  double lAP = 0.0, lAM = 0.0;
  bool done = false;
  if (HLLC) {
    const double fdl = L.D * vl, fdr = R.D * vr;
    const double sl = mom_of<D>(L), sr = mom_of<D>(R);
    const double fsl = sl * vl + L.P, fsr = sr * vr + R.P;
    const double MD = AP * R.D + AM * L.D - fdr + fdl;
    const double SN = AP * sr + AM * sl - fsr + fsl;
#if GFX_FAST_MATH
    const double m = fmax2(MD, 0.0) * recip(fmax2(MD * MD, kTiny));  // as the forward
#else
    const double m = fmax2(MD, 0.0) / fmax2(MD * MD, kTiny);
#endif
    const double AC = SN * m;
    if (!diffusive && AP != 0.0 && AM != 0.0) {
      done = true;
      const bool left = AC >= 0.0;
      const FaceState& S = left ? L : R;
      FaceStateAdj& aS = left ? aL : aR;
      const double sg = left ? 1.0 : -1.0;
      const double vs = vel_of<D>(S);
      const double A_V = left ? AM + vs : AP - vs;
      const double A_AC = left ? AM + AC : AP - AC;
      const double den = fmax2(fabs(A_AC), kSqrtTiny);
      const double inv = recip(den);
      const double Dc = S.D * A_V * inv;
      double v[3] = {S.V1, S.V2, S.V3};
      v[D] = AC;
      const double s[3] = {Dc * v[0], Dc * v[1], Dc * v[2]};
      const double mS = mom_of<D>(S);
      const double Pc = S.P + sg * (mS * A_V - s[D] * A_AC);
      const double T = S.G * A_V + sg * (vs * S.P - AC * Pc);
      const double Gc = T * inv;
      // F0 = Dc AC; F(1+i) = s_i AC (+ Pc at i = D); F4 = (Gc + Pc) AC
      double lAC = lF[0] * Dc + lF[4] * (Gc + Pc);
      double lDc = lF[0] * AC;
      double ls[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        ls[i] = lF[1 + i] * AC;
        lAC += lF[1 + i] * s[i];
      }
      double lPc = lF[1 + D] + lF[4] * AC;
      const double lGc = lF[4] * AC;
      // Gc = T inv
      const double lT = lGc * inv;
      double linv = lGc * T;
      // T = S.G A_V + sg (vs S.P - AC Pc)
      double lA_V = lT * S.G;
      aS.G += lT * A_V;
      double lvs = sg * lT * S.P;
      aS.P += sg * lT * vs;
      lAC += -sg * lT * Pc;
      lPc += -sg * lT * AC;
      // Pc = S.P + sg (mS A_V - s_D A_AC)
      aS.P += lPc;
      aS.S[D] += sg * lPc * A_V;
      lA_V += sg * lPc * mS;
      ls[D] += -sg * lPc * A_AC;
      double lA_AC = -sg * lPc * s[D];
      // s_i = Dc v_i
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        lDc += ls[i] * v[i];
        if (i == D)
          lAC += ls[i] * Dc;
        else
          aS.V[i] += ls[i] * Dc;
      }
      // Dc = S.D A_V inv
      aS.D += lDc * A_V * inv;
      lA_V += lDc * S.D * inv;
      linv += lDc * S.D * A_V;
      // inv = 1 / max(|A_AC|, sqrt(tiny))
      if (fabs(A_AC) > kSqrtTiny) lA_AC += -linv * inv * inv * copysign(1.0, A_AC);
      // A_V = AM + vs | AP - vs; A_AC = AM + AC | AP - AC
      if (left) {
        lAM += lA_V + lA_AC;
      } else {
        lAP += lA_V + lA_AC;
      }
      lvs += sg * lA_V;
      lAC += sg * lA_AC;
      aS.V[D] += lvs;
      // AC = SN m, m = max(MD, 0) / max(MD^2, tiny)
      const double lSN = lAC * m;
      double dm = 0.0;
      if (MD > 0.0) dm = (MD * MD > kTiny) ? -m * m : 1.0 / kTiny;
      const double lMD = lAC * SN * dm;
      // MD = AP R.D + AM L.D - fdr + fdl
      lAP += lMD * R.D;
      aR.D += lMD * AP;
      lAM += lMD * L.D;
      aL.D += lMD * AM;
      const double lfdr = -lMD, lfdl = lMD;
      // SN = AP sr + AM sl - fsr + fsl
      lAP += lSN * sr;
      aR.S[D] += lSN * AP;
      lAM += lSN * sl;
      aL.S[D] += lSN * AM;
      const double lfsr = -lSN, lfsl = lSN;
      // fd = D v; fs = S_D v + P
      aL.D += lfdl * vl;
      aL.V[D] += lfdl * L.D + lfsl * sl;
      aL.S[D] += lfsl * vl;
      aL.P += lfsl;
      aR.D += lfdr * vr;
      aR.V[D] += lfdr * R.D + lfsr * sr;
      aR.S[D] += lfsr * vr;
      aR.P += lfsr;
    }
  }
  if (!done) {
    // HLL: F = (AP FL + AM FR - AP AM (UR - UL)) / max(AP + AM, tiny)
    const double UL[5] = {L.D, L.S1, L.S2, L.S3, L.G};
    const double UR[5] = {R.D, R.S1, R.S2, R.S3, R.G};
    double FL[5], FR[5];
    FL[0] = L.D * vl;
    FR[0] = R.D * vr;
    FL[1] = L.S1 * vl;
    FR[1] = R.S1 * vr;
    FL[2] = L.S2 * vl;
    FR[2] = R.S2 * vr;
    FL[3] = L.S3 * vl;
    FR[3] = R.S3 * vr;
    FL[1 + D] += L.P;
    FR[1 + D] += R.P;
    FL[4] = (L.G + L.P) * vl;
    FR[4] = (R.G + R.P) * vr;
    const double sum = AP + AM;
    const bool live = sum > kTiny;
    const double rden = recip(live ? sum : kTiny);
    double lden = 0.0;
    double lFL[5], lFR[5];
#pragma unroll
    for (int u = 0; u < 5; ++u) {
      const double num = AP * FL[u] + AM * FR[u] - AP * AM * (UR[u] - UL[u]);
      const double ln = lF[u] * rden;
      if (live) lden += -ln * num * rden;
      lAP += ln * (FL[u] - AM * (UR[u] - UL[u]));
      lAM += ln * (FR[u] - AP * (UR[u] - UL[u]));
      lFL[u] = AP * ln;
      lFR[u] = AM * ln;
      const double lU = AP * AM * ln;
      // -AP AM (UR - UL)
      if (u == 0) {
        aR.D -= lU;
        aL.D += lU;
      } else if (u < 4) {
        aR.S[u - 1] -= lU;
        aL.S[u - 1] += lU;
      } else {
        aR.G -= lU;
        aL.G += lU;
      }
    }
    lAP += lden;
    lAM += lden;
    // raw fluxes
    aL.D += lFL[0] * vl;
    aR.D += lFR[0] * vr;
    double lvl = lFL[0] * L.D, lvr = lFR[0] * R.D;
    const double SLv[3] = {L.S1, L.S2, L.S3}, SRv[3] = {R.S1, R.S2, R.S3};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      aL.S[i] += lFL[1 + i] * vl;
      aR.S[i] += lFR[1 + i] * vr;
      lvl += lFL[1 + i] * SLv[i];
      lvr += lFR[1 + i] * SRv[i];
    }
    aL.P += lFL[1 + D];
    aR.P += lFR[1 + D];
    aL.G += lFL[4] * vl;
    aL.P += lFL[4] * vl;
    lvl += lFL[4] * (L.G + L.P);
    aR.G += lFR[4] * vr;
    aR.P += lFR[4] * vr;
    lvr += lFR[4] * (R.G + R.P);
    aL.V[D] += lvl;
    aR.V[D] += lvr;
  }
  wave_speed_adjoint<D>(L, R, lAP, lAM, aL, aR);
  double wl[5], wr[5];
  face_state_adjoint(l, L, ph, aL, wl);
  face_state_adjoint(r, R, ph, aR, wr);
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    ll[q] += wl[q];
    lr[q] += wr[q];
  }
}

// Adjoint of cons_to_prim (Compute_N_V_E_G_Kernel, Fluid_P__Kernel.f90:94-192)
// at the primitives w it produced: N = D, V = S / D, E = G - (S.V) / 2, so
//   dE/dG = 1, dE/dS_i = -V_i, dE/dD = |V|^2 / 2, dV_i/dS_i = 1 / D,
//   dV_i/dD = -V_i / D.
// A floored value (N <= nmin: constant state) passes nothing back; a floored
// internal energy (E == 0) passes nothing through E.
__device__ __forceinline__ void c2p_adjoint(const double* w, const double* lw, double nmin,
                                            double* lu) {
  const double N = w[0];
  if (!(N > nmin)) {
#pragma unroll
    for (int q = 0; q < 5; ++q) lu[q] = 0.0;
    return;
  }
  const double V[3] = {w[1], w[2], w[3]};
  const double lE = (w[4] == 0.0) ? 0.0 : lw[4];
  const double rN = 1.0 / N;
  double lD = lw[0] + lE * 0.5 * (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    lD += -lw[1 + i] * V[i] * rN;
    lu[1 + i] = lw[1 + i] * rN - lE * V[i];
  }
  lu[0] = lD;
  lu[4] = lE;
}

// Adjoint of the uniform-gravity source of a stage (ApplyGravity_F with the
// gradient (0, 0, a)): K_S3 -= N a dt, K_G -= N V3 a dt, at the stage's
// primitives w; lK holds the adjoints of K (D, S1, S2, S3, G).
__device__ __forceinline__ void gravity_adjoint(const double* w, const double* lK, double a,
                                                double dt, double* lw) {
  lw[0] += -a * dt * (lK[3] + w[3] * lK[4]);
  lw[3] += -w[0] * a * dt * lK[4];
}

// Adjoint of the end of the step, ComputeFromConserved on Z = U^n + K1/2 +
// K2/2 (Fluid_P_I__Form.f90:604-722): the floored conserved values and
// DS = N SB with SB = c_v log(P N^-gamma).  w are the primitives of the new
// state, lU the adjoints of its six conserved fields; returns the adjoints of
// Z's D, S1, S2, S3, G.  In a cell whose internal energy was floored
// (G' = S.V / 2) the entropy is the constant -sqrt(huge) and passes nothing.
__device__ __forceinline__ void final_adjoint(const double* w, const double* lU,
                                              const Phys& ph, double* lz) {
  const double N = w[0];
  if (!(N > ph.nmin)) {
#pragma unroll
    for (int q = 0; q < 5; ++q) lz[q] = 0.0;
    return;
  }
  const double V[3] = {w[1], w[2], w[3]};
  const double E = w[4];
  if (E == 0.0) {
    // D' = D, S' = S, G' = |S|^2 / (2 D): dG'/dS_i = V_i, dG'/dD = -|V|^2 / 2
    lz[0] = lU[0] - 0.5 * (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]) * lU[4];
#pragma unroll
    for (int i = 0; i < 3; ++i) lz[1 + i] = lU[1 + i] + V[i] * lU[4];
    lz[4] = 0.0;
    return;
  }
  // DS = N c_v log(P N^-gamma): dDS/dN = SB - gamma c_v, dDS/dE = N c_v / E
  double lp[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  const double P = ph.gm1 * E;
  if (N > 0.0 && P > 0.0 && lU[5] != 0.0) {
    const double SB = ph.c_v * log(P * pow(1.0 / N, ph.gamma));
    lp[0] = lU[5] * (SB - ph.gamma * ph.c_v);
    lp[4] = lU[5] * N * ph.c_v / E;
  }
  double lu[5];
  c2p_adjoint(w, lp, ph.nmin, lu);
#pragma unroll
  for (int q = 0; q < 5; ++q) lz[q] = lU[q] + lu[q];
}

}  // namespace gfx

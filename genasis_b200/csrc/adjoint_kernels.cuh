// adjoint_kernels.cuh -- kernels of the discrete adjoint of one RK2 step.
//
// The forward step (Step_RK_C_ASC__Template.f90:504-542 with the RK2 tableau
// of Step_RK2_C_ASC__Form.f90:51-57) is, with W() the conserved-to-primitive
// recovery and L() the flux divergence plus sources of a stage,
//   W0 = W(U^n), K1 = dt L(W0), W1 = W(U^n + K1), K2 = dt L(W1),
//   Z = U^n + K1/2 + K2/2, U^n+1 = ComputeFromConserved(Z).
// Its adjoint, given lam^n+1, runs backwards:
//   lamZ = final^T lam^n+1, lamW1 = L^T(lamZ / 2), lamY = W^T(W1) lamW1,
//   lamK1 = lamY + lamZ / 2, lamW0 = L^T(lamK1),
//   lam^n = lamZ + lamY + W^T(W0) lamW0 = lamZ / 2 + lamK1 + W^T(W0) lamW0.
// The stages are recomputed from the checkpoint U^n (the stage kernels write
// W1), the shock features are those of U^n in both stages, and dt is held
// fixed.  L^T is one kernel per direction: a thread sweeps a segment of faces
// of one pencil in order, keeps the stencil window in registers and adds each
// cell's adjoint once (an atomic add per value, since neighbouring segments
// and the ghost images of the boundary reach the same cells).
#pragma once

#include "adjoint_physics.cuh"
#include "aux_kernels.cuh"

namespace gfx {

struct AdjDesc {
  int n[3];
  int bc[3][2];
  long long nP;
  const double* W;     // primitives of the stage input, compact [5][nP]
  const double* lamK;  // adjoint of the stage increment, compact [5][nP]
  double* lamW;        // adjoint of the stage primitives, compact [5][nP] (added to)
  const uint8_t* df;   // DIFFUSIVE_FLUX_I bits, compact (or null)
  AxisGeo geo[3];
  double dt;
  double kscale;       // factor on lamK (1/2 for the second stage's lamZ)
  int seg, nseg;       // faces per thread, segments per pencil
};

__device__ __forceinline__ void adj_load(const AdjDesc& A, int D, long long base, long long sD,
                                         int c, double* w) {
  bool neg;
  const int s = bc_map(c, A.n[D], A.bc[D][0], A.bc[D][1], neg);
  const double* p = A.W + base + s * sD;
#pragma unroll
  for (int q = 0; q < 5; ++q) w[q] = __ldg(p + q * A.nP);
  if (neg) w[1 + D] = -w[1 + D];
}

__device__ __forceinline__ void adj_flush(const AdjDesc& A, int D, long long base, long long sD,
                                          int c, const double* a) {
  bool neg;
  const int s = bc_map(c, A.n[D], A.bc[D][0], A.bc[D][1], neg);
  double* p = A.lamW + base + s * sD;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    const double v = (neg && q == 1 + D) ? -a[q] : a[q];
    if (v != 0.0) atomicAdd(p + q * A.nP, v);
  }
}

template <int D, bool HLLC>
__global__ void __launch_bounds__(128, 3) adj_face_kernel(const __grid_constant__ AdjDesc A,
                                                       const __grid_constant__ Phys ph) {
  constexpr int T1 = (D == 0) ? 1 : 0;
  constexpr int T2 = (D == 2) ? 1 : 2;
  const int nD = A.n[D], n1 = A.n[T1], n2 = A.n[T2];
  const long long total = (long long)A.nseg * n1 * n2;
  const long long st[3] = {1, A.n[0], (long long)A.n[0] * A.n[1]};
  const AxisGeo& G = A.geo[D];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    int seg, i1, i2;
    if (D == 0) {
      seg = (int)(t % A.nseg);
      const long long r = t / A.nseg;
      i1 = (int)(r % n1);
      i2 = (int)(r / n1);
    } else {
      i1 = (int)(t % n1);
      const long long r = t / n1;
      i2 = (int)(r % n2);
      seg = (int)(r / n2);
    }
    const long long base = i1 * st[T1] + i2 * st[T2];
    const long long sD = st[D];
    const int s0 = seg * A.seg, s1 = min(nD + 1, s0 + A.seg);
    // coefficient of the face fluxes in a cell's increment: dt A / V = dt / width
    auto coef = [&](int c) { return A.dt * __ldg(G.RW + c + 2) * A.kscale; };
    // forward slopes of a cell, with the limiter branch of each field (2 bits)
    auto slope = [&](const double* vm, const double* v0, const double* vp, int c, double* out,
                     int& branches) {
      const int tt = c + 2;
      const double dxl = __ldg(G.dXI + tt), dxr = __ldg(G.dXI + tt + 1);
      const double sql = __ldg(G.SQ + tt), sqr = __ldg(G.SQ + tt + 1), cden = __ldg(G.CDEN + tt);
      const double rdxl = __ldg(G.RDXI + tt), rdxr = __ldg(G.RDXI + tt + 1),
                   rcden = __ldg(G.RCDEN + tt);
      branches = 0;
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        int br;
        out[q] = limited_slope_branch(vm[q], v0[q], vp[q], dxl, dxr, sql, sqr, cden, rdxl, rdxr,
                                      rcden, ph.theta, ph.use_limiter, br);
        branches |= br << (2 * q);
      }
    };
    // adjoint of the slopes of cell c into its stencil cells c - 1, c, c + 1
    auto slope_back = [&](int branches, int c, const double* ls, double* am, double* a0,
                          double* ap) {
      const int tt = c + 2;
      const double sql = __ldg(G.SQ + tt), sqr = __ldg(G.SQ + tt + 1);
      const double rdxl = __ldg(G.RDXI + tt), rdxr = __ldg(G.RDXI + tt + 1),
                   rcden = __ldg(G.RCDEN + tt);
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        double gl, gr;
        slope_coeffs((branches >> (2 * q)) & 3, sql, sqr, rdxl, rdxr, rcden, ph.theta, gl, gr);
        am[q] -= gl * ls[q];
        a0[q] += (gl - gr) * ls[q];
        ap[q] += gr * ls[q];
      }
    };
    auto load_lamk = [&](int c, double* out) {
      if (c >= 0 && c < nD) {
        const double k = coef(c);
        const double* p = A.lamK + base + c * sD;
#pragma unroll
        for (int q = 0; q < 5; ++q) out[q] = k * __ldg(p + q * A.nP);
      } else {
#pragma unroll
        for (int q = 0; q < 5; ++q) out[q] = 0.0;
      }
    };

    double wm2[5], wm1[5], w0[5], wp1[5];
    double sm1[5], s0v[5];
    double am2[5], am1[5], a0[5];
    double lsm1[5], lkm1[5], lk0[5];
    int bm1, b0;  // limiter branches of slope(i - 1), slope(i)
    adj_load(A, D, base, sD, s0 - 2, wm2);
    adj_load(A, D, base, sD, s0 - 1, wm1);
    adj_load(A, D, base, sD, s0, w0);
    slope(wm2, wm1, w0, s0 - 1, sm1, bm1);
    load_lamk(s0 - 1, lkm1);
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      am2[q] = 0.0;
      am1[q] = 0.0;
      a0[q] = 0.0;
      lsm1[q] = 0.0;
    }
    for (int i = s0; i < s1; ++i) {
      adj_load(A, D, base, sD, i + 1, wp1);
      slope(wm1, w0, wp1, i, s0v, b0);
      const double wr = __ldg(G.WR + i + 1), wl = __ldg(G.WL + i + 2);
      double l[5], r[5];
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        l[q] = wm1[q] + wr * sm1[q];
        r[q] = w0[q] - wl * s0v[q];
      }
      load_lamk(i, lk0);
      // face i is the inner face of cell i and the outer face of cell i - 1
      double lF[5], ll[5], lr[5];
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        lF[q] = lk0[q] - lkm1[q];
        ll[q] = 0.0;
        lr[q] = 0.0;
      }
      bool diff = false;
      if (HLLC && A.df != nullptr && i < nD) diff = (A.df[base + i * sD] >> D) & 1;
      flux_adjoint<D, HLLC>(l, r, diff, lF, ph, ll, lr);
      double ls0[5];
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        am1[q] += ll[q];
        lsm1[q] += wr * ll[q];
        a0[q] += lr[q];
        ls0[q] = -wl * lr[q];
      }
      // slope(i - 1) has all of this segment's contributions
      slope_back(bm1, i - 1, lsm1, am2, am1, a0);
      adj_flush(A, D, base, sD, i - 2, am2);
      bm1 = b0;
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        wm2[q] = wm1[q];
        wm1[q] = w0[q];
        w0[q] = wp1[q];
        sm1[q] = s0v[q];
        lsm1[q] = ls0[q];
        am2[q] = am1[q];
        am1[q] = a0[q];
        a0[q] = 0.0;
        lkm1[q] = lk0[q];
      }
    }
    // the last slope of the segment: cells s1 - 2, s1 - 1, s1
    slope_back(bm1, s1 - 1, lsm1, am2, am1, a0);
    adj_flush(A, D, base, sD, s1 - 2, am2);
    adj_flush(A, D, base, sD, s1 - 1, am1);
    adj_flush(A, D, base, sD, s1, a0);
  }
}

// Primitives of the proper cells of U (ghost layout) into a compact array:
// the stage-1 input W0 of the step.
__device__ __forceinline__ long long ghost_index(const Box& b, long long c) {
  // proper-cell counts stay below 2^31 (gfx_fluid_step_adjoint checks), so
  // 32-bit division
  const unsigned cc = (unsigned)c, n0 = (unsigned)b.n[0], n1 = (unsigned)b.n[1];
  const unsigned r = cc / n0, i = cc - r * n0, k = r / n1, j = r - k * n1;
  return (i + 2) + (long long)b.m[0] * ((j + 2) + (long long)b.m[1] * (k + 2));
}

__global__ void adj_prims_kernel(Box b, Phys ph, const double* __restrict__ U,
                                 double* __restrict__ W) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < b.nP;
       c += (long long)gridDim.x * blockDim.x) {
    const long long g = ghost_index(b, c);
    Cons u{U[g], U[b.nV + g], U[2 * b.nV + g], U[3 * b.nV + g], U[4 * b.nV + g]};
    Prim w;
    cons_to_prim(u, w, ph.nmin);
    W[c] = w.N;
    W[b.nP + c] = w.V1;
    W[2 * b.nP + c] = w.V2;
    W[3 * b.nP + c] = w.V3;
    W[4 * b.nP + c] = w.E;
  }
}

// lamZ = final^T lam^n+1 at the primitives of U^n+1 (both ghost layout).
__global__ void adj_final_kernel(Box b, Phys ph, const double* __restrict__ lam,
                                 const double* __restrict__ U, double* __restrict__ lamZ) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < b.nP;
       c += (long long)gridDim.x * blockDim.x) {
    const long long g = ghost_index(b, c);
    Cons u{U[g], U[b.nV + g], U[2 * b.nV + g], U[3 * b.nV + g], U[4 * b.nV + g]};
    Prim p;
    cons_to_prim(u, p, ph.nmin);
    const double w[5] = {p.N, p.V1, p.V2, p.V3, p.E};
    double lU[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) lU[q] = lam[q * b.nV + g];
    double lz[5];
    final_adjoint(w, lU, ph, lz);
#pragma unroll
    for (int q = 0; q < 5; ++q) lamZ[q * b.nP + c] = lz[q];
  }
}

// After L^T of stage 2: lamY = W^T(W1)(lamW1 + gravity^T(lamZ / 2)) and
// lamK1 = lamY + lamZ / 2.
__global__ void adj_mid_kernel(Box b, Phys ph, double dt, const double* __restrict__ W1,
                               const double* __restrict__ lamZ, const double* __restrict__ lamW,
                               double* __restrict__ lamK1) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < b.nP;
       c += (long long)gridDim.x * blockDim.x) {
    double w[5], lw[5], lk2[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      w[q] = W1[q * b.nP + c];
      lw[q] = lamW[q * b.nP + c];
      lk2[q] = 0.5 * lamZ[q * b.nP + c];
    }
    if (ph.accel != 0.0) gravity_adjoint(w, lk2, ph.accel, dt, lw);
    double ly[5];
    c2p_adjoint(w, lw, ph.nmin, ly);
#pragma unroll
    for (int q = 0; q < 5; ++q) lamK1[q * b.nP + c] = ly[q] + lk2[q];
  }
}

// After L^T of stage 1: lam^n = lamZ + lamY + W^T(W0)(lamW0 + gravity^T(lamK1)),
// with lamZ + lamY = lamZ / 2 + lamK1; DS and the ghosts keep the zeros the
// caller's array was cleared to.
__global__ void adj_last_kernel(Box b, Phys ph, double dt, const double* __restrict__ W0,
                                const double* __restrict__ lamK1,
                                const double* __restrict__ lamZ,
                                const double* __restrict__ lamW, double* __restrict__ lam) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < b.nP;
       c += (long long)gridDim.x * blockDim.x) {
    double w[5], lw[5], lk[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      w[q] = W0[q * b.nP + c];
      lw[q] = lamW[q * b.nP + c];
      lk[q] = lamK1[q * b.nP + c];
    }
    if (ph.accel != 0.0) gravity_adjoint(w, lk, ph.accel, dt, lw);
    double lu[5];
    c2p_adjoint(w, lw, ph.nmin, lu);
    const long long g = ghost_index(b, c);
#pragma unroll
    for (int q = 0; q < 5; ++q) lam[q * b.nV + g] = 0.5 * lamZ[q * b.nP + c] + lk[q] + lu[q];
  }
}

}  // namespace gfx

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
                                          int c, const double* a, int stride = 1) {
  bool neg;
  const int s = bc_map(c, A.n[D], A.bc[D][0], A.bc[D][1], neg);
  double* p = A.lamW + base + s * sD;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    const double v = (neg && q == 1 + D) ? -a[q * stride] : a[q * stride];
    if (v != 0.0) atomicAdd(p + q * A.nP, v);
  }
}

// CTAs of 128 threads per SM that the y / z sweep's registers must allow,
// its accumulators living in shared memory (25.6 KB a CTA): 4 in the exact
// build (128 registers, 48 B of spills), 5 in the fast build (96 registers);
// measured at 128^3 against 3 and 4 (y / z launches 235 -> 222 us exact,
// 195 -> 189 us fast)
#ifndef GFX_ADJ_MIN_BLOCKS
#if GFX_FAST_MATH
#define GFX_ADJ_MIN_BLOCKS 5
#else
#define GFX_ADJ_MIN_BLOCKS 4
#endif
#endif

constexpr int kAdjThreads = 128;  // threads of an L^T block

template <int D, bool HLLC>
__global__ void __launch_bounds__(kAdjThreads, GFX_ADJ_MIN_BLOCKS)
    adj_face_kernel(const __grid_constant__ AdjDesc A, const __grid_constant__ Phys ph) {
  __shared__ double s_adj[25 * kAdjThreads];
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
    // (the accumulators' columns, stride kAdjThreads)
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
        const double l = ls[q * kAdjThreads];
        am[q * kAdjThreads] -= gl * l;
        a0[q * kAdjThreads] += (gl - gr) * l;
        ap[q * kAdjThreads] += gr * l;
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

    // in registers: the stencil window and the slopes; in shared memory, one
    // column per thread ([element][thread]): the adjoint accumulators of the
    // cells i - 2, i - 1, i (a ring of three slots, slot (c + 3) % 3 for cell
    // c), the slope adjoint of cell i - 1 and lamK of cell i - 1, so that
    // little stays live across the flux adjoint
    double* my = s_adj + threadIdx.x;
    auto acc = [&](int c) { return my + ((c + 3) % 3) * 5 * kAdjThreads; };
    double* LS = my + 15 * kAdjThreads;
    double* LK = my + 20 * kAdjThreads;
    double wm2[5], wm1[5], w0[5], wp1[5];
    double sm1[5], s0v[5];
    int bm1, b0;  // limiter branches of slope(i - 1), slope(i)
    adj_load(A, D, base, sD, s0 - 2, wm2);
    adj_load(A, D, base, sD, s0 - 1, wm1);
    adj_load(A, D, base, sD, s0, w0);
    slope(wm2, wm1, w0, s0 - 1, sm1, bm1);
    {
      double lk[5];
      load_lamk(s0 - 1, lk);
#pragma unroll
      for (int q = 0; q < 5; ++q) LK[q * kAdjThreads] = lk[q];
    }
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      acc(s0 - 2)[q * kAdjThreads] = 0.0;
      acc(s0 - 1)[q * kAdjThreads] = 0.0;
      acc(s0)[q * kAdjThreads] = 0.0;
      LS[q * kAdjThreads] = 0.0;
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
      // face i is the inner face of cell i and the outer face of cell i - 1
      double lF[5], ll[5], lr[5];
      {
        double lk0[5];
        load_lamk(i, lk0);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
          lF[q] = lk0[q] - LK[q * kAdjThreads];
          LK[q * kAdjThreads] = lk0[q];
          ll[q] = 0.0;
          lr[q] = 0.0;
        }
      }
      bool diff = false;
      if (HLLC && A.df != nullptr && i < nD) diff = (A.df[base + i * sD] >> D) & 1;
      flux_adjoint<D, HLLC>(l, r, diff, lF, ph, ll, lr);
      double* am2 = acc(i - 2);
      double* am1 = acc(i - 1);
      double* a0 = acc(i);
      double ls0[5];
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        am1[q * kAdjThreads] += ll[q];
        LS[q * kAdjThreads] += wr * ll[q];
        a0[q * kAdjThreads] += lr[q];
        ls0[q] = -wl * lr[q];
      }
      // slope(i - 1) has all of this segment's contributions
      slope_back(bm1, i - 1, LS, am2, am1, a0);
      adj_flush(A, D, base, sD, i - 2, am2, kAdjThreads);
      bm1 = b0;
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        am2[q * kAdjThreads] = 0.0;  // the slot of cell i + 1
        LS[q * kAdjThreads] = ls0[q];
        wm1[q] = w0[q];
        w0[q] = wp1[q];
        sm1[q] = s0v[q];
      }
    }
    // the last slope of the segment: cells s1 - 2, s1 - 1, s1
    slope_back(bm1, s1 - 1, LS, acc(s1 - 2), acc(s1 - 1), acc(s1));
    adj_flush(A, D, base, sD, s1 - 2, acc(s1 - 2), kAdjThreads);
    adj_flush(A, D, base, sD, s1 - 1, acc(s1 - 1), kAdjThreads);
    adj_flush(A, D, base, sD, s1, acc(s1), kAdjThreads);
  }
}

// L^T along x with one lane per face.  x pencils are contiguous, so a thread
// sweeping a segment of one (adj_face_kernel<0>) strides its warp's loads and
// atomic adds over many cache lines; here a warp takes kAdjXFaces
// consecutive faces x0 .. x0 + 28 of one pencil instead.  Lane L holds cell
// c = x0 - 2 + L: its primitives and lamK come in coalesced, the stencil
// neighbours by shuffles.  Lanes 1 .. 30 compute the slope of their cell,
// lanes 2 .. 30 the adjoint of face c (between cells c - 1 and c); the
// adjoints of the face states go back through the slopes of cells c - 1 and
// c to the cells c - 2 .. c + 1, and every lane adds its cell's sum into
// lamW with one coalesced atomic add per field (the three cells at each end
// of the warp's range are shared with the neighbouring warp).  A cell's sum
// is formed in the order of the sweep: face c, slope c - 1, face c + 1,
// slope c, slope c + 1.
constexpr int kAdjXFaces = 29;

// Four CTAs of 128 threads per SM on both builds: a lane holds one cell, not
// the sweep's stencil window, and fits 128 registers without spills.
template <bool HLLC>
__global__ void __launch_bounds__(128, 4)
    adj_face_x_kernel(const __grid_constant__ AdjDesc A, const __grid_constant__ Phys ph) {
  constexpr unsigned FULL = 0xffffffffu;
  const int n0 = A.n[0], n1 = A.n[1], n2 = A.n[2];
  const int chunks = (n0 + 1 + kAdjXFaces - 1) / kAdjXFaces;
  const long long warps = (long long)chunks * n1 * n2;
  const int lane = threadIdx.x & 31;
  const AxisGeo& G = A.geo[0];
  const long long first = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long stride = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long wi = first; wi < warps; wi += stride) {  // uniform over the warp
    const int chunk = (int)(wi % chunks);
    const long long row = wi / chunks;
    const long long base = row * n0;  // row = i1 + n1 i2
    const int c = chunk * kAdjXFaces - 2 + lane;
    // the cell's primitives (the boundary image for a ghost; lanes past the
    // ghosts read a mapped proper cell and contribute nothing)
    double w[5];
    adj_load(A, 0, base, 1, c, w);
    // the slope of the cell (needs c in [-1, n0] for its tables: clamped for
    // the lanes whose slope no face uses)
    const int tt = max(-1, min(c, n0)) + 2;
    const double dxl = __ldg(G.dXI + tt), dxr = __ldg(G.dXI + tt + 1);
    const double sql = __ldg(G.SQ + tt), sqr = __ldg(G.SQ + tt + 1), cden = __ldg(G.CDEN + tt);
    const double rdxl = __ldg(G.RDXI + tt), rdxr = __ldg(G.RDXI + tt + 1),
                 rcden = __ldg(G.RCDEN + tt);
    double wm[5], sl[5], sm[5];
    int branches = 0;
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      wm[q] = __shfl_up_sync(FULL, w[q], 1);
      const double wp = __shfl_down_sync(FULL, w[q], 1);
      int br;
      sl[q] = limited_slope_branch(wm[q], w[q], wp, dxl, dxr, sql, sqr, cden, rdxl, rdxr, rcden,
                                   ph.theta, ph.use_limiter, br);
      branches |= br << (2 * q);
      sm[q] = __shfl_up_sync(FULL, sl[q], 1);
    }
    // lamK of the cell times dt A / V, and the face's flux adjoint
    double lk[5];
    if (c >= 0 && c < n0) {
      const double k = A.dt * __ldg(G.RW + c + 2) * A.kscale;
#pragma unroll
      for (int q = 0; q < 5; ++q) lk[q] = k * __ldg(A.lamK + base + c + q * A.nP);
    } else {
#pragma unroll
      for (int q = 0; q < 5; ++q) lk[q] = 0.0;
    }
    const bool face = lane >= 2 && lane <= 30 && c <= n0;
    const int fc = max(0, min(c, n0));
    const double wr = __ldg(G.WR + fc + 1), wl = __ldg(G.WL + fc + 2);
    double ll[5], lr[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const double lkm = __shfl_up_sync(FULL, lk[q], 1);
      ll[q] = lk[q] - lkm;  // the flux adjoint lF, until the call below
      lr[q] = 0.0;
    }
    if (face) {
      double l[5], r[5], lF[5];
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        l[q] = wm[q] + wr * sm[q];
        r[q] = w[q] - wl * sl[q];
        lF[q] = ll[q];
        ll[q] = 0.0;
      }
      bool diff = false;
      if (HLLC && A.df != nullptr && c < n0) diff = A.df[base + c] & 1;
      flux_adjoint<0, HLLC>(l, r, diff, lF, ph, ll, lr);
    } else {
#pragma unroll
      for (int q = 0; q < 5; ++q) ll[q] = 0.0;
    }
    // face c + 1 (lane + 1) gives this cell ll and the slope adjoint wr ll;
    // then the slope of every cell goes back to its three cells
    double gl[5], gr[5], a[5], ls[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      double llp = __shfl_down_sync(FULL, ll[q], 1);
      double wllp = __shfl_down_sync(FULL, wr * ll[q], 1);
      if (lane == 31) llp = wllp = 0.0;
      ls[q] = -wl * lr[q] + wllp;
      slope_coeffs((branches >> (2 * q)) & 3, sql, sqr, rdxl, rdxr, rcden, ph.theta, gl[q],
                   gr[q]);
      double from_left = __shfl_up_sync(FULL, gr[q] * ls[q], 1);
      double from_right = __shfl_down_sync(FULL, gl[q] * ls[q], 1);
      if (lane == 0) from_left = 0.0;
      if (lane == 31) from_right = 0.0;
      a[q] = (((lr[q] + from_left) + llp) + (gl[q] - gr[q]) * ls[q]) - from_right;
    }
    adj_flush(A, 0, base, 1, c, a);
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

// ---- Branch signature of a forward stage --------------------------------------
// The adjoint is the derivative of the branch the forward takes at every
// limiter argument, wave-speed maximum, HLLC decision and floor.  A central
// difference (J(U + eps d) - J(U - eps d)) / (2 eps) measures that derivative
// only if both forwards take the same branches everywhere.  The signature of
// a stage is an order-independent hash of all its decisions (a sum of mixed
// position-decision codes, added atomically) and a count per kind of
// decision, so that two forwards can be compared without storing either.
enum {
  BR_SLOPE0 = 0,     // limiter: zero slope (BR_SLOPE0 + branch, 4 kinds)
  BR_AP0 = 4,        // argmax of AP = max(0, vl + CSl, vr + CSr) (3 kinds)
  BR_AM0 = 7,        // argmax of AM (3 kinds)
  BR_HLLC = 10,      // the HLLC centre state taken (not the HLL flux)
  BR_AC_POS = 11,    // AC >= 0 (left centre state) among those
  BR_MD_POS = 12,    // MD > 0 in the HLLC centre speed
  BR_FLOOR = 13,     // a floored value of the stage input (N = N_min or E = 0)
  BR_FLAG = 14,      // a DIFFUSIVE_FLUX_I bit set
  BR_KINDS = 15
};

__device__ __forceinline__ unsigned long long branch_mix(unsigned long long x) {
  // splitmix64's finaliser (S. Vigna, public domain)
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Cell c of stage `stage` (W: its input primitives, compact): for each
// direction the limiter branch of each primitive's slope and the decisions of
// the flux through the cell's inner face (between c - 1 and c); the floors of
// W at c; the flags of df at c.  out[0]: hash, out[1]: decisions counted,
// out[2 + k]: count of kind k.
template <bool HLLC>
__global__ void branch_signature_kernel(const __grid_constant__ AdjDesc A,
                                        const __grid_constant__ Phys ph, int stage,
                                        unsigned long long* __restrict__ out) {
  __shared__ unsigned long long s_acc[2 + BR_KINDS];
  for (int i = threadIdx.x; i < 2 + BR_KINDS; i += blockDim.x) s_acc[i] = 0;
  __syncthreads();
  unsigned long long hash = 0, n_dec = 0;
  unsigned long long cnt[BR_KINDS];
#pragma unroll
  for (int k = 0; k < BR_KINDS; ++k) cnt[k] = 0;
  const long long nP = A.nP;
  auto note = [&](unsigned long long pos, int code, int kind) {
    hash += branch_mix(pos * 64ull + (unsigned long long)code);
    ++n_dec;
    if (kind >= 0) ++cnt[kind];
  };
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nP;
       c += (long long)gridDim.x * blockDim.x) {
    int t[3];
    {
      const unsigned cc = (unsigned)c, n0 = (unsigned)A.n[0], n1 = (unsigned)A.n[1];
      const unsigned r = cc / n0;
      t[0] = (int)(cc - r * n0);
      t[2] = (int)(r / n1);
      t[1] = (int)(r - (unsigned)t[2] * n1);
    }
    const unsigned long long base = ((unsigned long long)stage * 8ull) * (unsigned long long)nP;
    // floors of the stage input
    {
      const double N = A.W[c], E = A.W[4 * nP + c];
      const bool fl = (N == ph.nmin && A.W[nP + c] == 0.0 && A.W[2 * nP + c] == 0.0 &&
                       A.W[3 * nP + c] == 0.0) || E == 0.0;
      note((base + 0) * 8 + (unsigned long long)c, fl ? 1 : 0, fl ? BR_FLOOR : -1);
    }
    if (A.df) {
      const int f = A.df[c];
      note((base + 1) * 8 + (unsigned long long)c, f, -1);
      cnt[BR_FLAG] += __popc(f);
    }
#pragma unroll 1
    for (int D = 0; D < 3; ++D) {
      const long long st = D == 0 ? 1 : (D == 1 ? A.n[0] : (long long)A.n[0] * A.n[1]);
      const long long cbase = c - (long long)t[D] * st;  // cell 0 of this pencil
      const AxisGeo& G = A.geo[D];
      // the stencil cells t - 2 .. t + 1 along D (boundary maps)
      double w[4][5];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        bool neg;
        const int sj = bc_map(t[D] - 2 + j, A.n[D], A.bc[D][0], A.bc[D][1], neg);
#pragma unroll
        for (int q = 0; q < 5; ++q) w[j][q] = A.W[q * nP + cbase + sj * st];
        if (neg) w[j][1 + D] = -w[j][1 + D];
      }
      // slopes of cells t - 1 (stencil 0, 1, 2) and t (1, 2, 3) with branches
      double sl[2][5];
      int br[2][5];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int tt = t[D] - 1 + e + 2;
        const double dxl = __ldg(G.dXI + tt), dxr = __ldg(G.dXI + tt + 1);
        const double sql = __ldg(G.SQ + tt), sqr = __ldg(G.SQ + tt + 1);
        const double cden = __ldg(G.CDEN + tt), rdxl = __ldg(G.RDXI + tt);
        const double rdxr = __ldg(G.RDXI + tt + 1), rcden = __ldg(G.RCDEN + tt);
#pragma unroll
        for (int q = 0; q < 5; ++q)
          sl[e][q] = limited_slope_branch(w[e][q], w[e + 1][q], w[e + 2][q], dxl, dxr, sql, sqr,
                                          cden, rdxl, rdxr, rcden, ph.theta, ph.use_limiter,
                                          br[e][q]);
      }
      // the cell's own slopes (each cell counted once per direction)
#pragma unroll
      for (int q = 0; q < 5; ++q)
        note(((base + 2 + D) * 8 + (unsigned long long)q) * (unsigned long long)nP +
                 (unsigned long long)c,
             br[1][q], BR_SLOPE0 + br[1][q]);
      // the inner face of the cell
      const int tf = t[D] + 2;
      const double wr = __ldg(G.WR + tf - 1), wl = __ldg(G.WL + tf);
      double l[5], r[5];
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        l[q] = w[1][q] + wr * sl[0][q];
        r[q] = w[2][q] - wl * sl[1][q];
      }
      FaceState L, R;
      face_state<5>(l[0], l[1], l[2], l[3], l[4], ph, L);
      face_state<5>(r[0], r[1], r[2], r[3], r[4], ph, R);
      const double vl = D == 0 ? L.V1 : (D == 1 ? L.V2 : L.V3);
      const double vr = D == 0 ? R.V1 : (D == 1 ? R.V2 : R.V3);
      int ap = 0, am = 0;
      double AP = 0.0, AM = 0.0;
      if (vl + L.CS > AP) {
        AP = vl + L.CS;
        ap = 1;
      }
      if (vr + R.CS > AP) {
        AP = vr + R.CS;
        ap = 2;
      }
      if (-(vl - L.CS) > AM) {
        AM = -(vl - L.CS);
        am = 1;
      }
      if (-(vr - R.CS) > AM) {
        AM = -(vr - R.CS);
        am = 2;
      }
      int code = ap + 3 * am;
      cnt[BR_AP0 + ap] += 1;
      cnt[BR_AM0 + am] += 1;
      if (HLLC) {
        const bool diff = A.df != nullptr && ((A.df[c] >> D) & 1);
        const double ml = D == 0 ? L.S1 : (D == 1 ? L.S2 : L.S3);
        const double mr = D == 0 ? R.S1 : (D == 1 ? R.S2 : R.S3);
        const double fdl = L.D * vl, fdr = R.D * vr;
        const double fsl = ml * vl + L.P, fsr = mr * vr + R.P;
        const double MD = AP * R.D + AM * L.D - fdr + fdl;
        const double SN = AP * mr + AM * ml - fsr + fsl;
        const double AC = SN * (fmax2(MD, 0.0) / fmax2(MD * MD, kTiny));
        const bool centre = !diff && AP != 0.0 && AM != 0.0;
        code += 9 * ((int)centre + 2 * (int)(AC >= 0.0) + 4 * (int)(MD > 0.0));
        if (centre) {
          cnt[BR_HLLC] += 1;
          if (AC >= 0.0) cnt[BR_AC_POS] += 1;
        }
        if (MD > 0.0) cnt[BR_MD_POS] += 1;
      }
      note((base + 5 + D) * 8ull * (unsigned long long)nP + (unsigned long long)c, code, -1);
    }
  }
  atomicAdd(&s_acc[0], hash);
  atomicAdd(&s_acc[1], n_dec);
#pragma unroll
  for (int k = 0; k < BR_KINDS; ++k)
    if (cnt[k]) atomicAdd(&s_acc[2 + k], cnt[k]);
  __syncthreads();
  for (int i = threadIdx.x; i < 2 + BR_KINDS; i += blockDim.x)
    if (s_acc[i]) atomicAdd(&out[i], s_acc[i]);
}

}  // namespace gfx

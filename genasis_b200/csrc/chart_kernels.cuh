// chart_kernels.cuh -- the kernels of a chart of several bricks on one GPU
// besides the fused stages: the initial state with the exchanged ghost
// primitives, shock features across brick faces with ClearBoundary on the
// chart's own boundary only, and the ghost values at the end of a step.
//
// The reference splits a chart into equal bricks, one per MPI rank
// (Chart_SLD, Chart_Template.f90:440-460), and exchanges the ghost layers of
// the faces and edges between them (Chart_SLD__Form.f90:131-201, 324-1097).
// Here every brick of the chart lives in the same device memory, so no ghost
// is copied: a value outside a brick is read where it lives, in the proper
// cells of the brick across the face.  A brick's faces are either linked (to
// the neighbouring brick inside the chart, or across a periodic boundary of
// the chart to the brick at the other end) or carry the chart's boundary
// condition (OUTFLOW, REFLECTING).
#pragma once

#include "aux_kernels.cuh"

namespace gfx {

struct ChartBrick {
  Box box;              // bc: BC_NEIGHBOR on faces inside the chart
  int nb[3][2];         // the linked brick across each face (-1: none)
  double* U;            // conserved state, ghost layout
  const double* prim;   // initial primitives, ghost layout (chart_from_primitive)
  double* Pst;          // the kept primitives of the proper cells, compact
  const double* wn;     // primitives the last stage 2 stored, compact
  uint8_t* df;          // DIFFUSIVE_FLUX_I bits, compact
  long long v_off;      // prefix sum of nV over the bricks
  long long c_off;      // prefix sum of nP
};

__device__ __forceinline__ int chart_find(const ChartBrick* cb, int n, long long x, bool cells) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const long long off = cells ? cb[mid].c_off : cb[mid].v_off;
    if (off <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// The brick holding proper coordinates c of brick b (possibly outside it),
// crossing linked faces one axis after the other (an edge lands in the
// diagonal brick); c is moved into that brick's frame.  Axes whose face is
// not linked are left outside.
__device__ __forceinline__ int chart_owner(const ChartBrick* cb, int b, int* c) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int side = c[a] < 0 ? 0 : (c[a] >= cb[b].box.n[a] ? 1 : -1);
    if (side >= 0 && cb[b].nb[a][side] >= 0) {
      const int o = cb[b].nb[a][side];
      c[a] += side ? -cb[b].box.n[a] : cb[o].box.n[a];
      b = o;
    }
  }
  return b;
}

__device__ __forceinline__ bool chart_inside(const Box& bx, const int* c) {
  return c[0] >= 0 && c[1] >= 0 && c[2] >= 0 && c[0] < bx.n[0] && c[1] < bx.n[1] &&
         c[2] < bx.n[2];
}

// A ghost value is written by the exchange when every axis on which it is a
// ghost is linked and it is not a corner (the faces and edges of
// Chart_SLD__Form.f90:131-201); on one brick with periodic axes this is the
// rule of the single-brick ghost refresh.
__device__ __forceinline__ bool chart_reachable(const ChartBrick& B, const int* p) {
  int nghost = 0;
  bool ok = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const bool lo = p[d] < 0, hi = p[d] >= B.box.n[d];
    nghost += lo || hi;
    if ((lo && B.nb[d][0] < 0) || (hi && B.nb[d][1] < 0)) ok = false;
  }
  return ok && nghost > 0 && nghost < 3;
}

__device__ __forceinline__ long long ghost_index(const Box& bx, const int* p) {
  return (p[0] + 2) + (long long)bx.m[0] * ((p[1] + 2) + (long long)bx.m[1] * (p[2] + 2));
}

// ComputeFromPrimitive on every value of every brick after the exchange of
// the primitives (Integrator_C_PS__Form.f90:194-203): an exchange-reachable
// ghost takes the primitives of the cell it images; the primitives of the
// proper cells are kept as the first step's state.
__global__ void chart_from_primitive_kernel(const ChartBrick* __restrict__ cb, int n,
                                            long long total, Phys ph) {
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total;
       x += (long long)gridDim.x * blockDim.x) {
    const int b = chart_find(cb, n, x, false);
    const ChartBrick& B = cb[b];
    const long long v = x - B.v_off, nV = B.box.nV;
    int t[3];
    decode3(v, B.box.m[0], B.box.m[1], t[0], t[1], t[2]);
    int p[3] = {t[0] - 2, t[1] - 2, t[2] - 2};
    const double* src = B.prim;
    long long sv = v, snV = nV;
    if (chart_reachable(B, p)) {
      int c[3] = {p[0], p[1], p[2]};
      const ChartBrick& S = cb[chart_owner(cb, b, c)];
      src = S.prim;
      sv = ghost_index(S.box, c);
      snV = S.box.nV;
    }
    FaceState s;
    face_state<6>(src[sv], src[snV + sv], src[2 * snV + sv], src[3 * snV + sv],
                  src[4 * snV + sv], ph, s);
    B.U[v] = s.D;
    B.U[nV + v] = s.S1;
    B.U[2 * nV + v] = s.S2;
    B.U[3 * nV + v] = s.S3;
    B.U[4 * nV + v] = s.G;
    B.U[5 * nV + v] = s.DS;
    if (chart_inside(B.box, p)) {
      const long long c = p[0] + (long long)B.box.n[0] * (p[1] + (long long)B.box.n[1] * p[2]);
      const long long nP = B.box.nP;
      B.Pst[c] = s.N;
      B.Pst[nP + c] = s.V1;
      B.Pst[2 * nP + c] = s.V2;
      B.Pst[3 * nP + c] = s.V3;
      B.Pst[4 * nP + c] = s.E;
    }
  }
}

// Pressure and velocities of proper cell c of a brick (exact recovery from
// the conserved state, or the stored primitives with PST).
template <bool PST>
__device__ __forceinline__ void chart_p_v(const ChartBrick& B, const Phys& ph, const int* c,
                                          double& P, double* v) {
  Prim w;
  if (PST) {
    const long long i = c[0] + (long long)B.box.n[0] * (c[1] + (long long)B.box.n[1] * c[2]);
    const long long nP = B.box.nP;
    w.E = B.wn[4 * nP + i];
    w.V1 = B.wn[nP + i];
    w.V2 = B.wn[2 * nP + i];
    w.V3 = B.wn[3 * nP + i];
  } else {
    const long long o = ghost_index(B.box, c), nV = B.box.nV;
    Cons u{B.U[o], B.U[nV + o], B.U[2 * nV + o], B.U[3 * nV + o], B.U[4 * nV + o]};
    cons_to_prim_exact(u, w, ph.nmin);
  }
  P = ph.gm1 * w.E;
  v[0] = w.V1;
  v[1] = w.V2;
  v[2] = w.V3;
}

// The state of a chart of equal bricks (nbx x nby x nbz of bn0 x bn1 x bn2
// cells, brick b = ix + nbx (iy + nby iz)) as the feature detection reads
// it, by the chart's global proper coordinates: the primitives the last
// stage 2 stored (PST), or the conserved state; and the bricks' flags.
template <bool PST>
struct DetectChart {
  const ChartBrick* cb;
  int nbx, nby, bn0, bn1, bn2;
  __device__ __forceinline__ const ChartBrick& brick(int i, int j, int k, int& li, int& lj,
                                                     int& lk) const {
    const int bx = i / bn0, by = j / bn1, bz = k / bn2;
    li = i - bx * bn0;
    lj = j - by * bn1;
    lk = k - bz * bn2;
    return cb[bx + nbx * (by + nby * bz)];
  }
  // starts the copies of the raw values of cell (i, j, k) into dst, dst +
  // stride, ... (cp.async)
  __device__ __forceinline__ void load_async(int i, int j, int k, double* dst, int stride) const {
    int li, lj, lk;
    const ChartBrick& B = brick(i, j, k, li, lj, lk);
    if (PST) {
      const long long nP = B.box.nP, o = li + (long long)bn0 * (lj + (long long)bn1 * lk);
      cp_async8(dst, B.wn + 4 * nP + o);
      cp_async8(dst + stride, B.wn + nP + o);
      cp_async8(dst + 2 * stride, B.wn + 2 * nP + o);
      cp_async8(dst + 3 * stride, B.wn + 3 * nP + o);
    } else {
      const int c[3] = {li, lj, lk};
      const long long nV = B.box.nV, o = ghost_index(B.box, c);
#pragma unroll
      for (int q = 0; q < 5; ++q) cp_async8(dst + q * stride, B.U + q * nV + o);
    }
  }
  __device__ __forceinline__ uint8_t* flags(int i, int j, int k) const {
    int li, lj, lk;
    const ChartBrick& B = brick(i, j, k, li, lj, lk);
    return B.df + (li + (long long)bn0 * (lj + (long long)bn1 * lk));
  }
};

// DetectShocks_CSL_Kernel and the DIFFUSIVE_FLUX_I flags after
// ClearBoundary_CSL_Kernel (FluidFeatures_P__Kernel.f90:12-313) on a chart of
// equal bricks: the single brick's tiled pass (detect_tile) over the chart's
// global cells, each value read from the brick that holds it.  The reference
// applies ClearBoundary on the faces of the chart's boundary only
// (FluidFeatures_P__Form.f90:313-336: InnerBoundary = iaBrick == 1,
// OuterBoundary = iaBrick == nBricks), which in the chart's global
// coordinates is the single brick's rule: no flags within one cell of a chart
// face (periodic ones included), and shock bits only between cells of the
// chart, so that across a face inside the chart the bits and flags see the
// neighbouring and the diagonal bricks.  Grid: tiles of the whole chart.
template <bool PST>
__global__ void __launch_bounds__(kDetThreads, 3)
    chart_detect_features_kernel(const ChartBrick* __restrict__ cb, int nbx, int nby, int nbz,
                                 Phys ph, const int* skip) {
  if (skip && *skip) return;
  const DetectChart<PST> src{cb, nbx, nby, cb[0].box.n[0], cb[0].box.n[1], cb[0].box.n[2]};
  const int n2 = nbz * src.bn2, kb = blockIdx.z * kDetKZ;
  detect_tile<PST>(src, ph, nbx * src.bn0, nby * src.bn1, n2, blockIdx.x * kDetTX,
                   blockIdx.y * kDetTY, kb, min(kb + kDetKZ, n2));
}

// Ghost values at the end of a step: an exchange-reachable ghost takes the
// value of the cell it images, in whichever brick that lies (the reference's
// exchanged increments keep it equal to that cell); every other ghost keeps
// its conserved values through the floors of ComputeFromConserved.
// The ghost values of every brick, one thread per value of the bricks' ghost
// shells (laid end to end: brick b's starts at v_off - c_off; shell_cell
// orders a shell).
__device__ __forceinline__ int chart_find_shell(const ChartBrick* cb, int n, long long x) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (cb[mid].v_off - cb[mid].c_off <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void chart_ghost_refresh_kernel(const ChartBrick* __restrict__ cb, int n,
                                           long long total, Phys ph, const int* skip) {
  if (skip && *skip) return;
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total;
       x += (long long)gridDim.x * blockDim.x) {
    const int b = chart_find_shell(cb, n, x);
    const ChartBrick& B = cb[b];
    const long long u = x - (B.v_off - B.c_off), nV = B.box.nV;
    long long i, j, k;
    shell_cell(B.box, u, i, j, k);
    const long long v = i + (long long)B.box.m[0] * (j + (long long)B.box.m[1] * k);
    int p[3] = {(int)i - 2, (int)j - 2, (int)k - 2};
    if (chart_reachable(B, p)) {
      int c[3] = {p[0], p[1], p[2]};
      const ChartBrick& S = cb[chart_owner(cb, b, c)];
      const long long s = ghost_index(S.box, c), snV = S.box.nV;
#pragma unroll
      for (int f = 0; f < 6; ++f) B.U[f * nV + v] = S.U[f * snV + s];
    } else {
      Cons u{B.U[v], B.U[nV + v], B.U[2 * nV + v], B.U[3 * nV + v], B.U[4 * nV + v]};
      Prim w;
      cons_to_prim(u, w, ph.nmin);
      double P, CS, SB;
      eos_cell(w.N, w.E, ph, P, CS, &SB);
      B.U[v] = u.D;
      B.U[nV + v] = u.S1;
      B.U[2 * nV + v] = u.S2;
      B.U[3 * nV + v] = u.S3;
      B.U[4 * nV + v] = u.G;
      B.U[5 * nV + v] = SB * w.N;
    }
  }
}

}  // namespace gfx

// stage_kernel.cuh -- fused finite-volume stage for sm_100a.
//
// One CTA owns a TX x TY column of cells of one brick and marches it along z
// over [z0, z1).  Per z plane it
//   1. brings the next plane's primitives into a 3-plane ring in shared memory
//      (cons->prim on load for a conserved input) and the x / y halo of the
//      current plane, with the boundary conditions applied as index maps,
//   2. computes the limited slopes of x / y (current plane) and z (next plane),
//   3. computes the Riemann fluxes of every x, y face of the plane and of the
//      next z face (each face once),
//   4. forms the divergence increment of every cell in the reference's order
//      (x, then y, then z contributions) and applies the RK stage epilogue.
// This replaces the ~40 full-array sweeps per direction of
// IncrementDivergence_FV % Compute (IncrementDivergence_FV__Form.f90:344-412)
// and the Copy / MultiplyAdd / ComputeFromConserved sweeps of the RK driver
// (Step_RK_C_ASC__Template.f90:761-1281) with one pass per stage.
#pragma once

#include "fluid_physics.cuh"

namespace gfx {

constexpr int TX = 32;          // tile width (x), one warp per row
constexpr int TY = 8;           // tile rows (y)
constexpr int NT = TX * TY;     // threads per CTA
constexpr int PW = TX + 4;      // plane pitch with the 2-cell halo
constexpr int PH = TY + 4;
constexpr int PS = PW * PH;     // doubles per plane per variable

enum { MODE_INCREMENT = 0, MODE_STAGE1 = 1, MODE_STAGE2 = 2 };
enum { BC_OUTFLOW = 0, BC_REFLECTING = 1, BC_PERIODIC = 2 };

// Per-axis tables over the ghost-inclusive index t in [0, n + 4) (t = cell + 2).
struct AxisGeo {
  const double* W;     // cell width WL + WR (GeometryFlat_Kernel.f90:22-24)
  const double* WL;    // centre - inner edge
  const double* WR;    // outer edge - centre
  const double* dXI;   // X(t) - X(t-1), Difference_Kernel.f90 on the centres
  const double* SQ;    // dXI(t)^2
  const double* CDEN;  // (dXI(t) dXI(t+1)) (dXI(t) + dXI(t+1))
};

struct BrickDesc {
  int n[3];              // proper cells
  int m[3];              // n + 4
  int bc[3][2];
  long long nV;          // values per field of the ghost layout
  long long nP;          // values per field of the compact (proper-only) layout
  const double* U_in;    // conserved input, ghost layout
  double* U_out;         // conserved output (stage 2), ghost layout
  double* K;             // increment output (increment mode), ghost layout, 6 fields
  const double* P_in;    // primitive input, compact layout
  double* Yp;            // primitives of the intermediate state, compact
  double* H;             // U^n + B1 K1, compact
  const uint8_t* df;     // DIFFUSIVE_FLUX_I bits, compact (or null)
  double* fluence;       // [6][6][face_size] or null
  long long face_size;
  const double* dt;      // device scalar
  double weight;         // Runge-Kutta weight of the stage (fluence)
  unsigned long long* tsi_bits;  // max inverse CFL time, ordered bits
  const int* skip;       // device flag: nonzero = do nothing (finished evolve)
  AxisGeo geo[3];
};

struct WorkItem {
  int brick;
  int x0, y0;
  int z0, z1;
};

// Boundary condition as an index map for a coordinate g of an axis with n
// proper cells: the proper cell whose value the ghost holds, and whether the
// normal velocity is reversed (Chart_SL__Kernel.f90:12-113 mirror / reverse;
// periodic images as the ghost exchange of Chart_SLD__Form.f90:131-201).
__device__ __forceinline__ int bc_map(int g, int n, int bc_lo, int bc_hi, bool& neg) {
  neg = false;
  if (g >= 0 && g < n) return g;
  const int bc = (g < 0) ? bc_lo : bc_hi;
  int s;
  if (bc == BC_PERIODIC) {
    s = g % n;
    if (s < 0) s += n;
  } else {
    s = (g < 0) ? -1 - g : 2 * n - 1 - g;
    neg = (bc == BC_REFLECTING);
  }
  return max(0, min(n - 1, s));
}

template <int MODE, bool IN_PRIM, bool HLLC, bool GRAV, int NF>
struct StageSmem {
  static constexpr int kRing = 3 * 5 * PS;
  static constexpr int kSzc = 2 * 5 * NT;
  static constexpr int kFzc = 2 * NF * NT;
  static constexpr int kSx = 5 * TY * (TX + 2);
  static constexpr int kSy = 5 * (TY + 2) * TX;
  static constexpr int kFx = NF * TY * (TX + 1);
  static constexpr int kFy = NF * (TY + 1) * TX;
  static constexpr int kDoubles = kRing + kSzc + kFzc + kSx + kSy + kFx + kFy;
  static constexpr size_t kBytes = sizeof(double) * kDoubles;
};

// Loads the primitives of cell (gx, gy) of plane gz (all possibly ghosts) into
// a ring plane at local (ly, lx).
template <bool IN_PRIM>
__device__ __forceinline__ void load_cell(const BrickDesc& B, const Phys& ph, double* plane,
                                          int lx, int ly, int gx, int gy, int gz) {
  bool nx, ny, nz;
  const int sx = bc_map(gx, B.n[0], B.bc[0][0], B.bc[0][1], nx);
  const int sy = bc_map(gy, B.n[1], B.bc[1][0], B.bc[1][1], ny);
  const int sz = bc_map(gz, B.n[2], B.bc[2][0], B.bc[2][1], nz);
  Prim w;
  if (IN_PRIM) {
    const long long o = sx + (long long)B.n[0] * (sy + (long long)B.n[1] * sz);
    const double* p = B.P_in;
    w.N = __ldg(p + o);
    w.V1 = __ldg(p + B.nP + o);
    w.V2 = __ldg(p + 2 * B.nP + o);
    w.V3 = __ldg(p + 3 * B.nP + o);
    w.E = __ldg(p + 4 * B.nP + o);
  } else {
    const long long o =
        (sx + 2) + (long long)B.m[0] * ((sy + 2) + (long long)B.m[1] * (sz + 2));
    const double* u = B.U_in;
    Cons c;
    c.D = __ldg(u + o);
    c.S1 = __ldg(u + B.nV + o);
    c.S2 = __ldg(u + 2 * B.nV + o);
    c.S3 = __ldg(u + 3 * B.nV + o);
    c.G = __ldg(u + 4 * B.nV + o);
    cons_to_prim(c, w, ph.nmin);
  }
  if (nx) w.V1 = -w.V1;
  if (ny) w.V2 = -w.V2;
  if (nz) w.V3 = -w.V3;
  const int o = (ly + 2) * PW + (lx + 2);
  plane[o] = w.N;
  plane[PS + o] = w.V1;
  plane[2 * PS + o] = w.V2;
  plane[3 * PS + o] = w.V3;
  plane[4 * PS + o] = w.E;
}

// Reconstructed face states of the face between cells (im) and (ip) along one
// axis, IncrementDivergence_FV__Kernel.f90:70-90: V_IL = V(i-1) + dXR(i-1) dVdX(i-1),
// V_IR = V(i) - dXL(i) dVdX(i).
template <int NF>
__device__ __forceinline__ void face_states(const double* vm, const double* sm_, int stride_m,
                                            const double* vp, const double* sp, int stride_p,
                                            int sstride_m, int sstride_p, double wr, double wl,
                                            const Phys& ph, FaceState& L, FaceState& R) {
  double l[5], r[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    l[v] = vm[v * stride_m] + wr * sm_[v * sstride_m];
    r[v] = vp[v * stride_p] - wl * sp[v * sstride_p];
  }
  face_state<NF>(l[0], l[1], l[2], l[3], l[4], ph, L);
  face_state<NF>(r[0], r[1], r[2], r[3], r[4], ph, R);
}

__device__ __forceinline__ bool df_bit(const BrickDesc& B, int d, int gx, int gy, int gz) {
  if (B.df == nullptr) return false;
  if (gx < 0 || gy < 0 || gz < 0 || gx >= B.n[0] || gy >= B.n[1] || gz >= B.n[2]) return false;
  return (B.df[gx + (long long)B.n[0] * (gy + (long long)B.n[1] * gz)] >> d) & 1;
}

template <int NF>
__device__ __forceinline__ void record_fluence(const BrickDesc& B, int face, int a, int na,
                                               int b, const double* F, double factor) {
  if (B.fluence == nullptr) return;
  const long long o = a + (long long)na * b;
#pragma unroll
  for (int u = 0; u < NF; ++u) {
    double* p = B.fluence + ((long long)u * 6 + face) * B.face_size + o;
    *p = *p + factor * F[u];
  }
}

template <int MODE, bool IN_PRIM, bool HLLC, bool GRAV, int NF>
__global__ void __launch_bounds__(NT, 1)
    stage_kernel(const __grid_constant__ BrickDesc single, const BrickDesc* __restrict__ many,
                 const WorkItem* __restrict__ items, int n_items, int* __restrict__ counter,
                 const __grid_constant__ Phys ph) {
  using SM = StageSmem<MODE, IN_PRIM, HLLC, GRAV, NF>;
  extern __shared__ double smem[];
  double* ring = smem;
  double* szc = ring + SM::kRing;
  double* fzc = szc + SM::kSzc;
  double* sxs = fzc + SM::kFzc;
  double* sys = sxs + SM::kSx;
  double* fxs = sys + SM::kSy;
  double* fys = fxs + SM::kFx;
  __shared__ int s_item;
  __shared__ double s_red[NT / 32];

  const int tid = threadIdx.x;
  const int tx = tid % TX, ty = tid / TX;

  for (;;) {
    if (tid == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n_items) break;
    const WorkItem W = items[it];
    const BrickDesc& B = many ? many[W.brick] : single;
    if (B.skip && *B.skip) {
      __syncthreads();
      continue;
    }
    const double dt = *B.dt;
    const int x0 = W.x0, y0 = W.y0, z0 = W.z0, z1 = W.z1;
    const int n0 = B.n[0], n1 = B.n[1], n2 = B.n[2];
    const int gx = x0 + tx, gy = y0 + ty;
    const bool own = (gx < n0) && (gy < n1);
    double tsi_max = -DBL_MAX;

    auto slot = [](int p) { return ((p % 3) + 3) % 3; };
    auto plane_ptr = [&](int p) { return ring + slot(p) * 5 * PS; };
    const int c_off = (ty + 2) * PW + (tx + 2);  // own cell in a plane

    // z slope at plane p (p-1, p, p+1 resident) for the own column -> dst[5][NT]
    auto z_slope = [&](int p, double* dst) {
      const double* a = plane_ptr(p - 1);
      const double* b = plane_ptr(p);
      const double* c = plane_ptr(p + 1);
      const int t = p + 2;
      const AxisGeo& G = B.geo[2];
      const double dxl = __ldg(G.dXI + t), dxr = __ldg(G.dXI + t + 1);
      const double sql = __ldg(G.SQ + t), sqr = __ldg(G.SQ + t + 1), cden = __ldg(G.CDEN + t);
#pragma unroll
      for (int v = 0; v < 5; ++v)
        dst[v * NT + tid] = limited_slope(a[v * PS + c_off], b[v * PS + c_off],
                                          c[v * PS + c_off], dxl, dxr, sql, sqr, cden,
                                          ph.theta, ph.use_limiter);
    };
    // z face between planes p-1 and p for the own column -> dst[NF][NT]
    auto z_face = [&](int p, const double* s_m, const double* s_p, double* dst) {
      const double* a = plane_ptr(p - 1);
      const double* b = plane_ptr(p);
      const AxisGeo& G = B.geo[2];
      FaceState L, R;
      face_states<NF>(a + c_off, s_m + tid, PS, b + c_off, s_p + tid, PS, NT, NT,
                      __ldg(G.WR + p + 1), __ldg(G.WL + p + 2), ph, L, R);
      double F[NF];
      riemann_flux<2, HLLC, NF>(L, R, HLLC && df_bit(B, 2, gx, gy, p), F);
#pragma unroll
      for (int u = 0; u < NF; ++u) dst[u * NT + tid] = F[u];
      if (own && (p == 0 || p == n2))
        record_fluence<NF>(B, p == 0 ? 4 : 5, gx, n0, gy, F, B.weight * dt);
    };

    // ---- prologue: planes z0-2 .. z0+1, slopes at z0-1, z0, face z0 ----
    load_cell<IN_PRIM>(B, ph, plane_ptr(z0 - 2), tx, ty, gx, gy, z0 - 2);
    load_cell<IN_PRIM>(B, ph, plane_ptr(z0 - 1), tx, ty, gx, gy, z0 - 1);
    load_cell<IN_PRIM>(B, ph, plane_ptr(z0), tx, ty, gx, gy, z0);
    __syncthreads();
    z_slope(z0 - 1, szc);
    __syncthreads();
    load_cell<IN_PRIM>(B, ph, plane_ptr(z0 + 1), tx, ty, gx, gy, z0 + 1);
    __syncthreads();
    z_slope(z0, szc + 5 * NT);
    __syncthreads();
    z_face(z0, szc, szc + 5 * NT, fzc);
    __syncthreads();
    int scur = 1, fcur = 0;

    for (int k = z0; k < z1; ++k) {
      double* pk = plane_ptr(k);
      // (1) next plane centre, current plane halo
      load_cell<IN_PRIM>(B, ph, plane_ptr(k + 2), tx, ty, gx, gy, k + 2);
      if (tid < 4 * TX) {
        const int s = tid / TX, lx = tid % TX;
        const int ly = (s < 2) ? s - 2 : TY + s - 2;
        load_cell<IN_PRIM>(B, ph, pk, lx, ly, x0 + lx, y0 + ly, k);
      } else if (tid < 4 * TX + 4 * TY) {
        const int j = tid - 4 * TX;
        const int ly = j / 4, s = j % 4;
        const int lx = (s < 2) ? s - 2 : TX + s - 2;
        load_cell<IN_PRIM>(B, ph, pk, lx, ly, x0 + lx, y0 + ly, k);
      }
      __syncthreads();

      // (2) slopes: x [TY][TX+2], y [TY+2][TX], z at k+1
      {
        constexpr int NXS = TY * (TX + 2), NYS = (TY + 2) * TX;
        constexpr int PXS = (NXS + 31) / 32 * 32, PYS = (NYS + 31) / 32 * 32;
        constexpr int NITEMS = PXS + PYS + NT;
        for (int i = tid; i < NITEMS; i += NT) {
          if (i < PXS) {
            if (i >= NXS) continue;
            const int ly = i / (TX + 2), lx = i % (TX + 2) - 1;
            const int cx = x0 + lx;
            if (cx > n0 || y0 + ly >= n1) continue;
            const AxisGeo& G = B.geo[0];
            const int t = cx + 2;
            const double dxl = __ldg(G.dXI + t), dxr = __ldg(G.dXI + t + 1);
            const double sql = __ldg(G.SQ + t), sqr = __ldg(G.SQ + t + 1),
                         cden = __ldg(G.CDEN + t);
            const int o = (ly + 2) * PW + (lx + 2);
#pragma unroll
            for (int v = 0; v < 5; ++v)
              sxs[(v * TY + ly) * (TX + 2) + lx + 1] =
                  limited_slope(pk[v * PS + o - 1], pk[v * PS + o], pk[v * PS + o + 1], dxl,
                                dxr, sql, sqr, cden, ph.theta, ph.use_limiter);
          } else if (i < PXS + PYS) {
            const int j = i - PXS;
            if (j >= NYS) continue;
            const int ly = j / TX - 1, lx = j % TX;
            const int cy = y0 + ly;
            if (cy > n1 || x0 + lx >= n0) continue;
            const AxisGeo& G = B.geo[1];
            const int t = cy + 2;
            const double dxl = __ldg(G.dXI + t), dxr = __ldg(G.dXI + t + 1);
            const double sql = __ldg(G.SQ + t), sqr = __ldg(G.SQ + t + 1),
                         cden = __ldg(G.CDEN + t);
            const int o = (ly + 2) * PW + (lx + 2);
#pragma unroll
            for (int v = 0; v < 5; ++v)
              sys[(v * (TY + 2) + ly + 1) * TX + lx] =
                  limited_slope(pk[v * PS + o - PW], pk[v * PS + o], pk[v * PS + o + PW], dxl,
                                dxr, sql, sqr, cden, ph.theta, ph.use_limiter);
          } else {
            z_slope(k + 1, szc + (scur ^ 1) * 5 * NT);
          }
        }
      }
      __syncthreads();

      // (3) faces: x [TY][TX+1], y [TY+1][TX], z face k+1
      {
        constexpr int NXF = TY * (TX + 1), NYF = (TY + 1) * TX;
        constexpr int PXF = (NXF + 31) / 32 * 32, PYF = (NYF + 31) / 32 * 32;
        constexpr int NITEMS = PXF + PYF + NT;
        const double factor = B.weight * dt;
        for (int i = tid; i < NITEMS; i += NT) {
          if (i < PXF) {
            if (i >= NXF) continue;
            const int ly = i / (TX + 1), lx = i % (TX + 1);
            const int cx = x0 + lx, cy = y0 + ly;
            if (cx > n0 || cy >= n1) continue;
            const AxisGeo& G = B.geo[0];
            const int o = (ly + 2) * PW + (lx + 2);
            const double* sl = sxs + ly * (TX + 2) + lx;  // slope of cell lx-1
            FaceState L, R;
            face_states<NF>(pk + o - 1, sl, PS, pk + o, sl + 1, PS, TY * (TX + 2),
                            TY * (TX + 2), __ldg(G.WR + cx + 1), __ldg(G.WL + cx + 2), ph, L,
                            R);
            double F[NF];
            riemann_flux<0, HLLC, NF>(L, R, HLLC && df_bit(B, 0, cx, cy, k), F);
#pragma unroll
            for (int u = 0; u < NF; ++u) fxs[(u * TY + ly) * (TX + 1) + lx] = F[u];
            if (cx == 0 || cx == n0) record_fluence<NF>(B, cx == 0 ? 0 : 1, cy, n1, k, F, factor);
          } else if (i < PXF + PYF) {
            const int j = i - PXF;
            if (j >= NYF) continue;
            const int ly = j / TX, lx = j % TX;
            const int cx = x0 + lx, cy = y0 + ly;
            if (cy > n1 || cx >= n0) continue;
            const AxisGeo& G = B.geo[1];
            const int o = (ly + 2) * PW + (lx + 2);
            const double* sl = sys + ly * TX + lx;  // slope of cell ly-1
            FaceState L, R;
            face_states<NF>(pk + o - PW, sl, PS, pk + o, sl + TX, PS, (TY + 2) * TX,
                            (TY + 2) * TX, __ldg(G.WR + cy + 1), __ldg(G.WL + cy + 2), ph, L,
                            R);
            double F[NF];
            riemann_flux<1, HLLC, NF>(L, R, HLLC && df_bit(B, 1, cx, cy, k), F);
#pragma unroll
            for (int u = 0; u < NF; ++u) fys[(u * (TY + 1) + ly) * TX + lx] = F[u];
            if (cy == 0 || cy == n1) record_fluence<NF>(B, cy == 0 ? 2 : 3, cx, n0, k, F, factor);
          } else {
            z_face(k + 1, szc + scur * 5 * NT, szc + (scur ^ 1) * 5 * NT,
                   fzc + (fcur ^ 1) * NF * NT);
          }
        }
      }
      __syncthreads();

      // (4) cell update and stage epilogue
      if (own) {
        const double w0 = __ldg(B.geo[0].W + gx + 2), w1 = __ldg(B.geo[1].W + gy + 2),
                     w2 = __ldg(B.geo[2].W + k + 2);
        const double vol = w0 * w1 * w2;
        const double ax = w1 * w2, ay = w2 * w0, az = w0 * w1;
        const double* fzm = fzc + fcur * NF * NT;
        const double* fzp = fzc + (fcur ^ 1) * NF * NT;
        const long long gidx =
            (gx + 2) + (long long)B.m[0] * ((gy + 2) + (long long)B.m[1] * (k + 2));
        const long long cidx = gx + (long long)n0 * (gy + (long long)n1 * k);
        double Kc[NF];
#pragma unroll
        for (int u = 0; u < NF; ++u) {
          const double dxu =
              dt * (ax * fxs[(u * TY + ty) * (TX + 1) + tx] -
                    ax * fxs[(u * TY + ty) * (TX + 1) + tx + 1]) / vol;
          const double dyu = dt * (ay * fys[(u * (TY + 1) + ty) * TX + tx] -
                                   ay * fys[(u * (TY + 1) + ty + 1) * TX + tx]) / vol;
          const double dzu = dt * (az * fzm[u * NT + tid] - az * fzp[u * NT + tid]) / vol;
          if (MODE == MODE_INCREMENT) {
            double* kp = B.K + (long long)u * B.nV + gidx;
            *kp = *kp + dxu + dyu + dzu;
          } else {
            Kc[u] = dxu + dyu + dzu;
          }
        }
        if (MODE != MODE_INCREMENT) {
          const double N = pk[c_off], V1 = pk[PS + c_off], V2 = pk[2 * PS + c_off],
                       V3 = pk[3 * PS + c_off], E = pk[4 * PS + c_off];
          if (GRAV) {
            // ApplyGravity_F (ApplyGravity_F__Command.f90:124-264) with the
            // uniform gradient (0, 0, a); the x and y momentum terms subtract
            // an exact +0.
            const double a = ph.accel;
            Kc[3] = Kc[3] - N * a * dt;
            Kc[4] = Kc[4] - N * (V1 * 0.0 + V2 * 0.0 + V3 * a) * dt;
          }
          if (MODE == MODE_STAGE1) {
            Cons u;
            {
              const double* U = B.U_in;
              Cons raw;
              raw.D = __ldg(U + gidx);
              raw.S1 = __ldg(U + B.nV + gidx);
              raw.S2 = __ldg(U + 2 * B.nV + gidx);
              raw.S3 = __ldg(U + 3 * B.nV + gidx);
              raw.G = __ldg(U + 4 * B.nV + gidx);
              if (IN_PRIM) {
                u = raw;
              } else {
                Prim w{N, V1, V2, V3, E};
                u = floored_cons(raw, w, ph.nmin);
              }
            }
            // Y = Solution + A21 K1 (A21 = 1); Solution + B1 K1 (B1 = 1/2)
            Cons y{u.D + Kc[0], u.S1 + Kc[1], u.S2 + Kc[2], u.S3 + Kc[3], u.G + Kc[4]};
            double* H = B.H;
            H[cidx] = u.D + 0.5 * Kc[0];
            H[B.nP + cidx] = u.S1 + 0.5 * Kc[1];
            H[2 * B.nP + cidx] = u.S2 + 0.5 * Kc[2];
            H[3 * B.nP + cidx] = u.S3 + 0.5 * Kc[3];
            H[4 * B.nP + cidx] = u.G + 0.5 * Kc[4];
            Prim wy;
            cons_to_prim(y, wy, ph.nmin);
            double* Y = B.Yp;
            Y[cidx] = wy.N;
            Y[B.nP + cidx] = wy.V1;
            Y[2 * B.nP + cidx] = wy.V2;
            Y[3 * B.nP + cidx] = wy.V3;
            Y[4 * B.nP + cidx] = wy.E;
          } else {  // MODE_STAGE2: Solution + B2 K2, then ComputeFromConserved
            const double* H = B.H;
            Cons u{H[cidx] + 0.5 * Kc[0], H[B.nP + cidx] + 0.5 * Kc[1],
                   H[2 * B.nP + cidx] + 0.5 * Kc[2], H[3 * B.nP + cidx] + 0.5 * Kc[3],
                   H[4 * B.nP + cidx] + 0.5 * Kc[4]};
            Prim w;
            cons_to_prim(u, w, ph.nmin);
            double P, CS, SB;
            eos_cell(w.N, w.E, ph, P, CS, &SB);
            double* U = B.U_out;
            U[gidx] = u.D;
            U[B.nV + gidx] = u.S1;
            U[2 * B.nV + gidx] = u.S2;
            U[3 * B.nV + gidx] = u.S3;
            U[4 * B.nV + gidx] = u.G;
            U[5 * B.nV + gidx] = SB * w.N;
            tsi_max = fmax2(tsi_max, inverse_cfl_time(w, CS, w0, w1, w2));
          }
        }
      }
      __syncthreads();
      scur ^= 1;
      fcur ^= 1;
    }

    if (MODE == MODE_STAGE2) {
      double v = tsi_max;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v = fmax2(v, __shfl_xor_sync(0xffffffffu, v, o));
      if ((tid & 31) == 0) s_red[tid >> 5] = v;
      __syncthreads();
      if (tid == 0) {
        double m = s_red[0];
        for (int w = 1; w < NT / 32; ++w) m = fmax2(m, s_red[w]);
        atomicMax(B.tsi_bits, ordered_bits(m));
      }
      __syncthreads();
    }
  }
}

}  // namespace gfx

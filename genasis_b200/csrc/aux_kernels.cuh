// aux_kernels.cuh -- the small kernels around the fused stages: state
// conversion over every value, shock features, ghost refresh, CFL reduction
// and the device-side time-step bookkeeping.
#pragma once

#include "stage_kernel.cuh"

namespace gfx {

struct Box {
  int n[3], m[3], bc[3][2];
  long long nV, nP;
};

// Coordinates (i, j, k) of the linear index v over an a x b x ... box, x
// fastest.  Every brick has fewer than 2^31 values (gfx_fluid_create checks),
// so 32-bit division suffices; the 64-bit one would be emulated.
__device__ __forceinline__ void decode3(long long v, int a, int b, int& i, int& j, int& k) {
  const unsigned u = (unsigned)v, ua = (unsigned)a, ub = (unsigned)b;
  const unsigned r = u / ua;
  i = (int)(u - r * ua);
  k = (int)(r / ub);
  j = (int)(r - (unsigned)k * ub);
}

__device__ __forceinline__ bool periodic_reachable(const Box& b, int i, int j, int k, int& si,
                                                   int& sj, int& sk) {
  // A ghost value is written by the single-brick exchange (faces and edges,
  // Chart_SLD__Form.f90:131-201) when every axis on which it is a ghost is
  // periodic and it is not a corner.
  const int t[3] = {i, j, k};
  int s[3], nghost = 0;
  bool ok = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int p = t[d] - 2;
    const bool ghost = (p < 0 || p >= b.n[d]);
    nghost += ghost;
    if (ghost && b.bc[d][0] != BC_PERIODIC) ok = false;
    s[d] = ghost ? ((p % b.n[d] + b.n[d]) % b.n[d]) + 2 : t[d];
  }
  si = s[0];
  sj = s[1];
  sk = s[2];
  return ok && nghost > 0 && nghost < 3;
}

// Fluid_P_I % ComputeFromPrimitive on every value after the periodic
// exchange of the primitives (Integrator_C_PS__Form.f90:194-203); keeps the
// primitives of the proper cells (with N clipped at 0 as Compute_D_S_G does)
// as the next step's state.
__global__ void from_primitive_kernel(Box b, Phys ph, const double* __restrict__ prim,
                                      double* __restrict__ U, double* __restrict__ Pst) {
  const long long nV = b.nV;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
       v += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    decode3(v, b.m[0], b.m[1], i, j, k);
    int si, sj, sk;
    long long src = v;
    if (periodic_reachable(b, i, j, k, si, sj, sk))
      src = si + (long long)b.m[0] * (sj + (long long)b.m[1] * sk);
    FaceState s;
    face_state<6>(prim[src], prim[nV + src], prim[2 * nV + src], prim[3 * nV + src],
                  prim[4 * nV + src], ph, s);
    U[v] = s.D;
    U[nV + v] = s.S1;
    U[2 * nV + v] = s.S2;
    U[3 * nV + v] = s.S3;
    U[4 * nV + v] = s.G;
    U[5 * nV + v] = s.DS;
    const int pi = i - 2, pj = j - 2, pk = k - 2;
    if (pi >= 0 && pj >= 0 && pk >= 0 && pi < b.n[0] && pj < b.n[1] && pk < b.n[2]) {
      const long long c = pi + (long long)b.n[0] * (pj + (long long)b.n[1] * pk);
      Pst[c] = s.N;
      Pst[b.nP + c] = s.V1;
      Pst[2 * b.nP + c] = s.V2;
      Pst[3 * b.nP + c] = s.V3;
      Pst[4 * b.nP + c] = s.E;
    }
  }
}

// Fluid_P_I % ComputeFromConserved on every value: floors written back to U,
// DS recomputed, optional primitives and (P, CS, SB).
__global__ void to_primitive_kernel(Box b, Phys ph, double* __restrict__ U,
                                    double* __restrict__ prim, double* __restrict__ aux) {
  const long long nV = b.nV;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nV;
       v += (long long)gridDim.x * blockDim.x) {
    Cons u{U[v], U[nV + v], U[2 * nV + v], U[3 * nV + v], U[4 * nV + v]};
    Prim w;
    cons_to_prim(u, w, ph.nmin);
    double P, CS, SB;
    eos_cell(w.N, w.E, ph, P, CS, &SB);
    U[v] = u.D;
    U[nV + v] = u.S1;
    U[2 * nV + v] = u.S2;
    U[3 * nV + v] = u.S3;
    U[4 * nV + v] = u.G;
    U[5 * nV + v] = SB * w.N;
    if (prim) {
      prim[v] = w.N;
      prim[nV + v] = w.V1;
      prim[2 * nV + v] = w.V2;
      prim[3 * nV + v] = w.V3;
      prim[4 * nV + v] = w.E;
    }
    if (aux) {
      aux[v] = P;
      aux[nV + v] = CS;
      aux[2 * nV + v] = SB;
    }
  }
}

// Ghost values at the end of a step: exchange-reachable periodic ghosts take
// their image (the reference adds the image's exchanged increments to an
// image copy); every other ghost keeps its conserved values through the
// floors of ComputeFromConserved, which also recompute its DS.
__device__ __forceinline__ void ghost_refresh_value(const Box& b, const Phys& ph, double* U,
                                                    long long v) {
  const long long nV = b.nV;
  int i, j, k;
  decode3(v, b.m[0], b.m[1], i, j, k);
  const bool ghost =
      i < 2 || j < 2 || k < 2 || i >= b.n[0] + 2 || j >= b.n[1] + 2 || k >= b.n[2] + 2;
  if (!ghost) return;
  int si, sj, sk;
  if (periodic_reachable(b, i, j, k, si, sj, sk)) {
    const long long s = si + (long long)b.m[0] * (sj + (long long)b.m[1] * sk);
#pragma unroll
    for (int f = 0; f < 6; ++f) U[f * nV + v] = U[f * nV + s];
  } else {
    Cons u{U[v], U[nV + v], U[2 * nV + v], U[3 * nV + v], U[4 * nV + v]};
    Prim w;
    cons_to_prim(u, w, ph.nmin);
    double P, CS, SB;
    eos_cell(w.N, w.E, ph, P, CS, &SB);
    U[v] = u.D;
    U[nV + v] = u.S1;
    U[2 * nV + v] = u.S2;
    U[3 * nV + v] = u.S3;
    U[4 * nV + v] = u.G;
    U[5 * nV + v] = SB * w.N;
  }
}

__global__ void ghost_refresh_kernel(Box b, Phys ph, double* __restrict__ U) {
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < b.nV;
       v += (long long)gridDim.x * blockDim.x)
    ghost_refresh_value(b, ph, U, v);
}

// The ghost-layout coordinates of the u-th value (u < nV - nP) of the ghost
// shell: the two z ghost planes at each end, then the y ghost rows and the x
// ghost columns of the proper planes.
__device__ __forceinline__ void shell_cell(const Box& b, long long u, long long& i, long long& j,
                                           long long& k) {
  const long long m0 = b.m[0], m1 = b.m[1], m2 = b.m[2];
  const long long n1 = b.n[1], n2 = b.n[2];
  const long long gz = 4 * m0 * m1, gy = 4 * m0 * n2;
  if (u < gz) {  // planes k = 0, 1, m2 - 2, m2 - 1
    const long long s = u / (m0 * m1), r = u - s * m0 * m1;
    k = (s < 2) ? s : m2 - 4 + s;
    j = r / m0;
    i = r - j * m0;
  } else if (u < gz + gy) {  // rows j = 0, 1, m1 - 2, m1 - 1 of planes 2 .. m2 - 3
    const long long w = u - gz, s = w / (m0 * n2), r = w - s * m0 * n2;
    j = (s < 2) ? s : m1 - 4 + s;
    k = 2 + r / m0;
    i = r - (k - 2) * m0;
  } else {  // columns i = 0, 1, m0 - 2, m0 - 1 of rows 2 .. m1 - 3
    const long long w = u - gz - gy, s = w / (n1 * n2), r = w - s * n1 * n2;
    i = (s < 2) ? s : m0 - 4 + s;
    k = 2 + r / n1;
    j = 2 + (r - (k - 2) * n1);
  }
}

// Its ghost-layout index.
__device__ __forceinline__ long long shell_value(const Box& b, long long u) {
  long long i, j, k;
  shell_cell(b, u, i, j, k);
  return i + (long long)b.m[0] * (j + (long long)b.m[1] * k);
}

// The same, visiting only the ghost shell.
__global__ void ghost_refresh_shell_kernel(Box b, Phys ph, double* __restrict__ U) {
  for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < b.nV - b.nP;
       u += (long long)gridDim.x * blockDim.x)
    ghost_refresh_value(b, ph, U, shell_value(b, u));
}

// The same over the values [v0, v1) only (whole planes of a z slab).
__global__ void ghost_refresh_range_kernel(Box b, Phys ph, double* __restrict__ U, long long v0,
                                           long long v1) {
  for (long long v = v0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; v < v1;
       v += (long long)gridDim.x * blockDim.x)
    ghost_refresh_value(b, ph, U, v);
}

// One brick of a batch for the element-wise kernels: its box, its state and
// feature storage, and the offsets of its values in the batch's flat ranges.
struct BatchBrick {
  Box box;
  double* U;
  uint8_t* df;
  const int* skip;
  long long v_off;  // prefix sum of nV
  long long c_off;  // prefix sum of nP
};

__device__ __forceinline__ int find_brick(const BatchBrick* bb, int n, long long x, bool cells) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const long long off = cells ? bb[mid].c_off : bb[mid].v_off;
    if (off <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// The ghost shells of every brick of a batch, one thread per shell value
// (the shells are laid end to end: brick b's starts at v_off - c_off).
__global__ void batch_ghost_refresh_kernel(const BatchBrick* __restrict__ bb, int n,
                                           long long total, Phys ph) {
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total;
       x += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (bb[mid].v_off - bb[mid].c_off <= x) lo = mid;
      else hi = mid - 1;
    }
    const BatchBrick& B = bb[lo];
    if (B.skip && *B.skip) continue;
    ghost_refresh_value(B.box, ph, B.U, shell_value(B.box, x - (B.v_off - B.c_off)));
  }
}

// Tiles of the feature detection over the planes [k0, k1): 32 x 8 cells of a
// plane per CTA, marching through up to kDetKZ planes of z.  The CTA has one
// thread per cell of the tile with a one-cell halo (34 x 10, in 12 warps).
constexpr int kDetTX = 32, kDetTY = 8, kDetKZ = 16;
constexpr int kDetRX = kDetTX + 2, kDetRY = kDetTY + 2, kDetNR = kDetRX * kDetRY;
constexpr int kDetThreads = (kDetNR + 31) / 32 * 32;

inline dim3 detect_grid(const Box& b, int k0, int k1) {
  return dim3((b.n[0] + kDetTX - 1) / kDetTX, (b.n[1] + kDetTY - 1) / kDetTY,
              (k1 - k0 + kDetKZ - 1) / kDetKZ);
}

// The state of one brick as the feature detection reads it: the compact
// primitives (PST: E, V1, V2, V3 at N's place skipped) or the conserved
// fields of the ghost layout, by proper coordinates; and its flags.  Offsets
// fit in 32 bits (every brick has fewer than 2^31 values).
template <bool PST>
struct DetectBrick {
  const double* F[5];
  int pitch, plane, gh;
  int n0, n1;
  uint8_t* df;
  __device__ DetectBrick(const Box& b, const double* U, const double* Pst, uint8_t* df_)
      : pitch(PST ? b.n[0] : b.m[0]), plane(PST ? b.n[0] * b.n[1] : b.m[0] * b.m[1]),
        gh(PST ? 0 : 2), n0(b.n[0]), n1(b.n[1]), df(df_) {
    const long long fs = PST ? b.nP : b.nV;
    F[0] = PST ? Pst + 4 * fs : U;  // E, or D
    F[1] = (PST ? Pst : U) + fs;
    F[2] = F[1] + fs;
    F[3] = F[2] + fs;
    F[4] = F[3] + fs;  // G (U only)
  }
  // starts the copies of the raw values of cell (i, j, k) into dst, dst +
  // stride, ... (cp.async)
  __device__ __forceinline__ void load_async(int i, int j, int k, double* dst, int stride) const {
    const int o = (i + gh) + pitch * (j + gh) + plane * (k + gh);
    cp_async8(dst, F[0] + o);
    cp_async8(dst + stride, F[1] + o);
    cp_async8(dst + 2 * stride, F[2] + o);
    cp_async8(dst + 3 * stride, F[3] + o);
    if (!PST) cp_async8(dst + 4 * stride, F[4] + o);
  }
  __device__ __forceinline__ uint8_t* flags(int i, int j, int k) const {
    return df + (i + n0 * (j + n1 * k));
  }
};

// Shock bits and DIFFUSIVE_FLUX_I flags of the proper cells of a tile of a box
// of n0 x n1 x n2 cells in one pass: DetectShocks_CSL_Kernel
// (FluidFeatures_P__Kernel.f90:12-186) sets bit e of a cell for a shock along
// e between it and the cell before it along e; after ClearBoundary_CSL_Kernel
// (:189-313) only cells not next to a face keep flags, and
// flag d is set by a shock along e != d at x, x + e_e, x - e_d or
// x + e_e - e_d (the positions DetectShocks_CSL_Kernel writes).  The state is
// the one that `src` reads (a brick, or a chart of bricks by its global
// coordinates; raw values: E, V1, V2, V3 with PST, else D, S1, S2, S3, G).
// The tile of this block: columns i0 .. i0 + 31, rows j0 .. j0 + 7, planes
// [kb, ke) (at most kDetKZ).  For every plane kk each thread recovers pressure and
// velocities of its halo-tile cell (the values of planes kk + 1 .. kk + D - 1
// are on their way meanwhile: asynchronous copies into a ring of D planes in
// shared memory, each thread reading back only its own copies, so that the
// ring needs no barrier of its own), forms the cell's shock bits from the -x and
// -y neighbours in shared memory and the -z neighbour kept in registers, and
// the CTA keeps three planes of bits in a ring; the flags of plane kk - 1
// (threads 0-255, one per tile cell) then read bits of planes kk - 2 to kk
// only.  A bit that no flag reads (x at the left halo column, y at the bottom
// halo row, z at the first plane) is left zero, and so is every bit outside
// the box, which only cells without flags would read.  Reads the state of
// planes kb - 1 to ke (those that exist); writes the flags of planes
// [kb, ke).
template <bool PST, class Src>
__device__ __forceinline__ void detect_tile(const Src& src, const Phys& ph, int n0, int n1,
                                            int n2, int i0, int j0, int kb, int ke) {
  constexpr int RX = kDetRX, NR = kDetNR, NT = kDetThreads;
  // planes in flight: three of the four primitive fields; two of the five
  // conserved ones (the static shared memory stays under 48 KB)
  constexpr int NRAW = PST ? 4 : 5, D = PST ? 3 : 2;
  __shared__ double sP[NR], sV1[NR], sV2[NR];
  __shared__ uint8_t sS[3][NR];
  __shared__ double sRaw[D][NRAW][NT];
  const int tid = threadIdx.x;
  const double thr = ph.shock_threshold;
  // the halo-tile cell of this thread
  const int rx = tid % RX, ry = tid / RX;
  const int gi = i0 - 1 + rx, gj = j0 - 1 + ry;
  const bool ok = tid < NR && gi >= 0 && gj >= 0 && gi < n0 && gj < n1;
  const bool has_xm = rx >= 1 && gi >= 1, has_ym = ry >= 1 && gj >= 1;
  // plane kk into ring slot `slot`: one group of copies per plane, empty
  // where there is nothing to read, so that the groups count planes
  auto fetch = [&](int kk, int slot) {
    if (ok && kk >= 0 && kk < n2 && kk <= ke) src.load_async(gi, gj, kk, &sRaw[slot][0][tid], NT);
    cp_async_commit();
  };
#pragma unroll
  for (int q = 0; q < D - 1; ++q) fetch(kb - 1 + q, q);
  double Pz = 0.0, Vz = 0.0;  // the plane below
  // the output cell of this thread (threads 0-255)
  const int ox = tid % kDetTX, oy = tid / kDetTX;
  const int i = i0 + ox, j = j0 + oy, ro = (ox + 1) + RX * (oy + 1);
  const bool out_in = tid < kDetTX * kDetTY && i < n0 && j < n1;
  const bool inner_xy = i >= 1 && j >= 1 && i <= n0 - 2 && j <= n1 - 2;
  // the ring slots of planes kk, kk - 1 and kk - 2
  uint8_t *s_new = sS[0], *s_cur = sS[2], *s_old = sS[1];
  for (int kk = kb - 1, slot = 0; kk <= ke; ++kk, slot = (slot + 1 == D) ? 0 : slot + 1) {
    // plane kk + D - 1 into the slot of plane kk - 1 (read back in the last
    // round); then plane kk, the oldest of the D groups in flight, has landed
    fetch(kk + D - 1, slot == 0 ? D - 1 : slot - 1);
    cp_async_wait_group<D - 1>();
    const bool live = ok && kk >= 0 && kk < n2;
    double P = 0.0, V1 = 0.0, V2 = 0.0, V3 = 0.0;
    if (live) {
      const double* raw = &sRaw[slot][0][tid];
      if (PST) {
        P = ph.gm1 * raw[0];
        V1 = raw[NT];
        V2 = raw[2 * NT];
        V3 = raw[3 * NT];
      } else {
        Cons u{raw[0], raw[NT], raw[2 * NT], raw[3 * NT], raw[4 * NT]};
        Prim w;
        cons_to_prim_exact(u, w, ph.nmin);
        P = ph.gm1 * w.E;
        V1 = w.V1;
        V2 = w.V2;
        V3 = w.V3;
      }
    }
    if (tid < NR) {
      sP[tid] = P;
      sV1[tid] = V1;
      sV2[tid] = V2;
    }
    __syncthreads();
    if (tid < NR) {
      uint8_t bits = 0;
      if (live) {
        if (has_xm && shock_between(P, sP[tid - 1], V1 - sV1[tid - 1], thr)) bits |= 1;
        if (has_ym && shock_between(P, sP[tid - RX], V2 - sV2[tid - RX], thr)) bits |= 2;
        if (kk >= 1 && kk >= kb && shock_between(P, Pz, V3 - Vz, thr)) bits |= 4;
      }
      s_new[tid] = bits;
    }
    Pz = P;
    Vz = V3;
    __syncthreads();
    const int k = kk - 1;
    if (k >= kb && out_in) {
      uint8_t bits = 0;
      if (inner_xy && k >= 1 && k <= n2 - 2) {
        const uint8_t* m = s_old;  // plane k - 1
        const uint8_t* c = s_cur;
        const uint8_t* p = s_new;
        const unsigned s0 = c[ro], sxp = c[ro + 1], sxm = c[ro - 1], syp = c[ro + RX],
                       sym = c[ro - RX], szp = p[ro], szm = m[ro];
        const unsigned sxp_ym = c[ro + 1 - RX], syp_xm = c[ro + RX - 1], sxp_zm = m[ro + 1],
                       syp_zm = m[ro + RX], szp_xm = p[ro - 1], szp_ym = p[ro - RX];
        // flag d from bit e at c, c + e_e, c - e_d and c + e_e - e_d (e != d)
        if (((s0 | syp | sxm | syp_xm) & 2) || ((s0 | szp | sxm | szp_xm) & 4)) bits |= 1;
        if (((s0 | sxp | sym | sxp_ym) & 1) || ((s0 | szp | sym | szp_ym) & 4)) bits |= 2;
        if (((s0 | sxp | szm | sxp_zm) & 1) || ((s0 | syp | szm | syp_zm) & 2)) bits |= 4;
      }
      *src.flags(i, j, k) = bits;
    }
    uint8_t* t = s_old;
    s_old = s_cur;
    s_cur = s_new;
    s_new = t;
  }
}

// The features of one brick (detect_tile over its planes [k0, k1)), from the
// conserved state U or (PST) from the compact primitives Pst (N, V1, V2, V3, E).
template <bool PST>
__global__ void __launch_bounds__(kDetThreads, 3)
    detect_features_kernel(Box b, Phys ph, const double* __restrict__ U,
                           const double* __restrict__ Pst, uint8_t* __restrict__ df, int k0,
                           int k1) {
  const DetectBrick<PST> src(b, U, Pst, df);
  const int kb = k0 + blockIdx.z * kDetKZ;
  detect_tile<PST>(src, ph, b.n[0], b.n[1], b.n[2], blockIdx.x * kDetTX, blockIdx.y * kDetTY, kb,
                   min(kb + kDetKZ, k1));
}

// A tile of the features of a batch: brick, and the tile's first column, row
// and plane.
struct DetItem {
  int brick, i0, j0, k0;
};

// The features of every brick of a batch from the conserved states, one
// block per tile of the work list (detect_tile on the tile's brick).
__global__ void __launch_bounds__(kDetThreads, 3)
    batch_detect_features_kernel(const BatchBrick* __restrict__ bb,
                                 const DetItem* __restrict__ items, Phys ph) {
  const DetItem it = items[blockIdx.x];
  const BatchBrick& B = bb[it.brick];
  if (B.skip && *B.skip) return;
  const DetectBrick<false> src(B.box, B.U, nullptr, B.df);
  detect_tile<false>(src, ph, B.box.n[0], B.box.n[1], B.box.n[2], it.i0, it.j0, it.k0,
                     min(it.k0 + kDetKZ, B.box.n[2]));
}

// Per-cell inverse CFL time of the state, reduced to one maximum
// (ComputeTimeStepKernel_CSL, Integrator_C_PS__Kernel.f90:97-142).
__global__ void inverse_timestep_kernel(Box b, Phys ph, const double* __restrict__ U,
                                        const double* __restrict__ Pst,
                                        AxisGeo G0, AxisGeo G1, AxisGeo G2,
                                        unsigned long long* __restrict__ tsi_bits) {
  __shared__ double s_red[32];
  const long long nP = b.nP;
  double m = -DBL_MAX;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nP;
       c += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    decode3(c, b.n[0], b.n[1], i, j, k);
    Prim w;
    if (Pst) {
      w.N = Pst[c];
      w.V1 = Pst[nP + c];
      w.V2 = Pst[2 * nP + c];
      w.V3 = Pst[3 * nP + c];
      w.E = Pst[4 * nP + c];
    } else {
      const long long o = (i + 2) + (long long)b.m[0] * ((j + 2) + (long long)b.m[1] * (k + 2));
      Cons u{U[o], U[b.nV + o], U[2 * b.nV + o], U[3 * b.nV + o], U[4 * b.nV + o]};
      cons_to_prim(u, w, ph.nmin);
    }
    double P, CS;
    eos_cell(w.N, w.E, ph, P, CS, nullptr);
    m = fmax2(m, inverse_cfl_time(w, CS, G0.W[i + 2], G1.W[j + 2], G2.W[k + 2], G0.RW[i + 2],
                                  G1.RW[j + 2], G2.RW[k + 2]));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax2(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = s_red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r = fmax2(r, s_red[w]);
    atomicMax(tsi_bits, ordered_bits(r));
  }
}

// Device-side integrator state of one brick (evolve loop).
struct Clock {
  double dt;       // step to take
  double time;     // current time
  double finish;   // FinishTime
  int cycle;       // iCycle
  int max_cycle;   // FinishCycle
  int done;        // nonzero: the loop has ended, kernels skip
  int pad;
};

// Integrator ComputeTimeStep (Integrator_Template.f90:896-939 and
// Integrator_C_PS__Form.f90:419) from the reduced inverse CFL time, plus the
// CheckpointTimeExact cut of ComputeNewTime (:842-893) at the finish time.
__global__ void finalize_dt_kernel(Phys ph, const unsigned long long* __restrict__ tsi_bits,
                                   Clock* __restrict__ clk, int n, int clip_to_finish) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  Clock& c = clk[b];
  if (c.done) return;
  double tsi = from_ordered_bits_dev(tsi_bits[b]);
  tsi = fmax2(kTiny, tsi);
  double dt = DBL_MAX;
  const double cand = 1.0 / tsi;
  if (cand < dt) dt = cand;
  dt = ph.courant * dt;
  double ramp = (double)(c.cycle + 1) / (double)ph.n_ramp;
  if (ramp > 1.0) ramp = 1.0;
  if (ramp < 1.0) dt = ramp * dt;
  if (clip_to_finish && c.time + dt > c.finish) dt = c.finish - c.time;
  c.dt = dt;
}

// Time += dt, iCycle += 1, loop condition of Integrator % Evolve (:311).
__global__ void advance_clock_kernel(Clock* __restrict__ clk, int n) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  Clock& c = clk[b];
  if (c.done) return;
  c.time = c.time + c.dt;
  c.cycle = c.cycle + 1;
  if (!(c.time < c.finish && c.cycle < c.max_cycle)) c.done = 1;
}

// Volume integrals of the six conserved fields over the proper cells
// (Current_ASC__Template.f90:203-349, VolumeIntegral_Form.f90:25-117): block b
// sums the cells [b chunk, (b + 1) chunk) and writes its six partial sums;
// the host adds the partials in block order, so the result does not depend
// on timing.
__global__ void totals_kernel(Box b, const double* __restrict__ U, AxisGeo G0, AxisGeo G1,
                              AxisGeo G2, long long chunk, double* __restrict__ partial) {
  __shared__ double s_red[6][32];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const long long c0 = blockIdx.x * chunk, c1 = min(b.nP, c0 + chunk);
  for (long long c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
    int i, j, k;
    decode3(c, b.n[0], b.n[1], i, j, k);
    const long long g = (i + 2) + (long long)b.m[0] * ((j + 2) + (long long)b.m[1] * (k + 2));
    const double dv = G0.W[i + 2] * G1.W[j + 2] * G2.W[k + 2];
#pragma unroll
    for (int q = 0; q < 6; ++q) acc[q] += U[q * b.nV + g] * dv;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    double v = acc[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) s_red[q][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += s_red[threadIdx.x][w];
    partial[blockIdx.x * 6 + threadIdx.x] = v;
  }
}

// Counts of proper cells holding a non-finite value in any field, and of
// cells at the density floor, for gfx_fluid_check_state.
__global__ void check_state_kernel(Box b, Phys ph, const double* __restrict__ U,
                                   unsigned long long* __restrict__ counts) {
  unsigned long long bad = 0, floor = 0;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < b.nP;
       c += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    decode3(c, b.n[0], b.n[1], i, j, k);
    const long long g = (i + 2) + (long long)b.m[0] * ((j + 2) + (long long)b.m[1] * (k + 2));
    bool finite = true;
#pragma unroll
    for (int q = 0; q < 6; ++q) finite &= isfinite(U[q * b.nV + g]);
    bad += finite ? 0 : 1;
    floor += (U[g] <= ph.nmin) ? 1 : 0;
  }
  if (bad) atomicAdd(counts, bad);
  if (floor) atomicAdd(counts + 1, floor);
}

// The Sources records of one RK2 stage, over the ghost layout of S [10][nV]:
//   S_u  = S_u + (B K_u) / dt, u < 6, every value (RecordDivergenceKernel,
//          Step_RK_C_ASC__Kernel.f90:12-46, after the stage's divergence,
//          Step_RK_C_ASC__Template.f90:1548-1595); K is that divergence alone,
//          with zero ghosts, so the ghosts record zero;
//   S_6  = S_6 - N (V . g) B          (Gravitational_G)
//   S_7+d = S_7+d - N g_d B, d < 3    (Gravitational_S_D)
//          on proper cells with the uniform gradient g = (0, 0, a)
//          (ApplyGravity_F__Command.f90:23-264, the Sources halves of
//          ApplyGravityMomentum and ApplyGravityEnergy; baryon mass 1);
//          zero elsewhere, and zero everywhere without gravity.
// FIRST: stage 1, where the records start from zero (the reference clears
// them there).  N, V: the primitives of the stage's input state, from P
// (compact) when given, else recovered from U as the stage recovers them.
template <bool FIRST>
__global__ void record_sources_kernel(Box b, Phys ph, const double* __restrict__ K,
                                      const double* __restrict__ dt_ptr, double weight,
                                      const double* __restrict__ U,
                                      const double* __restrict__ P, double* __restrict__ S) {
  const double dt = *dt_ptr;
  const bool grav = ph.accel != 0.0;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < b.nV;
       v += (long long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int u = 0; u < 6; ++u) {
      const double s = FIRST ? 0.0 : S[u * b.nV + v];
      S[u * b.nV + v] = s + weight * K[u * b.nV + v] / dt;
    }
    double g[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) g[q] = FIRST ? 0.0 : S[(6 + q) * b.nV + v];
    int i, j, k;
    decode3(v, b.m[0], b.m[1], i, j, k);
    i -= 2;
    j -= 2;
    k -= 2;
    if (grav && i >= 0 && j >= 0 && k >= 0 && i < b.n[0] && j < b.n[1] && k < b.n[2]) {
      Prim w;
      if (P) {
        const long long c = i + (long long)b.n[0] * (j + (long long)b.n[1] * k);
        w.N = P[c];
        w.V1 = P[b.nP + c];
        w.V2 = P[2 * b.nP + c];
        w.V3 = P[3 * b.nP + c];
        w.E = P[4 * b.nP + c];
      } else {
        Cons c{U[v], U[b.nV + v], U[2 * b.nV + v], U[3 * b.nV + v], U[4 * b.nV + v]};
        cons_to_prim(c, w, ph.nmin);
      }
      const double a = ph.accel;
      g[0] = g[0] - w.N * (w.V1 * 0.0 + w.V2 * 0.0 + w.V3 * a) * weight;
      g[1] = g[1] - w.N * 0.0 * weight;
      g[2] = g[2] - w.N * 0.0 * weight;
      g[3] = g[3] - w.N * a * weight;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) S[(6 + q) * b.nV + v] = g[q];
  }
}

__global__ void reset_bits_kernel(unsigned long long* __restrict__ bits, int n, int* counter,
                                  int n_counters) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n || i < n_counters;
       i += gridDim.x * blockDim.x) {
    if (i < n) bits[i] = 0x0010000000000000ull;  // ordered_bits(-DBL_MAX)
    if (i < n_counters) counter[i] = 0;
  }
}

}  // namespace gfx

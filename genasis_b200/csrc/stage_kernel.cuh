// stage_kernel.cuh -- fused finite-volume stage for sm_100a.
//
// One CTA owns a TX x TY column of cells of one brick and marches it along z
// over [z0, z1).  Per z plane k it
//   1. moves plane k into the plane buffer (the own cells from a ring of own
//      column values, the x / y halo from a halo buffer) and starts
//      asynchronous copies (cp.async) of the halo of plane k+1 and of the own
//      column's plane k+2, with the boundary conditions applied as index maps,
//   2. computes the limited x / y slopes of the tile's cells (those of the
//      halo cells were formed during plane k-1), then finishes the copies in
//      place (cons->prim for a conserved input, reversed velocities),
//   3. computes the Riemann fluxes of every x, y face of the plane (each face
//      once), the halo cells' slopes of plane k+1, and the z slope and z face
//      k+1 of every own column,
//   4. forms the divergence increment of every cell in the reference's order
//      (x, then y, then z contributions) and applies the RK stage epilogue.
// This replaces the ~40 full-array sweeps per direction of
// IncrementDivergence_FV % Compute (IncrementDivergence_FV__Form.f90:344-412)
// and the Copy / MultiplyAdd / ComputeFromConserved sweeps of the RK stepper
// (Step_RK_C_ASC__Template.f90:761-1281) with one pass per stage.
#pragma once

#include "fluid_physics.cuh"

namespace gfx {

constexpr int TX = 32;          // tile width (x), one warp per row
constexpr int kTileY = 16;      // default tile rows; 8 is the other height built

// The tile shape TX x TYt and what follows from it: NT threads per CTA.
// Functions that depend on the tile take TYt as a template parameter and
// open with GFX_TILE(TYt).
#define GFX_TILE(TYt)       \
  constexpr int TY = (TYt); \
  constexpr int NT = TX * TY; \
  (void)TY; (void)NT
// CTAs per SM the registers allow at 128 registers per thread
constexpr int tile_min_ctas(int ty) { return (TX * ty >= 512) ? 1 : 2; }
// Ring of halo cells around the tile in the full plane: two for PARABOLIC
// (each face reconstructs both its cells) and for 16-row tiles (where the
// compiler keeps more in registers with that pitch); one for 8-row tiles,
// whose two CTAs per SM need the smaller plane (faces and slopes read the
// neighbours only; the halo cells' own slopes come from the halo buffer).
__host__ __device__ constexpr int full_ring(bool parab, int ty) {
  return (parab || ty >= 16) ? 2 : 1;
}

enum { MODE_INCREMENT = 0, MODE_STAGE1 = 1, MODE_STAGE2 = 2 };
// BC_NEIGHBOR: a face of a brick inside a chart of several bricks, whose
// ghost cells are the proper cells of the brick across it (Chart_SLD's ghost
// exchange, Chart_SLD__Form.f90:131-201); no boundary condition applies there
enum { BC_OUTFLOW = 0, BC_REFLECTING = 1, BC_PERIODIC = 2, BC_NEIGHBOR = 3 };
// How a stage launch's work items map to bricks: one brick, a batch of
// independent bricks, or the bricks of one chart (ghosts across linked faces)
enum { BAT_SINGLE = 0, BAT_BRICKS = 1, BAT_CHART = 2 };

// Per-axis tables over the ghost-inclusive index t in [0, n + 4) (t = cell + 2).
struct AxisGeo {
  const double* W;      // cell width WL + WR (GeometryFlat_Kernel.f90:22-24)
  const double* WL;     // centre - inner edge
  const double* WR;     // outer edge - centre
  const double* dXI;    // X(t) - X(t-1), Difference_Kernel.f90 on the centres
  const double* SQ;     // dXI(t)^2
  const double* CDEN;   // (dXI(t) dXI(t+1)) (dXI(t) + dXI(t+1))
  const double* RDXI;   // RN(1 / dXI(t))
  const double* RCDEN;  // RN(1 / CDEN(t))
  const double* RW;     // RN(1 / W(t))
  const double* PAR;    // PARABOLIC tables [PG_N][m + 1] (fluid_physics.cuh), or null
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
  double* wn;            // compact primitives N, V1, V2, V3, E (or null): stage 2, of
                         // the new state; stage 1, of its input
  int tile_y;            // host side: tile rows of the work list (0 = kTileY)
  // chart bricks: the brick across each face ([axis][inner, outer]) as an
  // index into `links`, the descriptors of this stage for every brick of the
  // chart (-1: no brick, the face's boundary condition applies); the periodic
  // faces of a chart link its end bricks
  int nb[3][2];
  const struct BrickDesc* links;
  int pad_;
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

// The brick that holds the value at coordinates c (possibly ghosts) of brick
// B, with c moved into that brick's frame.  Chart bricks (CH) cross the
// linked faces into the neighbours, one axis after the other, so that an
// edge ghost lands in the diagonal brick; what stays outside is for the
// boundary maps.  Every brick of a chart has at least 4 cells per axis and a
// ghost lies at most 2 cells out, so one crossing per axis suffices.
template <bool CH>
__device__ __forceinline__ const BrickDesc& cell_owner(const BrickDesc& B, int* c) {
  if (!CH) return B;
  if ((unsigned)c[0] < (unsigned)B.n[0] && (unsigned)c[1] < (unsigned)B.n[1] &&
      (unsigned)c[2] < (unsigned)B.n[2])
    return B;  // the common case: inside the brick
  const BrickDesc* S = &B;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int side = c[a] < 0 ? 0 : (c[a] >= S->n[a] ? 1 : -1);
    if (side >= 0) {
      const int nbi = S->nb[a][side];
      if (nbi >= 0) {
        const BrickDesc* N = B.links + nbi;
        c[a] += side ? -S->n[a] : N->n[a];
        S = N;
      }
    }
  }
  return *S;
}

// The input value of cell (gx, gy, gz) of brick B: the address of its first
// field (the stored primitives N, V1, V2, V3, E, compact, for IN_PRIM; else
// the conserved D, S1, S2, S3, G, ghost layout), the stride between fields
// and the velocity components the boundary maps reverse (bit d: V_d+1).
template <bool IN_PRIM, bool CH>
__device__ __forceinline__ const double* cell_src(const BrickDesc& B, int gx, int gy, int gz,
                                                  long long& fs, int& flips) {
  int c[3] = {gx, gy, gz};
  const BrickDesc& S = cell_owner<CH>(B, c);
  bool nx, ny, nz;
  const int sx = bc_map(c[0], S.n[0], S.bc[0][0], S.bc[0][1], nx);
  const int sy = bc_map(c[1], S.n[1], S.bc[1][0], S.bc[1][1], ny);
  const int sz = bc_map(c[2], S.n[2], S.bc[2][0], S.bc[2][1], nz);
  flips = (int)nx | ((int)ny << 1) | ((int)nz << 2);
  if (IN_PRIM) {
    fs = S.nP;
    return S.P_in + (sx + (long long)S.n[0] * (sy + (long long)S.n[1] * sz));
  }
  fs = S.nV;
  return S.U_in + ((sx + 2) + (long long)S.m[0] * ((sy + 2) + (long long)S.m[1] * (sz + 2)));
}

// The primitives of cell (gx, gy, gz) of brick B (possibly a ghost), after
// the boundary maps: recovered from the conserved values for a conserved
// input, with the reversed velocities negated.
template <bool IN_PRIM, bool CH>
__device__ __forceinline__ Prim load_prim(const BrickDesc& B, const Phys& ph, int gx, int gy,
                                          int gz) {
  long long fs;
  int flips;
  const double* p = cell_src<IN_PRIM, CH>(B, gx, gy, gz, fs, flips);
  Prim w;
  if (IN_PRIM) {
    w.N = __ldg(p);
    w.V1 = __ldg(p + fs);
    w.V2 = __ldg(p + 2 * fs);
    w.V3 = __ldg(p + 3 * fs);
    w.E = __ldg(p + 4 * fs);
  } else {
    Cons c;
    c.D = __ldg(p);
    c.S1 = __ldg(p + fs);
    c.S2 = __ldg(p + 2 * fs);
    c.S3 = __ldg(p + 3 * fs);
    c.G = __ldg(p + 4 * fs);
    cons_to_prim(c, w, ph.nmin);
  }
  if (flips & 1) w.V1 = -w.V1;
  if (flips & 2) w.V2 = -w.V2;
  if (flips & 4) w.V3 = -w.V3;
  return w;
}

// Loads the primitives of cell (gx, gy) of plane gz (all possibly ghosts) into
// a ring plane at local (ly, lx).
template <bool IN_PRIM, int TYt, int FR, bool CH>
__device__ __forceinline__ void load_cell(const BrickDesc& B, const Phys& ph, double* plane,
                                          int lx, int ly, int gx, int gy, int gz) {
  GFX_TILE(TYt);
  constexpr int FW = TX + 2 * FR, FS = FW * (TY + 2 * FR);
  const Prim w = load_prim<IN_PRIM, CH>(B, ph, gx, gy, gz);
  const int o = (ly + FR) * FW + (lx + FR);
  plane[o] = w.N;
  plane[FS + o] = w.V1;
  plane[2 * FS + o] = w.V2;
  plane[3 * FS + o] = w.V3;
  plane[4 * FS + o] = w.E;
}

// Loads the primitives of one cell into 5 shared slots at stride `stride`.
template <bool IN_PRIM, bool CH>
__device__ __forceinline__ void load_cell_to(const BrickDesc& B, const Phys& ph, double* dst,
                                             int stride, int gx, int gy, int gz) {
  const Prim w = load_prim<IN_PRIM, CH>(B, ph, gx, gy, gz);
  dst[0] = w.N;
  dst[stride] = w.V1;
  dst[2 * stride] = w.V2;
  dst[3 * stride] = w.V3;
  dst[4 * stride] = w.E;
}

// Loads the primitives of one cell into a column slot (5 values at stride NT).
template <bool IN_PRIM, int TYt, bool CH>
__device__ __forceinline__ void load_cell_col(const BrickDesc& B, const Phys& ph, double* dst,
                                              int gx, int gy, int gz) {
  GFX_TILE(TYt);
  load_cell_to<IN_PRIM, CH>(B, ph, dst, NT, gx, gy, gz);
}

// Asynchronous 8-byte copies from global to shared memory (cp.async, which
// needs no registers and lets the thread go on until cp_async_wait_all).
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}
// Waits until at most N of this thread's committed groups of copies are
// still in flight.
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Starts the asynchronous copy of the input values of cell (gx, gy, gz)
// (possibly ghosts) into 5 shared slots at stride `stride`: the stored
// primitives N, V1, V2, V3, E (IN_PRIM, compact layout) or the conserved D,
// S1, S2, S3, G (ghost layout).  cell_flips: the velocity components the
// boundary map reverses there (bit d: V_d+1), which finish_cell applies once
// the copy has landed.
template <bool CH>
__device__ __forceinline__ int cell_flips(const BrickDesc& B, int gx, int gy, int gz) {
  int c[3] = {gx, gy, gz};
  const BrickDesc& S = cell_owner<CH>(B, c);
  bool nx, ny, nz;
  bc_map(c[0], S.n[0], S.bc[0][0], S.bc[0][1], nx);
  bc_map(c[1], S.n[1], S.bc[1][0], S.bc[1][1], ny);
  bc_map(c[2], S.n[2], S.bc[2][0], S.bc[2][1], nz);
  return (int)nx | ((int)ny << 1) | ((int)nz << 2);
}

template <bool IN_PRIM, bool CH>
__device__ __forceinline__ void copy_cell_async(const BrickDesc& B, double* dst, int stride,
                                               int gx, int gy, int gz) {
  long long fs;
  int flips;
  const double* p = cell_src<IN_PRIM, CH>(B, gx, gy, gz, fs, flips);
  (void)flips;
#pragma unroll
  for (int q = 0; q < 5; ++q) cp_async8(dst + q * stride, p + q * fs);
}

// After this thread's copy_cell_async into the slots has landed: the
// primitives of the cell there (recovered from the conserved values for a
// conserved input), with the reversed velocities negated -- the values
// load_cell_to gives.
template <bool IN_PRIM>
__device__ __forceinline__ void finish_cell(const Phys& ph, double* dst, int stride, int flips) {
  if (IN_PRIM && !flips) return;
  Prim w;
  if (IN_PRIM) {
    w.N = dst[0];
    w.V1 = dst[stride];
    w.V2 = dst[2 * stride];
    w.V3 = dst[3 * stride];
    w.E = dst[4 * stride];
  } else {
    Cons c{dst[0], dst[stride], dst[2 * stride], dst[3 * stride], dst[4 * stride]};
    cons_to_prim(c, w, ph.nmin);
  }
  if (flips & 1) w.V1 = -w.V1;
  if (flips & 2) w.V2 = -w.V2;
  if (flips & 4) w.V3 = -w.V3;
  dst[0] = w.N;
  dst[stride] = w.V1;
  dst[2 * stride] = w.V2;
  dst[3 * stride] = w.V3;
  dst[4 * stride] = w.E;
}

// DIFFUSIVE_FLUX_I bit d of cell (gx, gy, gz).  Outside the brick: the bit
// of the linked brick's cell (chart bricks), else 0 (the ghost layer of a
// chart boundary, which ClearBoundary clears).
template <bool CH>
__device__ __forceinline__ unsigned df_byte(const BrickDesc& B, int gx, int gy, int gz) {
  if (B.df == nullptr) return 0;
  if (gx < 0 || gy < 0 || gz < 0 || gx >= B.n[0] || gy >= B.n[1] || gz >= B.n[2]) {
    if (!CH) return 0;
    int c[3] = {gx, gy, gz};
    const BrickDesc& S = cell_owner<true>(B, c);
    if (c[0] < 0 || c[1] < 0 || c[2] < 0 || c[0] >= S.n[0] || c[1] >= S.n[1] ||
        c[2] >= S.n[2])
      return 0;
    return S.df[c[0] + (long long)S.n[0] * (c[1] + (long long)S.n[1] * c[2])];
  }
  return B.df[gx + (long long)B.n[0] * (gy + (long long)B.n[1] * gz)];
}
template <bool CH>
__device__ __forceinline__ bool df_bit(const BrickDesc& B, int d, int gx, int gy, int gz) {
  return (df_byte<CH>(B, gx, gy, gz) >> d) & 1;
}

// Whether face `side` of axis a records the boundary fluence: every face of
// a single brick, only the chart's own boundary for a chart brick
// (RecordBoundaryFluence_CSL, IncrementDivergence_FV__Form.f90:1002-1069).
__device__ __forceinline__ bool records_fluence(const BrickDesc& B, int a, int side) {
  return B.bc[a][side] != BC_NEIGHBOR;
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

// Boundary fluence of one face.  The stages evolve five fields (the DS
// increment is dead: ComputeFromConserved rewrites DS = N SB), but the
// reference records all six fluxes on the boundary faces, so the six-field
// flux is formed there from the same reconstructed primitives.  Kept out of
// line: it runs on boundary faces only.
struct FacePrims {
  double l[5], r[5];
};

template <int D, bool HLLC>
__device__ __noinline__ void boundary_fluence6(const BrickDesc& B, const Phys& ph, FacePrims p,
                                               bool diffusive, int face, int a, int na, int b,
                                               double factor) {
  FaceState L, R;
  face_state<6>(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], ph, L);
  face_state<6>(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], ph, R);
  double F6[6];
  riemann_flux<D, HLLC, 6>(L, R, diffusive, F6);
  record_fluence<6>(B, face, a, na, b, F6, factor);
}

template <int D, bool HLLC, int NF>
__device__ __forceinline__ void boundary_fluence(const BrickDesc& B, const Phys& ph,
                                                 const double* l, const double* r,
                                                 bool diffusive, const double* F, int face,
                                                 int a, int na, int b, double factor) {
  if constexpr (NF == 6) {
    record_fluence<6>(B, face, a, na, b, F, factor);
  } else {
    FacePrims p;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      p.l[v] = l[v];
      p.r[v] = r[v];
    }
    boundary_fluence6<D, HLLC>(B, ph, p, diffusive, face, a, na, b, factor);
  }
}

// Relabels the velocity and momentum components of a face state so that
// direction d comes first (d = 1: swap 1 and 2).  The sums that depend on the
// component order (G) are formed before, in the reference's frame; the flux
// formulas treat every component alike, so the relabelled solve is exact.
__device__ __forceinline__ void to_normal_frame_y(FaceState& s) {
  const double v = s.V1, m = s.S1;
  s.V1 = s.V2;
  s.S1 = s.S2;
  s.V2 = v;
  s.S2 = m;
}

// The reconstructed primitives of a face, IncrementDivergence_FV__Kernel.f90:
// 70-90: V_IL = V(i-1) + dXR(i-1) dVdX(i-1), V_IR = V(i) - dXL(i) dVdX(i).
__device__ __forceinline__ void face_prims(const double* vm, const double* sm_, int stride_m,
                                           const double* vp, const double* sp, int stride_p,
                                           int sstride_m, int sstride_p, double wr, double wl,
                                           double* l, double* r) {
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    l[v] = vm[v * stride_m] + wr * sm_[v * sstride_m];
    r[v] = vp[v * stride_p] - wl * sp[v * sstride_p];
  }
}

// Per-tile copy of the geometry tables of one axis, entries t0 .. t0 + L - 1.
enum { G_W, G_WL, G_WR, G_DXI, G_SQ, G_CDEN, G_RDXI, G_RCDEN, G_RW, G_NTAB };

template <int TYt>
__device__ __forceinline__ void fill_geo(const AxisGeo& G, int m, int t0, int L, double* dst,
                                         int tid) {
  GFX_TILE(TYt);
  const double* tabs[G_NTAB] = {G.W, G.WL, G.WR, G.dXI, G.SQ, G.CDEN, G.RDXI, G.RCDEN, G.RW};
  for (int i = tid; i < G_NTAB * L; i += NT) {
    const int q = i / L, j = i % L, t = t0 + j;
    dst[i] = (t >= 0 && t <= m) ? __ldg(tabs[q] + t) : 0.0;
  }
}

template <int NF, int TYt, bool PARAB = false>
struct StageLayout {
  static constexpr int TY = TYt, NT = TX * TYt;
  static constexpr int FR = full_ring(PARAB, TYt), FW = TX + 2 * FR, FS = FW * (TY + 2 * FR);
  static constexpr int kFull = 5 * FS;            // plane k with its x / y halo ring
  static constexpr int kCen = 2 * 5 * NT;         // centres of planes k+1, k+2
  static constexpr int kZs = 5 * NT;              // z slope of plane k (own column)
  static constexpr int kZf = NF * NT;             // z flux of face k (own column)
  // HS (all but PARABOLIC, which has no slope phase): the slopes of the x / y
  // halo cells of plane k+1 are formed during plane k (from the halo copied
  // ahead) into a double-buffered array, so that the slope phase holds the
  // tile's own cells only
  static constexpr bool HS = !PARAB;
  static constexpr int kNHS = 2 * TX + 2 * TYt;  // halo slopes of a plane
  static constexpr int kSx = HS ? 5 * NT : 0;  // x slopes of the tile's cells
  static constexpr int kSy = HS ? 5 * NT : 0;  // y slopes
  static constexpr int kFx = NF * TY * (TX + 1);
  static constexpr int kFy = NF * (TY + 1) * TX;
  static constexpr int kGx = G_NTAB * (TX + 4);
  static constexpr int kGy = G_NTAB * (TY + 4);
  static constexpr int kNH = 4 * TX + 4 * TY;  // x / y halo cells of a plane
  static constexpr int kHalo = 5 * kNH;        // halo of plane k+1
  static constexpr int kHs = HS ? 2 * 5 * kNHS : 0;
  static constexpr int kDoubles =
      kFull + kCen + kZs + kZf + kSx + kSy + kFx + kFy + kGx + kGy + kHalo + kHs;
  static constexpr size_t kBytes = sizeof(double) * kDoubles;
};

// Limited slopes of the 5 primitives of one cell; v points at the cell in a
// buffer with variable stride vs and neighbour stride st; g is a per-tile
// geometry cache (entry c = the cell's own index).
__device__ __forceinline__ void cell_slopes(const double* v, int vs, int st, const double* g,
                                            int L, int c, const Phys& ph, double* out,
                                            int ostride) {
  const double dxl = g[G_DXI * L + c], dxr = g[G_DXI * L + c + 1];
  const double sql = g[G_SQ * L + c], sqr = g[G_SQ * L + c + 1], cden = g[G_CDEN * L + c];
  const double rdxl = g[G_RDXI * L + c], rdxr = g[G_RDXI * L + c + 1],
               rcden = g[G_RCDEN * L + c];
#pragma unroll
  for (int q = 0; q < 5; ++q)
    out[q * ostride] = limited_slope(v[q * vs - st], v[q * vs], v[q * vs + st], dxl, dxr, sql,
                                     sqr, cden, rdxl, rdxr, rcden, ph.theta, ph.use_limiter);
}

// Limited z slopes of the 5 primitives of the own column at plane p from the
// values a (plane p-1), b (p), c (p+1) at strides sa, sb, sc.
__device__ __forceinline__ void z_slope(const AxisGeo& GZ, const Phys& ph, int p,
                                        const double* a, int sa, const double* b, int sb,
                                        const double* c, int sc, double* out) {
  const int t = p + 2;
  const double dxl = __ldg(GZ.dXI + t), dxr = __ldg(GZ.dXI + t + 1);
  const double sql = __ldg(GZ.SQ + t), sqr = __ldg(GZ.SQ + t + 1), cden = __ldg(GZ.CDEN + t);
  const double rdxl = __ldg(GZ.RDXI + t), rdxr = __ldg(GZ.RDXI + t + 1),
               rcden = __ldg(GZ.RCDEN + t);
#pragma unroll
  for (int q = 0; q < 5; ++q)
    out[q] = limited_slope(a[q * sa], b[q * sb], c[q * sc], dxl, dxr, sql, sqr, cden, rdxl,
                           rdxr, rcden, ph.theta, ph.use_limiter);
}

// Flux through the z face between planes p-1 (values a, slopes sm_) and p
// (values b, slopes sp) of the own column (gx, gy), with its boundary fluence;
// diff: the face's DIFFUSIVE_FLUX_I bit (z bit of cell p).
template <bool HLLC, int NF, bool CH>
__device__ __forceinline__ void z_face_lr(const BrickDesc& B, const Phys& ph, int p,
                                          const double* l, const double* r, int gx, int gy,
                                          bool own, double dt, bool diff, double* F) {
  FaceState L, R;
  face_state<NF>(l[0], l[1], l[2], l[3], l[4], ph, L);
  face_state<NF>(r[0], r[1], r[2], r[3], r[4], ph, R);
  riemann_flux<2, HLLC, NF>(L, R, diff, F);
  if (own && (p == 0 || p == B.n[2]) && B.fluence &&
      (!CH || records_fluence(B, 2, p == 0 ? 0 : 1)))
    boundary_fluence<2, HLLC, NF>(B, ph, l, r, diff, F, p == 0 ? 4 : 5, gx, B.n[0], gy,
                                  B.weight * dt);
}

template <bool HLLC, int NF, bool CH>
__device__ __forceinline__ void z_face(const BrickDesc& B, const Phys& ph, int p,
                                       const double* a, int sa, const double* sm_, int ssm,
                                       const double* b, int sb, const double* sp, int ssp,
                                       int gx, int gy, bool own, double dt, bool diff,
                                       double* F) {
  const AxisGeo& GZ = B.geo[2];
  double l[5], r[5];
  face_prims(a, sm_, sa, b, sp, sb, ssm, ssp, __ldg(GZ.WR + p + 1), __ldg(GZ.WL + p + 2), l,
             r);
  z_face_lr<HLLC, NF, CH>(B, ph, p, l, r, gx, gy, own, dt, diff, F);
}

// PARABOLIC: inner and outer face values of the 5 primitives of the own
// column's cell at plane p from the values a (p-1), b (p), c (p+1).
__device__ __forceinline__ void z_parabolic(const BrickDesc& B, int p, const double* a, int sa,
                                            const double* b, int sb, const double* c, int sc,
                                            double* vI, double* vO) {
  const int L = B.m[2] + 1;
#pragma unroll 1
  for (int q = 0; q < 5; ++q) {
    const FaceVals f = parabolic_cell(a[q * sa], b[q * sb], c[q * sc], B.geo[2].PAR, L, p + 2);
    vI[q] = f.vI;
    vO[q] = f.vO;
  }
}

// Prologue of a work item (own column only): planes z0-2 .. z0+1, the z
// slopes at z0-1 and z0 and the z face z0, left in zss / zfs and the centre
// slots for the plane loop.  Out of line: it runs once per item, and a second
// inlined copy of the slope and face code would only crowd the instruction
// cache of the plane loop.
// PARABOLIC (PARAB): zss keeps the outer face values of plane z0 instead of
// its slopes.
template <bool IN_PRIM, bool HLLC, int NF, bool PARAB, int TYt, bool CH>
__device__ __noinline__ void stage_prologue(const BrickDesc& B, const Phys& ph, double* full,
                                            double* cen, double* zss, double* zfs, int tid,
                                            int tx, int ty, int gx, int gy, int z0, bool own,
                                            double dt) {
  GFX_TILE(TYt);
  constexpr int FR = full_ring(PARAB, TYt), FW = TX + 2 * FR, FS = FW * (TY + 2 * FR);
  auto cslot = [&](int p) { return cen + (p & 1) * 5 * NT + tid; };
  double* fc = full + (ty + FR) * FW + (tx + FR);
  load_cell<IN_PRIM, TYt, FR, CH>(B, ph, full, tx, ty, gx, gy, z0 - 2);
  load_cell_col<IN_PRIM, TYt, CH>(B, ph, cslot(z0 - 1), gx, gy, z0 - 1);
  load_cell_col<IN_PRIM, TYt, CH>(B, ph, cslot(z0), gx, gy, z0);
  double s_m[5], s_0[5], vI0[5];
  if (PARAB)
    z_parabolic(B, z0 - 1, fc, FS, cslot(z0 - 1), NT, cslot(z0), NT, vI0, s_m);
  else
    z_slope(B.geo[2], ph, z0 - 1, fc, FS, cslot(z0 - 1), NT, cslot(z0), NT, s_m);
  load_cell<IN_PRIM, TYt, FR, CH>(B, ph, full, tx, ty, gx, gy, z0 + 1);
  if (PARAB)
    z_parabolic(B, z0, cslot(z0 - 1), NT, cslot(z0), NT, fc, FS, vI0, s_0);
  else
    z_slope(B.geo[2], ph, z0, cslot(z0 - 1), NT, cslot(z0), NT, fc, FS, s_0);
  double F[NF];
  const bool diff = HLLC && df_bit<CH>(B, 2, gx, gy, z0);
  if (PARAB)
    z_face_lr<HLLC, NF, CH>(B, ph, z0, s_m, vI0, gx, gy, own, dt, diff, F);
  else
    z_face<HLLC, NF, CH>(B, ph, z0, cslot(z0 - 1), NT, s_m, 1, cslot(z0), NT, s_0, 1, gx, gy, own,
                         dt, diff, F);
#pragma unroll
  for (int q = 0; q < 5; ++q) zss[q * NT + tid] = s_0[q];
#pragma unroll
  for (int u = 0; u < NF; ++u) zfs[u * NT + tid] = F[u];
  // plane z0+1 into its centre slot (the slot of z0-1)
  double* d = cslot(z0 + 1);
#pragma unroll
  for (int q = 0; q < 5; ++q) d[q * NT] = fc[q * FS];
}

// BATCHED: the work items span many bricks; each item's brick descriptor is
// copied from `many` into shared memory.  Otherwise `single` describes the one
// brick (read from the constant bank).
// PARAB: PARABOLIC reconstruction (single bricks): no slope phase; each face
// reconstructs its two cells, the own column carries outer face values in z.
template <int MODE, bool IN_PRIM, bool HLLC, bool GRAV, int NF, int BAT, bool PARAB = false,
          int TYt = kTileY>
__global__ void __launch_bounds__(TX * TYt, tile_min_ctas(TYt))
    stage_kernel(const __grid_constant__ BrickDesc single, const BrickDesc* __restrict__ many,
                 const WorkItem* __restrict__ items, int n_items, int* __restrict__ counter,
                 const __grid_constant__ Phys ph) {
  GFX_TILE(TYt);
  using SL = StageLayout<NF, TYt, PARAB>;
  constexpr int FR = SL::FR, FW = SL::FW, FS = SL::FS;
  extern __shared__ double smem[];
  double* full = smem;
  double* cen = full + SL::kFull;
  double* zss = cen + SL::kCen;
  double* zfs = zss + SL::kZs;
  double* sxs = zfs + SL::kZf;
  double* sys = sxs + SL::kSx;
  double* fxs = sys + SL::kSy;
  double* fys = fxs + SL::kFx;
  double* gxc = fys + SL::kFy;
  double* gyc = gxc + SL::kGx;
  double* hbuf = gyc + SL::kGy;
  double* hsl = hbuf + SL::kHalo;
  constexpr int NH = SL::kNH, NHS = SL::kNHS;
  constexpr bool HS = SL::HS;
  __shared__ int s_item;
  __shared__ double s_red[NT / 32];
  // HLLC on 8-row tiles (DFS): the DIFFUSIVE_FLUX_I bytes of the cells
  // (x0 .. x0 + TX, y0 .. y0 + TY) of plane k, the cells after every x and y
  // face of the tile, loaded at the start of the plane and kept here, so that
  // no face waits on a global load.  The three registers that carry them
  // across the slope phase would spill on 16-row tiles (512 threads at the
  // 128-register cap), which keep one load per face.
  constexpr bool DFS = HLLC && TYt == 8;
  constexpr int NDF = (TX + 1) * (TYt + 1);
  static_assert(NDF <= 2 * NT, "two flag bytes per thread at most");
  __shared__ uint8_t s_df[DFS ? NDF : 1];
  __shared__ BrickDesc s_desc;
  constexpr int LX = TX + 4, LY = TY + 4;

  const int tid = threadIdx.x;
  const int tx = tid % TX, ty = tid / TX;
  const int c_off = (ty + FR) * FW + (tx + FR);  // own cell in the full plane
  constexpr bool BATCHED = BAT != BAT_SINGLE;
  constexpr bool CH = BAT == BAT_CHART;
  const BrickDesc& B = BATCHED ? s_desc : single;

  for (;;) {
    if (tid == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n_items) break;
    const WorkItem W = items[it];
    if (BATCHED) {
      constexpr int nw = (int)(sizeof(BrickDesc) / sizeof(long long));
      static_assert(sizeof(BrickDesc) % sizeof(long long) == 0, "descriptor size");
      if (tid < nw)
        reinterpret_cast<long long*>(&s_desc)[tid] =
            reinterpret_cast<const long long*>(many + W.brick)[tid];
      __syncthreads();
    }
    if (B.skip && *B.skip) {
      __syncthreads();
      continue;
    }
    const int n0 = B.n[0], n1 = B.n[1];
    const AxisGeo& GZ = B.geo[2];
    const double dt = *B.dt;
    const int x0 = W.x0, y0 = W.y0, z0 = W.z0, z1 = W.z1;
    const int gx = x0 + tx, gy = y0 + ty;
    const bool own = (gx < n0) && (gy < n1);
    double tsi_max = -DBL_MAX;
    fill_geo<TYt>(B.geo[0], B.m[0], x0, LX, gxc, tid);
    fill_geo<TYt>(B.geo[1], B.m[1], y0, LY, gyc, tid);

    // own column helpers: a "column pointer" addresses 5 values at stride NT
    // (centre slots) or FS (full plane)
    auto cslot = [&](int p) { return cen + (p & 1) * 5 * NT + tid; };
    // ---- prologue (own column only): slopes at z0-1, z0 and the face z0 ----
    stage_prologue<IN_PRIM, HLLC, NF, PARAB, TYt, CH>(B, ph, full, cen, zss, zfs, tid, tx, ty, gx,
                                                  gy, z0, own, dt);
    // the halo cell of this thread (threads below NH): two rows below and
    // above the tile, two columns left and right; hbuf holds its primitives
    // for the next plane (copied asynchronously, then finished in place),
    // starting with plane z0
    int hx = 0, hy = 0;
    if (tid < 4 * TX) {
      const int s = tid / TX;
      hx = tid % TX;
      hy = (s < 2) ? s - 2 : TY + s - 2;
    } else if (tid < NH) {
      const int j = tid - 4 * TX, s = j % 4;
      hy = j / 4;
      hx = (s < 2) ? s - 2 : TX + s - 2;
    }

    // HS: the limited slopes of the x / y halo cells of plane p (rows -1 and
    // TY, columns -1 and TX) from hbuf (plane p's halo) and the own centres
    // of plane p (cslot(p)) of the tile's edge threads, into hsl[p & 1]
    auto halo_slope = [&](int h, int p) {
      const double* cc = cen + (p & 1) * 5 * NT;
      const double *a, *b, *c, *g;
      int sa, sb, sc, L, ci;
      if (h < 2 * TX) {  // y slope of row -1 (s = 0) or row TY (s = 1)
        const int s = h / TX, lx = h % TX, ly = s ? TY : -1;
        if (y0 + ly > n1 || x0 + lx >= n0) return;
        g = gyc;
        L = LY;
        ci = ly + 2;
        if (s == 0) {
          a = hbuf + lx, sa = NH;
          b = hbuf + TX + lx, sb = NH;
          c = cc + lx, sc = NT;
        } else {
          a = cc + (TY - 1) * TX + lx, sa = NT;
          b = hbuf + 2 * TX + lx, sb = NH;
          c = hbuf + 3 * TX + lx, sc = NH;
        }
      } else {  // x slope of column -1 (s = 0) or column TX (s = 1)
        const int j = h - 2 * TX, s = j / TY, ly = j % TY, lx = s ? TX : -1;
        if (x0 + lx > n0 || y0 + ly >= n1) return;
        g = gxc;
        L = LX;
        ci = lx + 2;
        const int hb = 4 * TX + 4 * ly;  // hbuf index of the cell (-2, ly)
        if (s == 0) {
          a = hbuf + hb, sa = NH;
          b = hbuf + hb + 1, sb = NH;
          c = cc + ly * TX, sc = NT;
        } else {
          a = cc + ly * TX + TX - 1, sa = NT;
          b = hbuf + hb + 2, sb = NH;
          c = hbuf + hb + 3, sc = NH;
        }
      }
      const double dxl = g[G_DXI * L + ci], dxr = g[G_DXI * L + ci + 1];
      const double sql = g[G_SQ * L + ci], sqr = g[G_SQ * L + ci + 1];
      const double cden = g[G_CDEN * L + ci], rdxl = g[G_RDXI * L + ci],
                   rdxr = g[G_RDXI * L + ci + 1], rcden = g[G_RCDEN * L + ci];
      double* out = hsl + (p & 1) * 5 * NHS + h;
#pragma unroll
      for (int q = 0; q < 5; ++q)
        out[q * NHS] = limited_slope(a[q * sa], b[q * sb], c[q * sc], dxl, dxr, sql, sqr, cden,
                                     rdxl, rdxr, rcden, ph.theta, ph.use_limiter);
    };
    if (tid < NH) copy_cell_async<IN_PRIM, CH>(B, hbuf + tid, NH, x0 + hx, y0 + hy, z0);
    cp_async_commit();
    cp_async_wait_all();
    if (tid < NH)
      finish_cell<IN_PRIM>(ph, hbuf + tid, NH, cell_flips<CH>(B, x0 + hx, y0 + hy, z0));
    __syncthreads();  // geometry caches, the halo of plane z0, the own centres
    if (HS) {
      if (tid < NHS) halo_slope(tid, z0);
      __syncthreads();  // (hbuf is refilled next)
    }

    for (int k = z0; k < z1; ++k) {
      // (1) plane k into the full buffer: own centre from its slot, the
      // x / y halo from hbuf; then plane k+2 of the own column into the freed
      // slot and the halo of plane k+1 into hbuf
      {
        double* src = cslot(k);
#pragma unroll
        for (int q = 0; q < 5; ++q) full[q * FS + c_off] = src[q * NT];
      }
      copy_cell_async<IN_PRIM, CH>(B, cslot(k + 2), NT, gx, gy, k + 2);
      // the flag bytes of plane k for the x / y faces and of plane k+1 for the
      // own column's z face: loaded now, used after the slope phase
      unsigned dfa = 0, dfb = 0, dfz = 0;
      if (DFS) {
        dfa = df_byte<CH>(B, x0 + tid % (TX + 1), y0 + tid / (TX + 1), k);
        if (tid + NT < NDF)
          dfb = df_byte<CH>(B, x0 + (tid + NT) % (TX + 1), y0 + (tid + NT) / (TX + 1), k);
        dfz = df_byte<CH>(B, gx, gy, k + 1);
      }
      if (tid < NH) {
        if (hx >= -FR && hx < TX + FR && hy >= -FR && hy < TY + FR) {  // in the ring
          const int o = (hy + FR) * FW + (hx + FR);
#pragma unroll
          for (int q = 0; q < 5; ++q) full[q * FS + o] = hbuf[q * NH + tid];
        }
        if (k + 1 < z1)
          copy_cell_async<IN_PRIM, CH>(B, hbuf + tid, NH, x0 + hx, y0 + hy, k + 1);
      }
      cp_async_commit();
      __syncthreads();

      // (2) slopes of plane k: x [TY][TX] and y [TY][TX] of the tile's cells
      // (the halo cells' slopes came with the previous plane); PARABOLIC has
      // no slope phase
      if (HS) {
        for (int i = tid; i < 2 * NT; i += NT) {
          const bool isx = i < NT;
          const int j = isx ? i : i - NT, ly = j / TX, lx = j % TX;
          if (isx ? (x0 + lx > n0 || y0 + ly >= n1) : (y0 + ly > n1 || x0 + lx >= n0)) continue;
          cell_slopes(full + (ly + FR) * FW + (lx + FR), FS, isx ? 1 : FW, isx ? gxc : gyc,
                      isx ? LX : LY, isx ? lx + 2 : ly + 2, ph, (isx ? sxs : sys) + j, NT);
        }
      }
      // this thread's copies (plane k+2 of its column, the halo of plane
      // k+1) have landed and become primitives; the barrier shows them to
      // the CTA
      cp_async_wait_all();
      finish_cell<IN_PRIM>(ph, cslot(k + 2), NT, cell_flips<CH>(B, gx, gy, k + 2));
      if (tid < NH && k + 1 < z1)
        finish_cell<IN_PRIM>(ph, hbuf + tid, NH, cell_flips<CH>(B, x0 + hx, y0 + hy, k + 1));
      if (DFS) {
        s_df[tid] = (uint8_t)dfa;
        if (tid + NT < NDF) s_df[tid + NT] = (uint8_t)dfb;
      }
      __syncthreads();

      // (3) faces: x [TY][TX+1], y [TY+1][TX] of plane k, one code path for
      // both directions (the y states are relabelled so that y is first)
      {
        constexpr int NXF = TY * (TX + 1), NYF = (TY + 1) * TX;
        constexpr int PXF = (NXF + 31) / 32 * 32;
        const double factor = B.weight * dt;
        for (int i = tid; i < PXF + NYF; i += NT) {
          const bool isx = i < PXF;
          if (isx && i >= NXF) continue;
          const int j = isx ? i : i - PXF;
          const int ly = isx ? j / (TX + 1) : j / TX;
          const int lx = isx ? j % (TX + 1) : j % TX;
          const int cx = x0 + lx, cy = y0 + ly;
          if (isx ? (cx > n0 || cy >= n1) : (cy > n1 || cx >= n0)) continue;
          const int o = (ly + FR) * FW + (lx + FR);
          const int step = isx ? 1 : FW;
          // slopes of the cells before (sm_) and after (sp) the face, with
          // their strides between primitives: the tile's own slopes, or the
          // halo slopes of plane k at the tile's edges (HS)
          const double *sm_, *sp;
          int ssm, ssp;
          if (HS) {
            const double* hc = hsl + (k & 1) * 5 * NHS;
            const int e = ly * TX + lx;
            if (isx) {
              sm_ = (lx == 0) ? hc + 2 * TX + ly : sxs + e - 1;
              sp = (lx == TX) ? hc + 2 * TX + TY + ly : sxs + e;
              ssm = (lx == 0) ? NHS : NT;
              ssp = (lx == TX) ? NHS : NT;
            } else {
              sm_ = (ly == 0) ? hc + lx : sys + e - TX;
              sp = (ly == TY) ? hc + TX + lx : sys + e;
              ssm = (ly == 0) ? NHS : NT;
              ssp = (ly == TY) ? NHS : NT;
            }
          }
          const double wr = isx ? gxc[G_WR * LX + lx + 1] : gyc[G_WR * LY + ly + 1];
          const double wl = isx ? gxc[G_WL * LX + lx + 2] : gyc[G_WL * LY + ly + 2];
          double l[5], r[5];
          if (PARAB) {
            // V_IL = outer value of the cell before, V_IR = inner value of the cell after
            const double* g = isx ? B.geo[0].PAR : B.geo[1].PAR;
            const int L = (isx ? B.m[0] : B.m[1]) + 1;
            const int tm = (isx ? cx : cy) + 1;  // ghost-layout index of the cell before
#pragma unroll 1
            for (int q = 0; q < 5; ++q) {
              const double* v = full + q * FS + o - step;
              l[q] = parabolic_cell(v[-step], v[0], v[step], g, L, tm).vO;
              r[q] = parabolic_cell(v[0], v[step], v[2 * step], g, L, tm + 1).vI;
            }
          } else {
            face_prims(full + o - step, sm_, FS, full + o, sp, FS, ssm, ssp, wr, wl, l, r);
          }
          FaceState L, R;
          face_state<NF>(l[0], l[1], l[2], l[3], l[4], ph, L);
          face_state<NF>(r[0], r[1], r[2], r[3], r[4], ph, R);
          if (!isx) {
            to_normal_frame_y(L);
            to_normal_frame_y(R);
          }
          const bool diff =
              HLLC && (DFS ? ((s_df[ly * (TX + 1) + lx] >> (isx ? 0 : 1)) & 1)
                           : df_bit<CH>(B, isx ? 0 : 1, cx, cy, k));
          double F[NF];
          riemann_flux<0, HLLC, NF>(L, R, diff, F);
          if (!isx) {
            const double f = F[1];
            F[1] = F[2];
            F[2] = f;
          }
          double* out = isx ? fxs + ly * (TX + 1) + lx : fys + ly * TX + lx;
          const int ostride = isx ? TY * (TX + 1) : (TY + 1) * TX;
#pragma unroll
          for (int u = 0; u < NF; ++u) out[u * ostride] = F[u];
          if (B.fluence && (isx ? (cx == 0 || cx == n0) : (cy == 0 || cy == n1)) &&
              (!CH || records_fluence(B, isx ? 0 : 1,
                                      isx ? (cx == 0 ? 0 : 1) : (cy == 0 ? 0 : 1)))) {
            if (isx)
              boundary_fluence<0, HLLC, NF>(B, ph, l, r, diff, F, cx == 0 ? 0 : 1, cy, n1, k,
                                            factor);
            else
              boundary_fluence<1, HLLC, NF>(B, ph, l, r, diff, F, cy == 0 ? 2 : 3, cx, n0, k,
                                            factor);
          }
        }
        // HS: the halo slopes of plane k+1, on the threads without a face in
        // the last round of the loop above
        if (HS && k + 1 < z1) {
          constexpr int TAIL = (PXF + NYF) % NT;
          static_assert(TAIL + NHS <= NT, "halo slopes fit beside the last faces");
          if (tid >= TAIL && tid < TAIL + NHS) halo_slope(tid - TAIL, k + 1);
        }
      }

      // (4) z slope at k+1 and z face k+1 of the own column
      double zsn[5], zfn[NF];
      if (PARAB) {
        // zsn: the outer values of plane k+1; the face takes the outer
        // values of plane k (zss) and the inner ones of plane k+1
        double zI[5], zl[5];
        z_parabolic(B, k + 1, full + c_off, FS, cslot(k + 1), NT, cslot(k + 2), NT, zI, zsn);
#pragma unroll
        for (int q = 0; q < 5; ++q) zl[q] = zss[q * NT + tid];
        z_face_lr<HLLC, NF, CH>(B, ph, k + 1, zl, zI, gx, gy, own, dt,
                                HLLC && (DFS ? (dfz >> 2) & 1 : df_bit<CH>(B, 2, gx, gy, k + 1)),
                                zfn);
      } else {
        z_slope(GZ, ph, k + 1, full + c_off, FS, cslot(k + 1), NT, cslot(k + 2), NT, zsn);
        z_face<HLLC, NF, CH>(B, ph, k + 1, full + c_off, FS, zss + tid, NT, cslot(k + 1), NT, zsn,
                             1, gx, gy, own, dt,
                             HLLC && (DFS ? (dfz >> 2) & 1 : df_bit<CH>(B, 2, gx, gy, k + 1)),
                             zfn);
      }
      // 8-row tiles (EPI): the update's own inputs (U^n of the cell in
      // stage 1, U^n + K1/2 in stage 2), loaded before the barrier so that
      // their latency passes while the CTA synchronises; 16-row tiles, at the
      // register cap, load them in the update
      constexpr bool EPI = TYt == 8 && MODE != MODE_INCREMENT;
      double ein[5];
      if (EPI && own) {
        if (MODE == MODE_STAGE1) {
          const long long g =
              (gx + 2) + (long long)B.m[0] * ((gy + 2) + (long long)B.m[1] * (k + 2));
#pragma unroll
          for (int q = 0; q < 5; ++q) ein[q] = __ldg(B.U_in + q * B.nV + g);
        } else {
          const long long c = gx + (long long)n0 * (gy + (long long)n1 * k);
#pragma unroll
          for (int q = 0; q < 5; ++q) ein[q] = __ldg(B.H + q * B.nP + c);
        }
      }
      __syncthreads();

      // (5) cell update and stage epilogue
      if (own) {
        const double w0 = gxc[G_W * LX + tx + 2], w1 = gyc[G_W * LY + ty + 2],
                     w2 = __ldg(GZ.W + k + 2);
        const double vol = w0 * w1 * w2;
        const double rvol = recip(vol);
        const double ax = w1 * w2, ay = w2 * w0, az = w0 * w1;
        const long long gidx =
            (gx + 2) + (long long)B.m[0] * ((gy + 2) + (long long)B.m[1] * (k + 2));
        const long long cidx = gx + (long long)n0 * (gy + (long long)n1 * k);
        // dU += dT (A_I F_I(i) - A_I F_I(i+1)) / V per direction
        // (IncrementDivergence_FV__Kernel.f90:729-748)
#if GFX_FAST_MATH
        // the speed build: dT A_d / V once per direction, times the
        // direction's flux difference, the three terms summed with fused
        // multiply-adds (a few ulps of the increment from the reference's
        // order of operations, which the exact build keeps)
        double Kc[NF];
        {
          const double cx = dt * ax * rvol, cy = dt * ay * rvol, cz = dt * az * rvol;
#pragma unroll
          for (int u = 0; u < NF; ++u) {
            const double fx = fxs[(u * TY + ty) * (TX + 1) + tx] -
                              fxs[(u * TY + ty) * (TX + 1) + tx + 1];
            const double fy = fys[(u * (TY + 1) + ty) * TX + tx] -
                              fys[(u * (TY + 1) + ty + 1) * TX + tx];
            const double fz = zfs[u * NT + tid] - zfn[u];
            Kc[u] = cx * fx + cy * fy + cz * fz;
          }
          if (MODE == MODE_INCREMENT) {
#pragma unroll
            for (int u = 0; u < NF; ++u) {
              double* kp = B.K + (long long)u * B.nV + gidx;
              *kp = *kp + Kc[u];
            }
          }
        }
#else
        // all quotients at once
        double nx_[NF], ny_[NF], nz_[NF], qx[NF], qy[NF], qz[NF];
        bool ok = true;
#pragma unroll
        for (int u = 0; u < NF; ++u) {
          nx_[u] = dt * (ax * fxs[(u * TY + ty) * (TX + 1) + tx] -
                         ax * fxs[(u * TY + ty) * (TX + 1) + tx + 1]);
          ny_[u] = dt * (ay * fys[(u * (TY + 1) + ty) * TX + tx] -
                         ay * fys[(u * (TY + 1) + ty + 1) * TX + tx]);
          nz_[u] = dt * (az * zfs[u * NT + tid] - az * zfn[u]);
          qx[u] = markstein(nx_[u], vol, rvol);
          qy[u] = markstein(ny_[u], vol, rvol);
          qz[u] = markstein(nz_[u], vol, rvol);
          ok &= geo_quotient_in_range(nx_[u]) & geo_quotient_in_range(ny_[u]) &
                geo_quotient_in_range(nz_[u]);
        }
        if (!ok) {
#pragma unroll
          for (int u = 0; u < NF; ++u) {
            qx[u] = div_ieee(nx_[u], vol);
            qy[u] = div_ieee(ny_[u], vol);
            qz[u] = div_ieee(nz_[u], vol);
          }
        }
        double Kc[NF];
#pragma unroll
        for (int u = 0; u < NF; ++u) {
          if (MODE == MODE_INCREMENT) {
            double* kp = B.K + (long long)u * B.nV + gidx;
            *kp = *kp + qx[u] + qy[u] + qz[u];
          } else {
            Kc[u] = qx[u] + qy[u] + qz[u];
          }
        }
#endif
        if (MODE != MODE_INCREMENT) {
          const double N = full[c_off], V1 = full[FS + c_off], V2 = full[2 * FS + c_off],
                       V3 = full[3 * FS + c_off], E = full[4 * FS + c_off];
          if (GRAV) {
            // ApplyGravity_F (ApplyGravity_F__Command.f90:124-264) with the
            // uniform gradient (0, 0, a); the x and y momentum terms subtract
            // an exact +0.
            const double a = ph.accel;
            Kc[3] = Kc[3] - N * a * dt;
            Kc[4] = Kc[4] - N * (V1 * 0.0 + V2 * 0.0 + V3 * a) * dt;
          }
          if (MODE == MODE_STAGE1) {
            if (B.wn) {
              B.wn[cidx] = N;
              B.wn[B.nP + cidx] = V1;
              B.wn[2 * B.nP + cidx] = V2;
              B.wn[3 * B.nP + cidx] = V3;
              B.wn[4 * B.nP + cidx] = E;
            }
            Cons u;
            {
              Cons raw;
              if (EPI) {
                raw = Cons{ein[0], ein[1], ein[2], ein[3], ein[4]};
              } else {
                const double* U = B.U_in;
                raw.D = __ldg(U + gidx);
                raw.S1 = __ldg(U + B.nV + gidx);
                raw.S2 = __ldg(U + 2 * B.nV + gidx);
                raw.S3 = __ldg(U + 3 * B.nV + gidx);
                raw.G = __ldg(U + 4 * B.nV + gidx);
              }
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
            if (!EPI) {
              const double* H = B.H;
#pragma unroll
              for (int q = 0; q < 5; ++q) ein[q] = H[q * B.nP + cidx];
            }
            Cons u{ein[0] + 0.5 * Kc[0], ein[1] + 0.5 * Kc[1], ein[2] + 0.5 * Kc[2],
                   ein[3] + 0.5 * Kc[3], ein[4] + 0.5 * Kc[4]};
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
            if (B.wn) {
              B.wn[cidx] = w.N;
              B.wn[B.nP + cidx] = w.V1;
              B.wn[2 * B.nP + cidx] = w.V2;
              B.wn[3 * B.nP + cidx] = w.V3;
              B.wn[4 * B.nP + cidx] = w.E;
            }
            tsi_max = fmax2(tsi_max,
                            inverse_cfl_time(w, CS, w0, w1, w2, gxc[G_RW * LX + tx + 2],
                                             gyc[G_RW * LY + ty + 2], __ldg(GZ.RW + k + 2)));
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 5; ++q) zss[q * NT + tid] = zsn[q];
#pragma unroll
      for (int u = 0; u < NF; ++u) zfs[u * NT + tid] = zfn[u];
      // no barrier here: the next plane's phase (1) writes only this
      // thread's centre and slots and the halo cells, none of which the
      // update above reads from other threads (it reads their x / y fluxes,
      // rewritten only after two more barriers)
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

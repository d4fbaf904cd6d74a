/*
 * fluid_oracle.c -- CPU oracle for the GenASiS Fluid_P_I finite-volume step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  Only tests/, the smoke check and
 * bench.py's cpu_baseline / reference legs load this code; the product
 * library (genasis_b200) never links or calls it.
 *
 * Parity status: unpinned by reference-run outputs.  The reference is
 * Fortran 2008 + MPI with no Fortran compiler available here and no golden
 * vectors for this path, so this file restates the reference's host-side
 * OpenMP loops statement by statement (citations below) and is pinned by the
 * known-answer tests and invariants in tests/test_oracle.py.
 *
 * What is restated, in the reference's own order of operations (all paths
 * relative to the GenASiS tree):
 *   geometry     Chart_Template.f90:478-560 (edges, float ghost widths),
 *                :827-841, :973-990, GeometryFlat_Kernel.f90:12-47
 *   BCs          Atlas_SC__Template.f90:244-406, Chart_SL__Template.f90:400-538,
 *                Chart_SL__Kernel.f90:12-113
 *   differences  Difference_Kernel.f90:12-81
 *   limiter      Gradient_Kernel.f90:166-190 (theta-only path)
 *   PLM faces    IncrementDivergence_FV__Kernel.f90:11-94
 *   prim->cons   Fluid_P_I__Form.f90:509-601, Fluid_P_I__Kernel.f90:197-271,
 *                Fluid_D__Kernel.f90:12-101, Fluid_P__Kernel.f90:12-91,242-316
 *   raw fluxes   Fluid_D__Kernel.f90:220-262, Fluid_P__Kernel.f90:671-709
 *   HLL          Current_Template.f90:609-698, Current_Kernel.f90:12-137
 *   HLLC         Fluid_P__Template.f90:445-518, Fluid_P__Kernel.f90:319-668
 *   increment    IncrementDivergence_FV__Kernel.f90:672-752
 *   fluence      IncrementDivergence_FV__Form.f90:1002-1069, _Kernel.f90:755-800
 *   cons->prim   Fluid_P_I__Form.f90:604-722, Fluid_P__Kernel.f90:94-192
 *   features     FluidFeatures_P__Form.f90:145-344, FluidFeatures_P__Kernel.f90
 *   RK2 step     Step_RK__Template.f90:207-288, Step_RK2_C_ASC__Form.f90:51-57,
 *                Step_RK_C_ASC__Template.f90:504-1281
 *   ghosts       Chart_SLD__Form.f90:131-201 (periodic faces + edges)
 *   gravity      ApplyGravity_F__Command.f90:23-264, Geometry_ASC__Kernel.f90:68-90
 *   time step    Integrator_C_PS__Kernel.f90:12-144, Integrator_C_PS__Form.f90:374-423,
 *                Integrator_Template.f90:896-939
 *
 * Build with -ffp-contract=off -fno-fast-math so every operation rounds
 * separately, as the Fortran source is written.
 */
#include "fluid_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NPRIM 5
#define NCONS 6

/* Fortran intrinsics with the argument order and tie behaviour of gfortran:
 * the first argument wins ties. */
static inline double fmax2(double a, double b) { return (b > a) ? b : a; }
static inline double fmax3(double a, double b, double c) {
  double r = a;
  if (b > r) r = b;
  if (c > r) r = c;
  return r;
}
static inline double fmin3(double a, double b, double c) {
  double r = a;
  if (b < r) r = b;
  if (c < r) r = c;
  return r;
}
/* Fortran sign(a, b) with -fsign-zero (gfortran default): |a| with b's sign bit. */
static inline double fsign(double a, double b) { return copysign(fabs(a), b); }

struct ora_fluid {
  ora_config c;
  int n[3], g, m[3];
  size_t nV, st[3];
  /* per-axis geometry, index t in [0, m) <-> Fortran cell t + 1 - g */
  double *X[3], *WL[3], *WR[3];
  /* physical constants (Fluid_P_I__Form.f90:201-223, Fluid_ASC__Form.f90:122-126) */
  double gamma, c_v, n0, p0, mass;
  /* the Current: primitives, conserved, auxiliaries */
  double *N, *V[3], *E, *D, *S[3], *Gc, *DS, *P, *SB, *CS, *FEP[3], *FEM[3];
  /* features: DIFFUSIVE_FLUX_I(3), SHOCK, SHOCK_I(3) */
  double *DF[3], *SHOCK, *SHOCK_I[3];
  /* scratch of the divergence increment */
  double *dX_I, *dV_I, *dVdX[NPRIM], *F_I[NCONS];
  double *VO[NPRIM]; /* PARABOLIC: outer face value of each cell (dVdX holds the inner) */
  /* RK storages */
  double *Sol[NCONS], *Y[NCONS], *K[2][NCONS];
};

static double *alloc_field(size_t n) {
  double *p = (double *)calloc(n, sizeof(double));
  return p;
}

static inline size_t idx3(const ora_fluid *f, int i, int j, int k) {
  return (size_t)i + (size_t)f->m[0] * ((size_t)j + (size_t)f->m[1] * (size_t)k);
}

int ora_n_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* Chart_Template.f90 SetEdgeEqual (:699-723), ghost edges (:541-548 with the
 * width variables declared real(KDL), i.e. default-real single precision),
 * SetCenterRectangular (:827-841), SetWidthLeftRight (:973-990). */
static void build_axis(ora_fluid *f, int d) {
  int n = f->n[d], g = f->g, m = f->m[d];
  double *edge = (double *)malloc(sizeof(double) * (size_t)(m + 1));
  /* edge[t] = Edge(t + 1 - g) */
  double *E1 = edge + g - 1; /* E1[i] = Edge(i), i in [1-g, n+g+1] */
  double mn = f->c.min_coordinate[d], mx = f->c.max_coordinate[d];
  double width = (mx - mn) / (double)n;
  E1[1] = mn;
  for (int i = 2; i <= n + 1; ++i) E1[i] = E1[i - 1] + width;
  for (int iC = 1; iC <= g; ++iC) {
    float w_ig = (float)(E1[iC + 1] - E1[iC]);
    float w_og = (float)(E1[n - iC + 2] - E1[n - iC + 1]);
    E1[1 - iC] = E1[2 - iC] - (double)w_ig;
    E1[n + 1 + iC] = E1[n + iC] + (double)w_og;
  }
  for (int t = 0; t < m; ++t) {
    double c = 0.5 * (edge[t] + edge[t + 1]);
    f->X[d][t] = c;
    f->WL[d][t] = c - edge[t];
    f->WR[d][t] = edge[t + 1] - c;
  }
  free(edge);
}

ora_fluid *ora_create(const ora_config *cfg) {
  ora_fluid *f = (ora_fluid *)calloc(1, sizeof(ora_fluid));
  f->c = *cfg;
  f->g = cfg->n_ghost_layers;
  for (int d = 0; d < 3; ++d) {
    f->n[d] = cfg->n_cells[d];
    f->m[d] = f->n[d] + 2 * f->g;
  }
  f->nV = (size_t)f->m[0] * f->m[1] * f->m[2];
  f->st[0] = 1;
  f->st[1] = (size_t)f->m[0];
  f->st[2] = (size_t)f->m[0] * f->m[1];
  for (int d = 0; d < 3; ++d) {
    f->X[d] = alloc_field(f->m[d]);
    f->WL[d] = alloc_field(f->m[d]);
    f->WR[d] = alloc_field(f->m[d]);
    build_axis(f, d);
  }
  /* Fluid_P_I__Form.f90:201-223: k = 1, mu = 1, c_v = k / (mu (gamma - 1)) */
  f->gamma = cfg->adiabatic_index;
  f->c_v = 1.0 / (1.0 * (f->gamma - 1.0));
  f->n0 = 1.0;
  f->p0 = 1.0;
  f->mass = 1.0;
  size_t nV = f->nV;
  f->N = alloc_field(nV); f->E = alloc_field(nV); f->D = alloc_field(nV);
  f->Gc = alloc_field(nV); f->DS = alloc_field(nV); f->P = alloc_field(nV);
  f->SB = alloc_field(nV); f->CS = alloc_field(nV);
  for (int d = 0; d < 3; ++d) {
    f->V[d] = alloc_field(nV); f->S[d] = alloc_field(nV);
    f->FEP[d] = alloc_field(nV); f->FEM[d] = alloc_field(nV);
    f->DF[d] = alloc_field(nV); f->SHOCK_I[d] = alloc_field(nV);
  }
  f->SHOCK = alloc_field(nV);
  f->dX_I = alloc_field(nV); f->dV_I = alloc_field(nV);
  for (int v = 0; v < NPRIM; ++v) {
    f->dVdX[v] = alloc_field(nV);
    f->VO[v] = alloc_field(nV);
  }
  for (int v = 0; v < NCONS; ++v) {
    f->F_I[v] = alloc_field(nV);
    f->Sol[v] = alloc_field(nV); f->Y[v] = alloc_field(nV);
    f->K[0][v] = alloc_field(nV); f->K[1][v] = alloc_field(nV);
  }
  return f;
}

void ora_destroy(ora_fluid *f) {
  if (!f) return;
  for (int d = 0; d < 3; ++d) {
    free(f->X[d]); free(f->WL[d]); free(f->WR[d]);
    free(f->V[d]); free(f->S[d]); free(f->FEP[d]); free(f->FEM[d]);
    free(f->DF[d]); free(f->SHOCK_I[d]);
  }
  free(f->N); free(f->E); free(f->D); free(f->Gc); free(f->DS); free(f->P);
  free(f->SB); free(f->CS); free(f->SHOCK); free(f->dX_I); free(f->dV_I);
  for (int v = 0; v < NPRIM; ++v) {
    free(f->dVdX[v]);
    free(f->VO[v]);
  }
  for (int v = 0; v < NCONS; ++v) {
    free(f->F_I[v]); free(f->Sol[v]); free(f->Y[v]); free(f->K[0][v]); free(f->K[1][v]);
  }
  free(f);
}

size_t ora_n_values(const ora_fluid *f) { return f->nV; }

size_t ora_fluence_face_size(const ora_fluid *f) {
  size_t a = (size_t)f->n[1] * f->n[2], b = (size_t)f->n[0] * f->n[2],
         c = (size_t)f->n[0] * f->n[1];
  size_t r = a > b ? a : b;
  return r > c ? r : c;
}

void ora_geometry(const ora_fluid *f, int axis, double *center, double *wl, double *wr) {
  memcpy(center, f->X[axis], sizeof(double) * f->m[axis]);
  memcpy(wl, f->WL[axis], sizeof(double) * f->m[axis]);
  memcpy(wr, f->WR[axis], sizeof(double) * f->m[axis]);
}

/* width of cell t along axis d: GeometryFlat_Kernel.f90:22-24 */
static inline double cell_width(const ora_fluid *f, int d, int t) {
  return f->WL[d][t] + f->WR[d][t];
}

/* ---------------------------------------------------------------------- */
/* Equation of state and prim<->cons, pointwise                            */
/* ---------------------------------------------------------------------- */

/* Apply_EOS_I_E_Kernel, Fluid_P_I__Kernel.f90:197-271 (T is not needed). */
static inline void eos_i_e(const ora_fluid *f, double N, double E, double *P, double *SB,
                           double *CS) {
  const double sqrt_huge = sqrt(DBL_MAX);
  double p = (f->gamma - 1.0) * E;
  *P = p;
  if (N > 0.0 && p > 0.0) {
    *SB = f->c_v * log(p / f->p0 * pow(f->n0 / N, f->gamma));
    *CS = sqrt(f->gamma * p / (f->mass * N));
  } else {
    *SB = -sqrt_huge;
    *CS = 0.0;
  }
}

typedef struct {
  double N, V[3], E;       /* primitives (N may be clipped to 0) */
  double D, S[3], G, DS;   /* conserved */
  double P, CS, FEP, FEM;  /* aux (fast speeds along the sweep direction) */
} face_state;

/* ComputeFromPrimitiveCommon (Fluid_P_I__Form.f90:509-601) on one face value:
 * Compute_M, Apply_EOS_I_E, Compute_D_S_G (Fluid_D__Kernel.f90:47-101),
 * Compute_G_G (Fluid_P__Kernel.f90:12-52), Compute_DS_G (:55-91),
 * Compute_FE_P_G (:242-316).  Metric entries are 1 (rectangular). */
static inline void prim_to_cons(const ora_fluid *f, const double prim[NPRIM], int d,
                                face_state *s) {
  const double M = f->mass, M_DD_22 = 1.0, M_DD_33 = 1.0, M_UU_22 = 1.0, M_UU_33 = 1.0;
  double N = prim[0], V1 = prim[1], V2 = prim[2], V3 = prim[3], E = prim[4];
  double P, SB, CS;
  eos_i_e(f, N, E, &P, &SB, &CS);
  if (N < 0.0) N = 0.0;
  double D = N;
  double S1 = M * N * V1;
  double S2 = M * N * M_DD_22 * V2;
  double S3 = M * N * M_DD_33 * V3;
  double G = E + 0.5 * (S1 * V1 + S2 * V2 + S3 * V3);
  double DS = SB * N;
  double fep[3], fem[3];
  fep[0] = V1 + CS;
  fep[1] = V2 + sqrt(M_UU_22) * CS;
  fep[2] = V3 + sqrt(M_UU_33) * CS;
  fem[0] = V1 - CS;
  fem[1] = V2 - sqrt(M_UU_22) * CS;
  fem[2] = V3 - sqrt(M_UU_33) * CS;
  s->N = N; s->V[0] = V1; s->V[1] = V2; s->V[2] = V3; s->E = E;
  s->D = D; s->S[0] = S1; s->S[1] = S2; s->S[2] = S3; s->G = G; s->DS = DS;
  s->P = P; s->CS = CS; s->FEP = fep[d]; s->FEM = fem[d];
}

/* ComputeFromConservedCommon (Fluid_P_I__Form.f90:604-722) on the Current at
 * value iV: Compute_M, Compute_N_V_E_G (Fluid_P__Kernel.f90:94-192, both
 * loops), Apply_EOS_I_E, Compute_DS_G, Compute_FE_P_G. */
static inline void cons_to_prim_at(ora_fluid *f, size_t iV) {
  const double M = f->mass, M_UU_22 = 1.0, M_UU_33 = 1.0;
  const double N_Min = f->c.baryon_density_min;
  double D = f->D[iV], S1 = f->S[0][iV], S2 = f->S[1][iV], S3 = f->S[2][iV],
         G = f->Gc[iV];
  double N, V1, V2, V3, E;
  if (D > N_Min) {
    N = D;
    V1 = S1 / (M * D);
    V2 = M_UU_22 * S2 / (M * D);
    V3 = M_UU_33 * S3 / (M * D);
    E = G - 0.5 * (S1 * V1 + S2 * V2 + S3 * V3);
  } else {
    N = N_Min; V1 = 0.0; V2 = 0.0; V3 = 0.0; E = 0.0;
    D = N_Min; S1 = 0.0; S2 = 0.0; S3 = 0.0; G = 0.0;
  }
  if (E < 0.0) {
    E = 0.0;
    G = E + 0.5 * (S1 * V1 + S2 * V2 + S3 * V3);
  }
  double P, SB, CS;
  eos_i_e(f, N, E, &P, &SB, &CS);
  f->N[iV] = N; f->V[0][iV] = V1; f->V[1][iV] = V2; f->V[2][iV] = V3; f->E[iV] = E;
  f->D[iV] = D; f->S[0][iV] = S1; f->S[1][iV] = S2; f->S[2][iV] = S3; f->Gc[iV] = G;
  f->P[iV] = P; f->SB[iV] = SB; f->CS[iV] = CS;
  f->DS[iV] = SB * N;
  f->FEP[0][iV] = V1 + CS;
  f->FEP[1][iV] = V2 + sqrt(M_UU_22) * CS;
  f->FEP[2][iV] = V3 + sqrt(M_UU_33) * CS;
  f->FEM[0][iV] = V1 - CS;
  f->FEM[1][iV] = V2 - sqrt(M_UU_22) * CS;
  f->FEM[2][iV] = V3 - sqrt(M_UU_33) * CS;
}

static void cons_to_prim_all(ora_fluid *f) {
  long long nV = (long long)f->nV;
#pragma omp parallel for schedule(static)
  for (long long iV = 0; iV < nV; ++iV) cons_to_prim_at(f, (size_t)iV);
}

/* ComputeFromPrimitiveCommon on the Current at value iV. */
static inline void prim_to_cons_at(ora_fluid *f, size_t iV) {
  double prim[NPRIM] = {f->N[iV], f->V[0][iV], f->V[1][iV], f->V[2][iV], f->E[iV]};
  face_state s;
  prim_to_cons(f, prim, 0, &s);
  double P, SB, CS;
  eos_i_e(f, prim[0], prim[4], &P, &SB, &CS);
  f->N[iV] = s.N;
  f->D[iV] = s.D; f->S[0][iV] = s.S[0]; f->S[1][iV] = s.S[1]; f->S[2][iV] = s.S[2];
  f->Gc[iV] = s.G; f->DS[iV] = s.DS; f->P[iV] = P; f->SB[iV] = SB; f->CS[iV] = CS;
  for (int d = 0; d < 3; ++d) {
    f->FEP[d][iV] = s.V[d] + CS;
    f->FEM[d][iV] = s.V[d] - CS;
  }
}

/* ---------------------------------------------------------------------- */
/* Ghost exchange (single brick): periodic faces and edges                 */
/* ---------------------------------------------------------------------- */

static inline int wrap_index(const ora_fluid *f, int d, int t) {
  int g = f->g, n = f->n[d];
  if (t < g) return t + n;
  if (t >= g + n) return t - n;
  return t;
}

/* Chart_SLD__Form.f90:131-201: faces (nGL x n x n) and edges (nGL x nGL x n)
 * are received from the periodic image; corners are not exchanged. */
static void exchange_ghosts(ora_fluid *f, double **fields, int nfields) {
  int per[3];
  for (int d = 0; d < 3; ++d) per[d] = (f->c.boundary[d][0] == ORA_BC_PERIODIC);
  int g = f->g;
  for (int k = 0; k < f->m[2]; ++k)
    for (int j = 0; j < f->m[1]; ++j)
      for (int i = 0; i < f->m[0]; ++i) {
        int t[3] = {i, j, k}, ghost[3], nghost = 0;
        for (int d = 0; d < 3; ++d) {
          ghost[d] = (t[d] < g || t[d] >= g + f->n[d]);
          nghost += ghost[d];
        }
        if (nghost == 0 || nghost == 3) continue;
        int ok = 1, s[3];
        for (int d = 0; d < 3; ++d) {
          if (ghost[d] && !per[d]) ok = 0;
          s[d] = ghost[d] ? wrap_index(f, d, t[d]) : t[d];
        }
        if (!ok) continue;
        size_t dst = idx3(f, i, j, k), src = idx3(f, s[0], s[1], s[2]);
        for (int v = 0; v < nfields; ++v) fields[v][dst] = fields[v][src];
      }
}

/* ---------------------------------------------------------------------- */
/* Boundary conditions on the reconstructed (primitive) fields             */
/* ---------------------------------------------------------------------- */

/* Atlas_SC__Template.f90:244-406 with Chart_SL__Template.f90:486-538 limits and
 * Chart_SL__Kernel.f90:12-113 kernels: mirror nGL interior layers into the
 * ghosts of face (d, side), transverse proper range only; REFLECTING also
 * negates V_d there; PERIODIC does nothing here. */
static void apply_bc(ora_fluid *f, int d, int side) {
  int bc = f->c.boundary[d][side];
  if (bc == ORA_BC_PERIODIC) return;
  double *fields[NPRIM] = {f->N, f->V[0], f->V[1], f->V[2], f->E};
  int g = f->g, n = f->n[d];
  int jd = (d + 1) % 3, kd = (jd + 1) % 3;
  for (int kk = 0; kk < f->n[kd]; ++kk)
    for (int jj = 0; jj < f->n[jd]; ++jj)
      for (int t = 0; t < g; ++t) {
        int ext[3], in[3];
        ext[jd] = in[jd] = g + jj;
        ext[kd] = in[kd] = g + kk;
        if (side == 0) {
          ext[d] = g - 1 - t;
          in[d] = g + t;
        } else {
          ext[d] = g + n + t;
          in[d] = g + n - 1 - t;
        }
        size_t e = idx3(f, ext[0], ext[1], ext[2]), s = idx3(f, in[0], in[1], in[2]);
        for (int v = 0; v < NPRIM; ++v) fields[v][e] = fields[v][s];
        if (bc == ORA_BC_REFLECTING) f->V[d][e] = -f->V[d][e];
      }
}

/* ---------------------------------------------------------------------- */
/* Fluxes at one face                                                      */
/* ---------------------------------------------------------------------- */

/* Raw fluxes along d: ComputeRawFluxes_G_Kernel (Fluid_D__Kernel.f90:220-262)
 * then ComputeRawFluxesTemplate_P_Kernel (Fluid_P__Kernel.f90:671-709). */
static inline void raw_flux(const double D, const double S[3], const double G,
                            const double DS, const double P, const double Vd, int d,
                            double F[NCONS]) {
  F[0] = D * Vd;
  F[1] = S[0] * Vd;
  F[2] = S[1] * Vd;
  F[3] = S[2] * Vd;
  F[1 + d] = F[1 + d] + P;
  F[4] = (G + P) * Vd;
  F[5] = DS * Vd;
}

/* HLL (Current_Template.f90:609-675 + Current_Kernel.f90) and optional HLLC
 * (Fluid_P__Template.f90:445-518 + Fluid_P__Kernel.f90:319-668) for one face
 * with left state L and right state R. */
static inline void face_flux(const ora_fluid *f, const face_state *L, const face_state *R,
                             int d, double df_feature, double F[NCONS]) {
  const double tiny = DBL_MIN, sqrt_tiny = sqrt(DBL_MIN);
  const double M = f->mass, M_UU = 1.0, M_DD_22 = 1.0, M_DD_33 = 1.0;
  double FL[NCONS], FR[NCONS];
  raw_flux(L->D, L->S, L->G, L->DS, L->P, L->V[d], d, FL);
  raw_flux(R->D, R->S, R->G, R->DS, R->P, R->V[d], d, FR);
  /* ComputeSolverSpeeds_HLL_Kernel */
  double AP = fmax3(0.0, +L->FEP, +R->FEP);
  double AM = fmax3(0.0, -L->FEM, -R->FEM);
  /* SetDiffusionFactorUnity: DF = 1 */
  const double DF = 1.0;
  double UL[NCONS] = {L->D, L->S[0], L->S[1], L->S[2], L->G, L->DS};
  double UR[NCONS] = {R->D, R->S[0], R->S[1], R->S[2], R->G, R->DS};
  for (int u = 0; u < NCONS; ++u)
    F[u] = (AP * FL[u] + AM * FR[u] - DF * AP * AM * (UR[u] - UL[u])) /
           fmax2(AP + AM, tiny);
  if (f->c.riemann_solver != ORA_HLLC) return;

  /* ComputeCenterSpeedKernel (Fluid_P__Kernel.f90:319-391) */
  double MD_Numerator = AP * M * R->D + AM * M * L->D - FR[0] + FL[0];
  double S_Numerator = AP * R->S[d] + AM * L->S[d] - FR[1 + d] + FL[1 + d];
  double MD_Numerator_Inv = fmax2(MD_Numerator, 0.0) / fmax2(MD_Numerator * MD_Numerator, tiny);
  double AC = M_UU * S_Numerator * MD_Numerator_Inv;

  /* ComputeCenterStatesKernel (Fluid_P__Kernel.f90:394-601) */
  double V_CL[3] = {L->V[0], L->V[1], L->V[2]}, V_CR[3] = {R->V[0], R->V[1], R->V[2]};
  V_CL[d] = AC;
  V_CR[d] = AC;
  double AM_VL = AM + L->V[d];
  double AM_AC = AM + AC;
  double AM_AC_Inv = 1.0 / fmax2(fabs(AM_AC), sqrt_tiny);
  double AP_VR = AP - R->V[d];
  double AP_AC = AP - AC;
  double AP_AC_Inv = 1.0 / fmax2(fabs(AP_AC), sqrt_tiny);
  double D_CL = L->D * AM_VL * AM_AC_Inv;
  double D_CR = R->D * AP_VR * AP_AC_Inv;
  double S_CL[3], S_CR[3];
  S_CL[0] = M * D_CL * V_CL[0];
  S_CR[0] = M * D_CR * V_CR[0];
  S_CL[1] = M_DD_22 * M * D_CL * V_CL[1];
  S_CR[1] = M_DD_22 * M * D_CR * V_CR[1];
  S_CL[2] = M_DD_33 * M * D_CL * V_CL[2];
  S_CR[2] = M_DD_33 * M * D_CR * V_CR[2];
  double P_CL = L->P + L->S[d] * AM_VL - S_CL[d] * AM_AC;
  double P_CR = R->P - R->S[d] * AP_VR + S_CR[d] * AP_AC;
  double G_CL = (L->G * AM_VL + L->V[d] * L->P - AC * P_CL) * AM_AC_Inv;
  double G_CR = (R->G * AP_VR - R->V[d] * R->P + AC * P_CR) * AP_AC_Inv;
  double DS_CL = L->DS * AM_VL * AM_AC_Inv;
  double DS_CR = R->DS * AP_VR * AP_AC_Inv;
  double FCL[NCONS], FCR[NCONS];
  raw_flux(D_CL, S_CL, G_CL, DS_CL, P_CL, V_CL[d], d, FCL);
  raw_flux(D_CR, S_CR, G_CR, DS_CR, P_CR, V_CR[d], d, FCR);

  /* ComputeFluxes_HLLC_Kernel (Fluid_P__Kernel.f90:604-668) */
  if (df_feature > 0.0) return;
  if (AP != 0.0 && AM != 0.0) {
    if (AC >= 0.0)
      for (int u = 0; u < NCONS; ++u) F[u] = FCL[u];
    else
      for (int u = 0; u < NCONS; ++u) F[u] = FCR[u];
  }
}

/* ---------------------------------------------------------------------- */
/* IncrementDivergence_FV % Compute (IncrementDivergence_FV__Form.f90:344-412) */
/* ---------------------------------------------------------------------- */

/* ComputeReconstructionParabolic_CSL_Kernel (IncrementDivergence_FV__Kernel.f90:
 * 296-596) for one cell, with the cell averages XA = X and X2A = X**2 that its
 * caller passes (IncrementDivergence_FV__Form.f90:850-927): a parabola through
 * the three cell values, adjusted where it has an extremum inside the cell
 * pair, then a second parabola through the face values and the cell value,
 * adjusted likewise.  Fortran's left-to-right evaluation and x**2 = x*x are
 * kept; SqrtTiny is tiny(0.0) as the reference sets it.  Returns the inner
 * (vI) and outer (vO) face values of the cell. */
static void parabolic_cell(double vM, double vC, double vP, double xM, double xC, double xP,
                           double xI, double xO, double *pvI, double *pvO) {
  const double SqrtTiny = DBL_MIN;
  const double xAM = xM, xAC = xC, xAP = xP;
  const double x2AM = xM * xM, x2AC = xC * xC, x2AP = xP * xP;
  double vI, vO, D, c0, c1, c2, c2_Safe, xE;
  if ((vC - vM) * (vP - vC) <= 0.0) {
    vI = vC;
    vO = vC;
  } else {
    /* first parabola */
    D = (x2AM - x2AP) * xAC + (x2AP - x2AC) * xAM + (x2AC - x2AM) * xAP;
    c0 = (vP * (x2AM * xAC - x2AC * xAM) + vM * (x2AC * xAP - x2AP * xAC) +
          vC * (x2AP * xAM - x2AM * xAP)) / D;
    c1 = (vP * (x2AC - x2AM) + vC * (x2AM - x2AP) + vM * (x2AP - x2AC)) / D;
    c2 = (vP * (xAM - xAC) + vM * (xAC - xAP) + vC * (xAP - xAM)) / D;
    c2_Safe = copysign(fmax2(fabs(c2), SqrtTiny), c2);
    xE = -(c1 / (2.0 * c2_Safe));
    vI = c0 + c1 * xI + c2 * (xI * xI);
    vO = c0 + c1 * xO + c2 * (xO * xO);
    /* extremum of the first parabola inside (xM, xC] or (xC, xP) */
    if (xE > xM && xE <= xC) {
      D = (x2AC - x2AM) + 2.0 * (xAM - xAC) * xAM;
      c0 = ((vM * x2AC - vC * x2AM) + 2.0 * (vC * xAM - vM * xAC) * xAM) / D;
      c1 = -(2.0 * (vC - vM) * xAM / D);
      c2 = (vC - vM) / D;
      vI = c0 + c1 * xI + c2 * (xI * xI);
    } else if (xE > xC && xE < xP) {
      D = (x2AC - x2AP) + 2.0 * (xAP - xAC) * xAP;
      c0 = ((vP * x2AC - vC * x2AP) + 2.0 * (vC * xAP - vP * xAC) * xAP) / D;
      c1 = -(2.0 * (vC - vP) * xAP / D);
      c2 = (vC - vP) / D;
      vO = c0 + c1 * xO + c2 * (xO * xO);
    }
    /* second parabola, through vI, vC (as the average) and vO */
    D = (xI - xO) * (x2AC + xI * xO - xAC * (xI + xO));
    c0 = (vO * xI * (x2AC - xAC * xI) + vC * xI * xO * (xI - xO) + vI * xO * (xAC * xO - x2AC)) /
         D;
    c1 = (vO * (xI * xI - x2AC) + vI * (x2AC - xO * xO) + vC * (xO * xO - xI * xI)) / D;
    c2 = (vO * (xAC - xI) + vC * (xI - xO) + vI * (xO - xAC)) / D;
    c2_Safe = copysign(fmax2(fabs(c2), SqrtTiny), c2);
    xE = -(c1 / (2.0 * c2_Safe));
    vI = c0 + c1 * xI + c2 * (xI * xI);
    vO = c0 + c1 * xO + c2 * (xO * xO);
    /* extremum of the second parabola inside (xI, xC] or (xC, xO) */
    if (xE > xI && xE <= xC) {
      D = (x2AC - xO * xO) + 2.0 * xI * (xO - xAC);
      c0 = ((vO * x2AC - vC * (xO * xO)) + 2.0 * xI * (vC * xO - vO * xAC)) / D;
      c1 = -(2.0 * (vC - vO) * xI / D);
      c2 = (vC - vO) / D;
      vI = c0 + c1 * xI + c2 * (xI * xI);
    } else if (xE > xC && xE < xO) {
      D = (x2AC - xI * xI) + 2.0 * xO * (xI - xAC);
      c0 = ((vI * x2AC - vC * (xI * xI)) + 2.0 * xO * (vC * xI - vI * xAC)) / D;
      c1 = -(2.0 * (vC - vI) * xO / D);
      c2 = (vC - vI) / D;
      vO = c0 + c1 * xO + c2 * (xO * xO);
    }
  }
  *pvI = vI;
  *pvO = vO;
}

static void compute_direction(ora_fluid *f, int d, double **dU, double dT, double weight,
                              double *fluence) {
  const int g = f->g;
  const size_t sd = f->st[d];
  double *prim[NPRIM] = {f->N, f->V[0], f->V[1], f->V[2], f->E};

  /* ComputeReconstruction: BCs on both faces of d (:625-628) */
  apply_bc(f, d, 0);
  apply_bc(f, d, 1);

  /* Index ranges (0-based) along d and transverse (proper). */
  int lo[3], hi[3];
  for (int e = 0; e < 3; ++e) {
    lo[e] = g;
    hi[e] = g + f->n[e] - 1;
  }

  /* Difference_Kernel.f90: dV_I(i) = V(i) - V(i-1) for i in [g-1, m-1]
   * along d; the coordinate difference comes from the cell centres. */
  /* Gradient_Kernel.f90:166-190: slope at i in [g-1, m-2] along d. */
  const double theta = f->c.limiter_parameter;
  for (int v = -1; v < NPRIM; ++v) {
    double *src = (v < 0) ? NULL : prim[v];
    double *dst = (v < 0) ? f->dX_I : f->dV_I;
    int l3[3] = {lo[0], lo[1], lo[2]}, h3[3] = {hi[0], hi[1], hi[2]};
    l3[d] = g - 1;
    h3[d] = f->m[d] - 1;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = l3[2]; k <= h3[2]; ++k)
      for (int j = l3[1]; j <= h3[1]; ++j)
        for (int i = l3[0]; i <= h3[0]; ++i) {
          int t[3] = {i, j, k};
          size_t iV = idx3(f, i, j, k);
          if (v < 0)
            dst[iV] = f->X[d][t[d]] - f->X[d][t[d] - 1];
          else
            dst[iV] = src[iV] - src[iV - sd];
        }
    if (v < 0) continue;
    h3[d] = f->m[d] - 2;
    double *slope = f->dVdX[v];
    if (f->c.reconstruction == ORA_PARABOLIC) {
      /* inner face values into dVdX, outer ones into VO */
      double *outer = f->VO[v];
#pragma omp parallel for collapse(2) schedule(static)
      for (int k = l3[2]; k <= h3[2]; ++k)
        for (int j = l3[1]; j <= h3[1]; ++j)
          for (int i = l3[0]; i <= h3[0]; ++i) {
            int t[3] = {i, j, k};
            size_t iV = idx3(f, i, j, k);
            const int c = t[d];
            const double xC = f->X[d][c];
            parabolic_cell(src[iV - sd], src[iV], src[iV + sd], f->X[d][c - 1], xC,
                           f->X[d][c + 1], xC - f->WL[d][c], xC + f->WR[d][c], &slope[iV],
                           &outer[iV]);
          }
      continue;
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = l3[2]; k <= h3[2]; ++k)
      for (int j = l3[1]; j <= h3[1]; ++j)
        for (int i = l3[0]; i <= h3[0]; ++i) {
          size_t iV = idx3(f, i, j, k);
          double dV_L = f->dV_I[iV], dV_R = f->dV_I[iV + sd];
          double dX_L = f->dX_I[iV], dX_R = f->dX_I[iV + sd];
          double central = (dX_R * dX_R * dV_L + dX_L * dX_L * dV_R) /
                           (dX_L * dX_R * (dX_L + dX_R));
          if (f->c.use_limiter)
            slope[iV] = (fsign(0.5, dV_L) + fsign(0.5, dV_R)) *
                        fmin3(fabs(theta * dV_L / dX_L), fabs(theta * dV_R / dX_R),
                              fabs(central));
          else
            slope[iV] = central;
        }
  }

  /* Faces i in [g, g+n] along d (IncrementDivergence_FV__Kernel.f90:30-41),
   * transverse proper: PLM states, ComputeFromPrimitive on both sides,
   * then the Riemann fluxes. */
  {
    int l3[3] = {lo[0], lo[1], lo[2]}, h3[3] = {hi[0], hi[1], hi[2]};
    h3[d] = g + f->n[d];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = l3[2]; k <= h3[2]; ++k)
      for (int j = l3[1]; j <= h3[1]; ++j)
        for (int i = l3[0]; i <= h3[0]; ++i) {
          int t[3] = {i, j, k};
          size_t iV = idx3(f, i, j, k), iM = iV - sd;
          double pl[NPRIM], pr[NPRIM];
          if (f->c.reconstruction == ORA_PARABOLIC) {
            /* V_IL(i) = vO(i-1), V_IR(i) = vI(i) (Kernel.f90:588-589) */
            for (int v = 0; v < NPRIM; ++v) {
              pl[v] = f->VO[v][iM];
              pr[v] = f->dVdX[v][iV];
            }
          } else {
            for (int v = 0; v < NPRIM; ++v) {
              pl[v] = prim[v][iM] + f->WR[d][t[d] - 1] * f->dVdX[v][iM];
              pr[v] = prim[v][iV] - f->WL[d][t[d]] * f->dVdX[v][iV];
            }
          }
          face_state L, R;
          prim_to_cons(f, pl, d, &L);
          prim_to_cons(f, pr, d, &R);
          double F[NCONS];
          face_flux(f, &L, &R, d, f->DF[d][iV], F);
          for (int u = 0; u < NCONS; ++u) f->F_I[u][iV] = F[u];
        }
  }

  /* ComputeIncrement_CSL_Kernel (IncrementDivergence_FV__Kernel.f90:672-752):
   * proper cells, areas and volumes per cell (GeometryFlat_Kernel.f90:22-41). */
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = lo[2]; k <= hi[2]; ++k)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int i = lo[0]; i <= hi[0]; ++i) {
        int t[3] = {i, j, k};
        size_t iV = idx3(f, i, j, k), iP = iV + sd;
        double w0 = cell_width(f, 0, i), w1 = cell_width(f, 1, j), w2 = cell_width(f, 2, k);
        double vol = w0 * w1 * w2;
        double area;
        if (d == 0) area = w1 * w2;
        else if (d == 1) area = w2 * w0;
        else area = w0 * w1;
        /* area at cell i+1: same transverse widths */
        int tp[3] = {t[0], t[1], t[2]};
        tp[d] += 1;
        double wp0 = cell_width(f, 0, tp[0]), wp1 = cell_width(f, 1, tp[1]),
               wp2 = cell_width(f, 2, tp[2]);
        double area_p;
        if (d == 0) area_p = wp1 * wp2;
        else if (d == 1) area_p = wp2 * wp0;
        else area_p = wp0 * wp1;
        for (int u = 0; u < NCONS; ++u)
          dU[u][iV] = dU[u][iV] + dT * (area * f->F_I[u][iV] - area_p * f->F_I[u][iP]) / vol;
      }

  /* RecordBoundaryFluence_CSL (IncrementDivergence_FV__Form.f90:1002-1069):
   * single brick, both faces; Factor = Weight_RK * dT. */
  if (fluence) {
    size_t fs = ora_fluence_face_size(f);
    int a = (d == 0) ? 1 : 0, b = (d == 2) ? 1 : 2;
    double factor = weight * dT;
    for (int side = 0; side < 2; ++side) {
      int face = 2 * d + side;
      int td = (side == 0) ? g : g + f->n[d];
      for (int u = 0; u < NCONS; ++u) {
        double *bf = fluence + ((size_t)u * 6 + face) * fs;
        for (int jb = 0; jb < f->n[b]; ++jb)
          for (int ja = 0; ja < f->n[a]; ++ja) {
            int t[3];
            t[d] = td;
            t[a] = g + ja;
            t[b] = g + jb;
            size_t iV = idx3(f, t[0], t[1], t[2]);
            size_t o = (size_t)ja + (size_t)f->n[a] * jb;
            bf[o] = bf[o] + factor * f->F_I[u][iV];
          }
      }
    }
  }
}

void ora_increment(ora_fluid *f, double *K, double dt, double weight, double *fluence) {
  double *dU[NCONS];
  for (int u = 0; u < NCONS; ++u) dU[u] = K + (size_t)u * f->nV;
  for (int d = 0; d < 3; ++d) compute_direction(f, d, dU, dt, weight, fluence);
}

/* ApplyGravity_F (ApplyGravity_F__Command.f90:23-264) with the uniform
 * potential gradient (0, 0, a) of Geometry_ASC__Kernel.f90:68-90. */
static void apply_gravity(ora_fluid *f, double **Kc, double dt, double weight, double *src) {
  const double a = f->c.uniform_acceleration;
  if (a == 0.0) return;
  const double M = f->mass;
  const double grad[3] = {0.0, 0.0, a};
  int g = f->g;
  /* Sources_F: Gravitational_G, then Gravitational_S_D (1:3) */
  double *SG = src ? src + (size_t)NCONS * f->nV : NULL;
  for (int d = 0; d < 3; ++d) {
    double *SS = src ? src + (size_t)(NCONS + 1 + d) * f->nV : NULL;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = g; k < g + f->n[2]; ++k)
      for (int j = g; j < g + f->n[1]; ++j)
        for (int i = g; i < g + f->n[0]; ++i) {
          size_t iV = idx3(f, i, j, k);
          Kc[1 + d][iV] = Kc[1 + d][iV] - M * f->D[iV] * grad[d] * dt;
          if (SS) SS[iV] = SS[iV] - M * f->D[iV] * grad[d] * weight;
        }
  }
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = g; k < g + f->n[2]; ++k)
    for (int j = g; j < g + f->n[1]; ++j)
      for (int i = g; i < g + f->n[0]; ++i) {
        size_t iV = idx3(f, i, j, k);
        Kc[4][iV] = Kc[4][iV] - M * f->D[iV] *
                                    (f->V[0][iV] * grad[0] + f->V[1][iV] * grad[1] +
                                     f->V[2][iV] * grad[2]) *
                                    dt;
        if (SG)
          SG[iV] = SG[iV] - M * f->D[iV] *
                                (f->V[0][iV] * grad[0] + f->V[1][iV] * grad[1] +
                                 f->V[2][iV] * grad[2]) *
                                weight;
      }
}

/* RecordDivergenceKernel (Step_RK_C_ASC__Kernel.f90:12-46) as
 * ApplyDivergence_C calls it after the stage's divergence
 * (Step_RK_C_ASC__Template.f90:1548-1595): the records are cleared in stage
 * 1, then S = S + Weight_RK * K / dt over every value of each conserved
 * field.  In stage 1 the gravitational records are cleared too
 * (ApplyGravity_F__Command.f90:68-92). */
static void record_divergence(ora_fluid *f, double **Kc, double dt, double weight, int s,
                              double *src) {
  const long long n = (long long)f->nV;
  if (s == 0) memset(src, 0, sizeof(double) * (NCONS + 4) * f->nV);
  for (int u = 0; u < NCONS; ++u) {
    double *S = src + (size_t)u * f->nV, *K = Kc[u];
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < n; ++i) S[i] = S[i] + weight * K[i] / dt;
  }
}

/* ---------------------------------------------------------------------- */
/* Features                                                                */
/* ---------------------------------------------------------------------- */

void ora_clear_features(ora_fluid *f) {
  for (int d = 0; d < 3; ++d) {
    memset(f->DF[d], 0, sizeof(double) * f->nV);
    memset(f->SHOCK_I[d], 0, sizeof(double) * f->nV);
  }
  memset(f->SHOCK, 0, sizeof(double) * f->nV);
}

/* FluidFeatures_P % Detect (FluidFeatures_P__Form.f90:145-171, 267-344):
 * DetectShocks_CSL_Kernel on [oV, size-oV+1] in every dimension, then
 * ClearBoundary_CSL_Kernel (single brick: inner and outer faces). */
void ora_detect_features(ora_fluid *f) {
  ora_clear_features(f);
  const double ST = f->c.shock_threshold, sqrt_tiny = sqrt(DBL_MIN);
  int lo = f->g - 1;
  for (int iD = 0; iD < 3; ++iD) {
    int jD = (iD + 1) % 3, kD = (jD + 1) % 3;
    size_t si = f->st[iD], sj = f->st[jD], sk = f->st[kD];
    for (int k = lo; k <= f->m[2] - f->g; ++k)
      for (int j = lo; j <= f->m[1] - f->g; ++j)
        for (int i = lo; i <= f->m[0] - f->g; ++i) {
          size_t c = idx3(f, i, j, k), ci = c - si;
          double dP = fabs(f->P[c] - f->P[ci]);
          double pmn = f->P[c] < f->P[ci] ? f->P[c] : f->P[ci];
          double P_Min = fmax2(pmn, sqrt_tiny);
          double dLnP = dP / P_Min;
          double dV_iD = f->V[iD][c] - f->V[iD][ci];
          if (dLnP > ST && dV_iD <= 0.0) {
            f->SHOCK_I[iD][c] = 1.0;
            f->SHOCK[c] = f->SHOCK[c] + 1.0;
            f->SHOCK[ci] = f->SHOCK[ci] + 1.0;
            f->DF[jD][c] = 1.0;
            f->DF[jD][ci] = 1.0;
            f->DF[jD][c + sj] = 1.0;
            f->DF[jD][ci + sj] = 1.0;
            f->DF[kD][c] = 1.0;
            f->DF[kD][ci] = 1.0;
            f->DF[kD][c + sk] = 1.0;
            f->DF[kD][ci + sk] = 1.0;
          }
        }
  }
  for (int iD = 0; iD < 3; ++iD) {
    int jD = (iD + 1) % 3, kD = (jD + 1) % 3;
    for (int side = 0; side < 2; ++side) {
      int l[3], u[3];
      for (int e = 0; e < 3; ++e) {
        l[e] = (side == 0) ? f->g - 1 : f->g - 2;
        u[e] = f->m[e] - f->g;
      }
      if (side == 0) {
        u[iD] = l[iD] + 1;
      } else {
        l[iD] = f->m[iD] - f->g - 1;
      }
      for (int k = l[2]; k <= u[2]; ++k)
        for (int j = l[1]; j <= u[1]; ++j)
          for (int i = l[0]; i <= u[0]; ++i) {
            size_t c = idx3(f, i, j, k);
            f->SHOCK[c] = 0.0;
            f->SHOCK_I[iD][c] = 0.0;
            f->DF[iD][c] = 0.0;
            f->DF[jD][c] = 0.0;
            f->DF[kD][c] = 0.0;
          }
    }
  }
}

void ora_get_features(const ora_fluid *f, double *feat) {
  size_t nV = f->nV;
  for (int d = 0; d < 3; ++d) memcpy(feat + d * nV, f->DF[d], sizeof(double) * nV);
  memcpy(feat + 3 * nV, f->SHOCK, sizeof(double) * nV);
  for (int d = 0; d < 3; ++d) memcpy(feat + (4 + d) * nV, f->SHOCK_I[d], sizeof(double) * nV);
}

void ora_set_features(ora_fluid *f, const double *feat) {
  size_t nV = f->nV;
  for (int d = 0; d < 3; ++d) memcpy(f->DF[d], feat + d * nV, sizeof(double) * nV);
  memcpy(f->SHOCK, feat + 3 * nV, sizeof(double) * nV);
  for (int d = 0; d < 3; ++d) memcpy(f->SHOCK_I[d], feat + (4 + d) * nV, sizeof(double) * nV);
}

/* ---------------------------------------------------------------------- */
/* State in / out                                                          */
/* ---------------------------------------------------------------------- */

void ora_set_primitive(ora_fluid *f, const double *prim) {
  size_t nV = f->nV;
  memcpy(f->N, prim, sizeof(double) * nV);
  for (int d = 0; d < 3; ++d) memcpy(f->V[d], prim + (1 + d) * nV, sizeof(double) * nV);
  memcpy(f->E, prim + 4 * nV, sizeof(double) * nV);
  /* Integrator_C_PS__Form.f90:201-203: exchange, then ComputeFromInitial */
  double *fields[NPRIM] = {f->N, f->V[0], f->V[1], f->V[2], f->E};
  exchange_ghosts(f, fields, NPRIM);
  long long n = (long long)nV;
#pragma omp parallel for schedule(static)
  for (long long iV = 0; iV < n; ++iV) prim_to_cons_at(f, (size_t)iV);
}

void ora_set_conserved(ora_fluid *f, const double *cons) {
  size_t nV = f->nV;
  memcpy(f->D, cons, sizeof(double) * nV);
  for (int d = 0; d < 3; ++d) memcpy(f->S[d], cons + (1 + d) * nV, sizeof(double) * nV);
  memcpy(f->Gc, cons + 4 * nV, sizeof(double) * nV);
  memcpy(f->DS, cons + 5 * nV, sizeof(double) * nV);
  cons_to_prim_all(f);
}

void ora_get_conserved(const ora_fluid *f, double *cons) {
  size_t nV = f->nV;
  memcpy(cons, f->D, sizeof(double) * nV);
  for (int d = 0; d < 3; ++d) memcpy(cons + (1 + d) * nV, f->S[d], sizeof(double) * nV);
  memcpy(cons + 4 * nV, f->Gc, sizeof(double) * nV);
  memcpy(cons + 5 * nV, f->DS, sizeof(double) * nV);
}

void ora_get_primitive(const ora_fluid *f, double *prim) {
  size_t nV = f->nV;
  memcpy(prim, f->N, sizeof(double) * nV);
  for (int d = 0; d < 3; ++d) memcpy(prim + (1 + d) * nV, f->V[d], sizeof(double) * nV);
  memcpy(prim + 4 * nV, f->E, sizeof(double) * nV);
}

void ora_get_aux(const ora_fluid *f, double *aux) {
  size_t nV = f->nV;
  memcpy(aux, f->P, sizeof(double) * nV);
  memcpy(aux + nV, f->CS, sizeof(double) * nV);
  for (int d = 0; d < 3; ++d) {
    memcpy(aux + (2 + d) * nV, f->FEP[d], sizeof(double) * nV);
    memcpy(aux + (5 + d) * nV, f->FEM[d], sizeof(double) * nV);
  }
  memcpy(aux + 8 * nV, f->SB, sizeof(double) * nV);
}

/* ---------------------------------------------------------------------- */
/* RK2 step (Step_RK_C_ASC__Template.f90:504-542 -> Step_RK__Template.f90:207-288) */
/* ---------------------------------------------------------------------- */

static double **cons_fields(ora_fluid *f, double **out) {
  out[0] = f->D; out[1] = f->S[0]; out[2] = f->S[1]; out[3] = f->S[2];
  out[4] = f->Gc; out[5] = f->DS;
  return out;
}

static void copy_fields(double **dst, double **src, size_t nV) {
  for (int u = 0; u < NCONS; ++u) memcpy(dst[u], src[u], sizeof(double) * nV);
}

/* MultiplyAdd_Command.f90:80-91: A = A + c * B over every value */
static void multiply_add(double **A, double **B, double c, size_t nV) {
  long long n = (long long)nV;
  for (int u = 0; u < NCONS; ++u) {
    double *a = A[u], *b = B[u];
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < n; ++i) a[i] = a[i] + c * b[i];
  }
}

/* ComputeStage_C (Step_RK_C_ASC__Template.f90:1148-1260) for stage s. */
static void compute_stage(ora_fluid *f, int s, double dt, double weight, double *fluence,
                          double *src) {
  double **Kc = f->K[s];
  for (int u = 0; u < NCONS; ++u) memset(Kc[u], 0, sizeof(double) * f->nV);
  for (int d = 0; d < 3; ++d) compute_direction(f, d, Kc, dt, weight, fluence);
  if (src) record_divergence(f, Kc, dt, weight, s, src);
  apply_gravity(f, Kc, dt, weight, src);
  exchange_ghosts(f, Kc, NCONS);
}

void ora_step(ora_fluid *f, double dt, double *fluence) { ora_step_sources(f, dt, fluence, NULL); }

/* src (may be NULL): [NCONS + 4][nV], the step's Sources records -- the
 * divergence sources of the conserved fields, then Gravitational_G and
 * Gravitational_S_D (1:3), Sources_F__Form.f90:157-167. */
void ora_step_sources(ora_fluid *f, double dt, double *fluence, double *src) {
  const double A21 = 1.0, B[2] = {0.5, 0.5};
  double *cur[NCONS];
  cons_fields(f, cur);
  if (fluence) memset(fluence, 0, sizeof(double) * NCONS * 6 * ora_fluence_face_size(f));
  /* LoadSolution: Solution = Current conserved */
  copy_fields(f->Sol, cur, f->nV);
  /* stage 1 */
  compute_stage(f, 0, dt, B[0], fluence, src);
  /* stage 2: Y = Solution; Y += A21 K1; StoreSolution_C(Y) without features */
  copy_fields(f->Y, f->Sol, f->nV);
  multiply_add(f->Y, f->K[0], A21, f->nV);
  copy_fields(cur, f->Y, f->nV);
  cons_to_prim_all(f);
  compute_stage(f, 1, dt, B[1], fluence, src);
  /* assemble: Solution += B_s K_s */
  multiply_add(f->Sol, f->K[0], B[0], f->nV);
  multiply_add(f->Sol, f->K[1], B[1], f->nV);
  /* StoreSolution with feature detection */
  copy_fields(cur, f->Sol, f->nV);
  cons_to_prim_all(f);
  ora_detect_features(f);
}

/* ComputeTimeStepKernel_CSL, 3-D branch (Integrator_C_PS__Kernel.f90:97-142) */
double ora_inverse_timestep(const ora_fluid *f) {
  int g = f->g;
  double tsi = -DBL_MAX;
  const double crsn_2 = 1.0, crsn_3 = 1.0;
#pragma omp parallel for collapse(2) reduction(max : tsi) schedule(static)
  for (int k = g; k < g + f->n[2]; ++k)
    for (int j = g; j < g + f->n[1]; ++j)
      for (int i = g; i < g + f->n[0]; ++i) {
        size_t iV = idx3(f, i, j, k);
        double v = fmax2(f->FEP[0][iV], -f->FEM[0][iV]) / (f->WL[0][i] + f->WR[0][i]) +
                   fmax2(f->FEP[1][iV], -f->FEM[1][iV]) /
                       (crsn_2 * (f->WL[1][j] + f->WR[1][j])) +
                   fmax2(f->FEP[2][iV], -f->FEM[2][iV]) /
                       (crsn_3 * (f->WL[2][k] + f->WR[2][k]));
        tsi = fmax2(tsi, v);
      }
  return tsi;
}

/* ComputeTimeStep (Integrator_Template.f90:896-939) with the Courant factor of
 * Integrator_C_PS__Form.f90:419. */
double ora_timestep(const ora_fluid *f, int i_cycle) {
  double tsi = ora_inverse_timestep(f);
  tsi = fmax2(DBL_MIN, tsi);
  double dt = DBL_MAX;
  double cand = 1.0 / tsi;
  if (cand < dt) dt = cand;
  dt = f->c.courant_factor * dt;
  double ramp = (double)(i_cycle + 1) / (double)f->c.n_ramp_cycles;
  if (ramp > 1.0) ramp = 1.0;
  if (ramp < 1.0) dt = ramp * dt;
  return dt;
}

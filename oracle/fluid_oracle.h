/*
 * fluid_oracle.h -- CPU oracle for the GenASiS Fluid_P_I finite-volume step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the
 * reference's CPU (OpenMP host) path, used by tests/, the smoke check and the
 * CPU-baseline leg of bench.py as the checker.  The product library never
 * links, loads or calls it.
 *
 * Parity status: UNPINNED by reference-run outputs.  The reference is
 * Fortran 2008 + MPI and there is no Fortran compiler in this environment, so
 * it cannot be built; the reference ships no golden vectors for this path.
 * The restatement follows the reference source statement by statement (file:line
 * citations in fluid_oracle.c) and is pinned by the hand-derived known-answer
 * tests and physics invariants in tests/test_oracle.py.
 */
#ifndef GFX_FLUID_ORACLE_H
#define GFX_FLUID_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORA_BC_OUTFLOW = 0, ORA_BC_REFLECTING = 1, ORA_BC_PERIODIC = 2 };
enum { ORA_HLL = 0, ORA_HLLC = 1 };
enum { ORA_LINEAR = 0, ORA_PARABOLIC = 1 };

typedef struct ora_config {
  int    n_cells[3];
  int    n_ghost_layers;
  double min_coordinate[3];
  double max_coordinate[3];
  int    boundary[3][2];
  int    riemann_solver;
  int    use_limiter;
  double limiter_parameter;
  double adiabatic_index;
  double shock_threshold;
  double courant_factor;
  double baryon_density_min;
  double uniform_acceleration;
  int    n_ramp_cycles;
  int    reconstruction;  /* 0 = LINEAR (PLM), 1 = PARABOLIC */
} ora_config;

typedef struct ora_fluid ora_fluid;

ora_fluid *ora_create(const ora_config *cfg);
void   ora_destroy(ora_fluid *f);
size_t ora_n_values(const ora_fluid *f);
size_t ora_fluence_face_size(const ora_fluid *f);
void   ora_geometry(const ora_fluid *f, int axis, double *center,
                    double *width_left, double *width_right);

/* Initial state from primitives [N, V1, V2, V3, E][nV] on every value,
 * followed by the ghost exchange of periodic faces (PrepareEvolution). */
void ora_set_primitive(ora_fluid *f, const double *prim);
/* State from conserved [D, S1, S2, S3, G, DS][nV] (ComputeFromConserved,
 * no feature detection). */
void ora_set_conserved(ora_fluid *f, const double *cons);
void ora_get_conserved(const ora_fluid *f, double *cons);
void ora_get_primitive(const ora_fluid *f, double *prim);
/* aux: [P, CS, FEP1, FEP2, FEP3, FEM1, FEM2, FEM3, SB][nV] */
void ora_get_aux(const ora_fluid *f, double *aux);

void ora_clear_features(ora_fluid *f);
void ora_detect_features(ora_fluid *f);
/* features: [DIFFUSIVE_FLUX_I 1..3, SHOCK, SHOCK_I 1..3][nV] */
void ora_get_features(const ora_fluid *f, double *feat);
void ora_set_features(ora_fluid *f, const double *feat);

/* IncrementDivergence_FV % Compute on the current state: K += dU (6 fields). */
void ora_increment(ora_fluid *f, double *K, double dt, double weight_rk,
                   double *fluence);
/* Step_RK2_C_ASC % Compute: one RK2 step of size dt. fluence may be NULL. */
void ora_step(ora_fluid *f, double dt, double *fluence);
/* ora_step that also keeps the Sources records in src ([10][nV]). */
void ora_step_sources(ora_fluid *f, double dt, double *fluence, double *src);
/* Integrator_C_PS ComputeTimeStep: Courant * CFL dt, ramped by iCycle. */
double ora_timestep(const ora_fluid *f, int i_cycle);
/* Max inverse time step over proper cells (before Courant / ramp). */
double ora_inverse_timestep(const ora_fluid *f);

int ora_n_threads(void);

#ifdef __cplusplus
}
#endif
#endif

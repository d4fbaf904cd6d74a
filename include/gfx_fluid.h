/*
 * gfx_fluid.h -- C ABI of the B200 finite-volume step for the GenASiS
 * polytropic / ideal-gas fluid (Fluid_P_I): PLM reconstruction with the
 * generalized-minmod limiter, HLL / HLLC fluxes, flux divergence, RK2 stages,
 * conserved-to-primitive recovery, shock features and the CFL time step.
 *
 * Every entry point returns an int status (GFX_OK = 0, negative on error) and
 * never aborts; gfx_fluid_last_error() gives the message of the last failure
 * on the calling thread.  The Fortran side reaches these through
 * ISO_C_BINDING interfaces (include/gfx_fluid_f.f90).
 *
 * Data layout (the reference's StorageForm % Value(nValues, nVariables),
 * Storage_Form.f90:30): one contiguous FP64 array per variable, x fastest,
 * over the brick including n_ghost_layers (= 2) ghosts on every side,
 * nV = (nx+4)(ny+4)(nz+4) values per variable.
 *   conserved U : [D, S1, S2, S3, G, DS][nV]   (Fluid_D__Form.f90:650-654,
 *                                               Fluid_P__Template.f90:718-725)
 *   primitive   : [N, V1, V2, V3, E][nV]
 * Pointers named *_dev are device pointers; *_host are host pointers.
 * `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 */
#ifndef GFX_FLUID_H
#define GFX_FLUID_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GFX_FLUID_ABI_VERSION 2

enum gfx_status {
  GFX_OK = 0,
  GFX_ERR_ARGUMENT = -1,    /* bad pointer, size or configuration value */
  GFX_ERR_CUDA = -2,        /* a CUDA runtime call or kernel launch failed */
  GFX_ERR_UNSUPPORTED = -3, /* option the reference has but this library does not */
  GFX_ERR_STATE = -4,       /* non-finite or non-positive state detected */
  GFX_ERR_TIMEOUT = -5,     /* a bounded device-side wait expired */
  GFX_ERR_NO_MEMORY = -6    /* device or host allocation failed */
};

/* Atlas boundary conditions (Atlas_SC__Template.f90:244-324) */
enum { GFX_BC_OUTFLOW = 0, GFX_BC_REFLECTING = 1, GFX_BC_PERIODIC = 2 };
/* Fluid_ASC RiemannSolverType (Fluid_ASC__Form.f90:128-137) */
enum { GFX_RIEMANN_HLL = 0, GFX_RIEMANN_HLLC = 1 };
/* IncrementDivergence_FV ReconstructionType (IncrementDivergence_FV__Form.f90:
 * 239, 637-655): PLM with the limiter, or PARABOLIC (Kernel.f90:296-596) */
enum { GFX_RECONSTRUCTION_LINEAR = 0, GFX_RECONSTRUCTION_PARABOLIC = 1 };

/* Parameters of one single-brick chart + Fluid_P_I + Step_RK2 + Integrator.
 * Names follow the reference's GetParameter names; gfx_fluid_config_default
 * fills the reference defaults. */
typedef struct gfx_fluid_config {
  int    n_cells[3];            /* nCells (proper cells per axis) */
  int    n_ghost_layers;        /* nGhostLayers; must be 2 */
  double min_coordinate[3];     /* MinCoordinate (0) */
  double max_coordinate[3];     /* MaxCoordinate (1) */
  int    boundary[3][2];        /* BoundaryConditionsFace, [axis][inner, outer] */
  int    riemann_solver;        /* RiemannSolverType (HLLC) */
  int    use_limiter;           /* UseLimiter (1) */
  double limiter_parameter;     /* LimiterParameter (1.4) */
  double adiabatic_index;       /* AdiabaticIndex (1.4) */
  double shock_threshold;       /* ShockThreshold (0.1) */
  double courant_factor;        /* CourantFactor (0.7) */
  double baryon_density_min;    /* BaryonDensityMin (0) */
  double uniform_acceleration;  /* UniformAcceleration along z (0 = no gravity) */
  int    n_ramp_cycles;         /* nRampCycles (100) */
  int    reconstruction;        /* ReconstructionType (LINEAR); PARABOLIC for single
                                   bricks' step and increment (not batch, adjoint,
                                   no-allocation step) */
} gfx_fluid_config;

typedef struct gfx_fluid gfx_fluid;

/* Reference defaults (ChartHeader_SL__Form.f90:345-366, Fluid_ASC__Form.f90,
 * FluidFeatures_ASC__Form.f90:61-65, Integrator_C_PS__Form.f90:136,
 * IntegratorHeader_Form.f90:95). */
int gfx_fluid_config_default(gfx_fluid_config *cfg);

/* Creates the handle: device geometry tables, scratch and feature storage.
 * Replaces FluidBox / Step_RK2_C_ASC Initialize (FluidBox_Form.f90:37-241). */
int gfx_fluid_create(const gfx_fluid_config *cfg, gfx_fluid **out);
int gfx_fluid_destroy(gfx_fluid *h);

int gfx_fluid_n_values(const gfx_fluid *h, size_t *n_values);

/* Cell centres and left / right half widths of one axis over the ghost-
 * inclusive index range (n_cells[axis] + 4 values each; host pointers).
 * Chart_Template.f90:478-560, 827-841, 973-990. */
int gfx_fluid_geometry(const gfx_fluid *h, int axis, double *center_host,
                       double *width_left_host, double *width_right_host);

/* Fluid_P_I % ComputeFromPrimitive on every value after the periodic ghost
 * exchange of the primitives (Integrator_C_PS__Form.f90:194-203,
 * Fluid_P_I__Form.f90:509-601): prim_dev -> U_dev.  The primitives are kept
 * as the state of the next step, as the reference's Current keeps them. */
int gfx_fluid_from_primitive(gfx_fluid *h, const double *prim_dev, double *U_dev,
                             void *stream);

/* Fluid_P_I % ComputeFromConserved on every value (Fluid_P_I__Form.f90:604-722):
 * U_dev is floored in place (and its DS recomputed); prim_dev ([5][nV], may be
 * NULL) receives N, V1, V2, V3, E; aux_dev ([3][nV], may be NULL) receives the
 * pressure P, sound speed CS and entropy per baryon SB. */
int gfx_fluid_to_primitive(gfx_fluid *h, double *U_dev, double *prim_dev, double *aux_dev,
                           void *stream);

/* FluidFeatures_P % Detect (FluidFeatures_P__Form.f90:145-171) on the state
 * U_dev; the flags feed the HLLC flux of the following increments / steps.
 * gfx_fluid_clear_features zeroes them (the state after initialisation). */
int gfx_fluid_detect_features(gfx_fluid *h, const double *U_dev, void *stream);
int gfx_fluid_clear_features(gfx_fluid *h, void *stream);
/* DIFFUSIVE_FLUX_I flags of every value as bytes, bit d = direction d. */
int gfx_fluid_get_features(gfx_fluid *h, uint8_t *flags_dev, void *stream);

/* IncrementDivergence_FV % Compute (IncrementDivergence_FV__Form.f90:344-412):
 * K_dev ([6][nV]) += the divergence increment of the state U_dev over proper
 * cells, all six conserved fields; fluence_dev ([6 fields][6 faces][face_size],
 * may be NULL) += weight_rk * dt * F on the boundary faces
 * (RecordBoundaryFluence_CSL, :1002-1069). */
int gfx_fluid_increment(gfx_fluid *h, const double *U_dev, double *K_dev, double dt,
                        double weight_rk, double *fluence_dev, void *stream);
int gfx_fluid_fluence_face_size(const gfx_fluid *h, size_t *face_size);

/* Step_RK_C_ASC % Compute (Step_RK_C_ASC__Template.f90:504-542): one RK2 step
 * of size dt on U_dev in place, ending with ComputeFromConserved and feature
 * detection of the new state.  fluence_dev (may be NULL) is cleared and
 * receives the step's boundary fluence.  Ghost values are refreshed as the
 * reference leaves them (periodic images; floors on physical ghosts). */
int gfx_fluid_step(gfx_fluid *h, double *U_dev, double dt, double *fluence_dev,
                   void *stream);

/* gfx_fluid_step that also keeps the reference's Sources records of the step
 * in sources_dev ([GFX_N_SOURCES][nV], ghost layout, overwritten):
 *   fields 0-5  the divergence sources of D, S_1, S_2, S_3, G, DS: the sum over
 *               the stages of B_s K_s / dt, K_s the stage's divergence
 *               increment (ApplyDivergence_C and RecordDivergenceKernel,
 *               Step_RK_C_ASC__Template.f90:1548-1595,
 *               Step_RK_C_ASC__Kernel.f90:12-46); zero on ghosts;
 *   field 6     Gravitational_G, fields 7-9 Gravitational_S_D (1:3): the sum
 *               over the stages of -B_s N (V . g) and -B_s N g_d on proper
 *               cells (ApplyGravity_F__Command.f90:23-264), zero elsewhere and
 *               without gravity.
 * These are Sources_F's fields 1-6, N_CONSERVED + 1 and N_CONSERVED + 9..11
 * (Sources_F__Form.f90:157-167), in that order.  The state, fluence and
 * shock flags are bit for bit those of gfx_fluid_step; the divergence of
 * each stage is computed a second time for the records.  Allocates a
 * [6][nV] scratch on the first call. */
#define GFX_N_SOURCES 10
int gfx_fluid_step_sources(gfx_fluid *h, double *U_dev, double dt, double *fluence_dev,
                           double *sources_dev, void *stream);

/* The same step with U in host memory (pinned for speed): copies in, steps,
 * copies out, and returns after the result is back on the host.  The copies
 * and the compute overlap over z slabs (bit-identical to gfx_fluid_step); the
 * DS field of U_host is not read. */
int gfx_fluid_step_host(gfx_fluid *h, double *U_host, double dt, double *fluence_host);

/* Integrator ComputeTimeStep (Integrator_Template.f90:896-939) on U_dev:
 * CourantFactor / max inverse CFL time (Integrator_C_PS__Kernel.f90:97-142),
 * ramped by min((i_cycle + 1) / nRampCycles, 1).  Synchronises the stream. */
int gfx_fluid_timestep(gfx_fluid *h, const double *U_dev, int i_cycle, double *dt_host,
                       void *stream);

/* Integrator % Evolve loop on the device (Integrator_Template.f90:291-346):
 * from (time, i_cycle) advance U_dev until finish_time (the last step is cut
 * to land on it, as CheckpointTimeExact does) or until n_cycles_max cycles,
 * each cycle = time step + RK2 step.  Uses a CUDA graph per cycle; returns
 * after the work completes with the final time and cycle count. */
int gfx_fluid_evolve(gfx_fluid *h, double *U_dev, double time, int i_cycle,
                     double finish_time, int n_cycles_max, double *time_out,
                     int *i_cycle_out, void *stream);

/* gfx_fluid_evolve that also gives the device milliseconds of its work in
 * ms_out: CUDA events recorded on the stream just before its first device
 * operation and just after its last (the reference's Evolve timer,
 * Integrator_Template.f90:291-346, on the device).  The call returns after
 * the work completes, like gfx_fluid_evolve, but a host delay before its
 * first launch or before the return stays out of ms_out; the results are
 * those of gfx_fluid_evolve bit for bit. */
int gfx_fluid_evolve_timed(gfx_fluid *h, double *U_dev, double time, int i_cycle,
                           double finish_time, int n_cycles_max, double *time_out,
                           int *i_cycle_out, double *ms_out, void *stream);

/* gfx_fluid_step with a CUDA event recorded around each launch (the
 * reference's per-phase timers, StorageDivergence_Form.f90:45-74): ms_out[4]
 * receives the device milliseconds of features, stage 1, stage 2 and the
 * ghost refresh.  Synchronises the stream.  It times the kernels of an
 * evolve cycle: when U_dev is the state that the last step, timed step or
 * evolve on this handle produced, features and stage 1 start from the
 * primitives that step's stage 2 stored, so U_dev must not have been changed
 * since by other means. */
int gfx_fluid_step_timed(gfx_fluid *h, double *U_dev, double dt, double *fluence_dev,
                         double *ms_out, void *stream);

/* Number of kernels this handle has launched (graph replays included). */
int gfx_fluid_kernel_launches(const gfx_fluid *h, long long *count);

/* ---- Batched bricks -------------------------------------------------------
 * Many independent bricks (each its own handle, state U and CFL time step)
 * advanced together: one persistent launch per RK stage covers every brick's
 * work, the whole cycle is one CUDA graph.  The handles must share the
 * Riemann solver, gravity and the fluid / limiter / Courant parameters; the
 * batch borrows them (destroy the batch first).  Each brick keeps its own
 * clock (time, cycle); gfx_fluid_batch_evolve advances every brick until its
 * finish_time (last step cut to land on it) or n_cycles more cycles.  The
 * reference runs such bricks as separate programs or ranks; this has no
 * single counterpart in it (Integrator_Template.f90:291-346 per brick). */
typedef struct gfx_fluid_batch gfx_fluid_batch;
int gfx_fluid_batch_create(int n_bricks, gfx_fluid *const *handles, double *const *U_dev,
                           gfx_fluid_batch **out);
int gfx_fluid_batch_destroy(gfx_fluid_batch *b);
int gfx_fluid_batch_set_clocks(gfx_fluid_batch *b, double time, int i_cycle);
int gfx_fluid_batch_evolve(gfx_fluid_batch *b, double finish_time, int n_cycles, void *stream);
/* time_host[n], cycle_host[n] (either may be NULL); synchronises the stream. */
int gfx_fluid_batch_clocks(gfx_fluid_batch *b, double *time_host, int *cycle_host,
                           void *stream);
int gfx_fluid_batch_kernel_launches(const gfx_fluid_batch *b, long long *count);

/* ---- A chart of several bricks --------------------------------------------
 * Chart_SLD (Chart_SLD__Form.f90, Chart_Template.f90:440-460): one domain
 * (cfg: the whole chart, n_cells its cells per axis) split into n_bricks[0] x
 * n_bricks[1] x n_bricks[2] equal bricks of n_cells / n_bricks cells (which
 * must divide evenly, at least 4 per axis), brick b = ix + nx (iy + ny iz).
 * The reference runs one brick per MPI rank and exchanges the ghost layers of
 * faces and edges between them each stage (ExchangeGhostData,
 * Chart_SLD__Form.f90:131-201, from Step_RK_C_ASC__Template.f90:1237-1246);
 * here all bricks share one device, and a stage reads a neighbour's cells
 * where they live.  Each brick's geometry is the slice of the chart's
 * (SetGeometryWidthCenter, Chart_SLD__Form.f90:273-320); the shock features
 * see across brick faces and ClearBoundary applies on the chart's boundary
 * only (FluidFeatures_P__Form.f90:313-336); the boundary fluence is recorded
 * on the chart's boundary faces only (IncrementDivergence_FV__Form.f90:
 * 1002-1069); the time step is the minimum over the chart (the MIN all-reduce
 * of Integrator_Template.f90:919).  The results on every cell are those of
 * one brick of the whole chart, bit for bit.  LINEAR reconstruction.
 *
 * gfx_fluid_chart_brick gives a brick's handle (for gfx_fluid_n_values,
 * gfx_fluid_geometry, gfx_fluid_fluence_face_size, gfx_fluid_totals,
 * gfx_fluid_get_features (the flags the chart last detected),
 * gfx_fluid_check_state; the step entry points of a single brick refuse it)
 * and its brick coordinates.  gfx_fluid_chart_bind gives the bricks' states
 * ([6][nV] each, caller-owned device arrays); the other calls act on them. */
typedef struct gfx_fluid_chart gfx_fluid_chart;
int gfx_fluid_chart_create(const gfx_fluid_config *cfg, const int n_bricks[3],
                           gfx_fluid_chart **out);
int gfx_fluid_chart_destroy(gfx_fluid_chart *c);
int gfx_fluid_chart_n_bricks(const gfx_fluid_chart *c, int *n);
int gfx_fluid_chart_brick(gfx_fluid_chart *c, int brick, gfx_fluid **handle,
                          int brick_index[3]);
int gfx_fluid_chart_bind(gfx_fluid_chart *c, double *const *U_dev);
/* ComputeFromPrimitive of every brick from prim_dev[b] ([5][nV] of brick b,
 * ghosts included); a ghost that the exchange reaches takes the primitives of
 * the cell it images (Integrator_C_PS__Form.f90:194-203). */
int gfx_fluid_chart_from_primitive(gfx_fluid_chart *c, const double *const *prim_dev,
                                   void *stream);
/* ComputeFromConserved on every value of every brick (floors, DS), then
 * FluidFeatures_P % Detect over the chart: the state set from conserved
 * values, as gfx_fluid_to_primitive and gfx_fluid_detect_features leave a
 * brick. */
int gfx_fluid_chart_set_conserved(gfx_fluid_chart *c, void *stream);
int gfx_fluid_chart_timestep(gfx_fluid_chart *c, int i_cycle, double *dt_host, void *stream);
/* One RK2 step of every brick; fluence_dev (may be NULL) holds one array per
 * brick ([6][6][face_size of the brick]), cleared and filled on the chart's
 * boundary faces. */
int gfx_fluid_chart_step(gfx_fluid_chart *c, double dt, double *const *fluence_dev,
                         void *stream);
int gfx_fluid_chart_evolve(gfx_fluid_chart *c, double time, int i_cycle, double finish_time,
                           int n_cycles_max, double *time_out, int *i_cycle_out, void *stream);
int gfx_fluid_chart_kernel_launches(const gfx_fluid_chart *c, long long *count);

/* ---- Discrete adjoint of one step -----------------------------------------
 * No counterpart in the reference (which has no adjoint); it is the reverse
 * mode of gfx_fluid_step, with dt held fixed.  Given lam_np1_dev ([6][nV],
 * the gradient of an objective with respect to the conserved state after the
 * step), writes lam_n_dev ([6][nV]): the gradient with respect to the
 * conserved state U_n_dev before the step, on proper cells (ghost values and
 * the dead DS field get 0; a periodic ghost's share goes to its image cell).
 * The stages are recomputed from the checkpoint U_n_dev; U_np1_dev (may be
 * NULL, then recomputed too) is the state after the step, as gfx_fluid_step
 * produced it.  detect_features: 1 if the forward step detected the shock
 * features of U_n (every step after the first), 0 if it ran on zero features
 * (the first step after initialisation).  The derivative is that of the
 * branch the forward step takes at every limiter, wave-speed maximum, HLLC
 * side and floor.  Cells shared by two threads' segments receive atomic
 * additions in no fixed order, so repeated calls agree to rounding, not bit
 * for bit.  Allocates a workspace of 20 values per proper cell on the first
 * call.  lam_n_dev must not alias lam_np1_dev. */
int gfx_fluid_step_adjoint(gfx_fluid *h, const double *U_n_dev, double dt,
                           const double *lam_np1_dev, double *lam_n_dev,
                           const double *U_np1_dev, int detect_features, void *stream);

/* The branches one step from U_n_dev takes, for finite-difference checks of
 * the adjoint: no counterpart in the reference.  The adjoint is the
 * derivative of the branch the forward takes at every limiter argument,
 * wave-speed maximum, HLLC decision and floor; a central difference measures
 * it only where the forwards at U + eps d and U - eps d take the same
 * branches.  Recomputes the step's two stages from U_n_dev (features detected
 * from it when detect_features is nonzero, as in gfx_fluid_step_adjoint) and
 * writes out_host[0] = an order-independent hash of every decision of both
 * stages (limiter branch of each slope, the two wave-speed maxima, the HLLC
 * path, side and centre-speed sign of each face, floored inputs, shock
 * flags), out_host[1] = the number of decisions and out_host[2 ..
 * 2 + GFX_BRANCH_KINDS - 1] = counts per kind: limiter zero / left / right /
 * centred slope, AP arg 0 / 1 / 2, AM arg 0 / 1 / 2, HLLC centre state, AC >=
 * 0, MD > 0, floored inputs, flags set.  Synchronises the stream. */
#define GFX_BRANCH_KINDS 15
int gfx_fluid_step_branches(gfx_fluid *h, const double *U_n_dev, double dt,
                            int detect_features, unsigned long long *out_host, void *stream);

/* ---- One step without allocation ------------------------------------------
 * No counterpart in the reference (which allocates its storage once per
 * run); added for callers that cannot call cudaMalloc: a host program whose
 * memory manager has claimed the device memory up front into its own pool, or
 * a code path that cannot afford the device-wide synchronisation that
 * cudaMalloc and cudaFree imply.
 *
 * gfx_fluid_step_noalloc is gfx_fluid_step without a handle, on a state U_dev
 * set from conserved values: the same kernels and results, features detected
 * from U_dev first when detect_features is nonzero (every step after the
 * first), zero features otherwise (the first step after initialisation).
 * It allocates nothing: its tables and stage buffers live in one fixed
 * array of GFX_FLUID_NOALLOC_SCRATCH_BYTES of device memory inside the
 * library, which every GPU that loads the library holds until exit.  That
 * bounds the brick at about 81 bytes per proper cell plus the chart tables
 * (37^3 proper cells fit, 38^3 do not); larger bricks get GFX_ERR_ARGUMENT.
 * Every call looks up the array's device address on the current device (the
 * first call on a device also loads the library's kernels there and sets up
 * the stage kernels' launch attributes for that device, if no step ran on it
 * before); make that first call before any stream capture.  Each device that
 * calls it has its own copy of the array.  Every call uses the same array: each
 * call rewrites what it reads and zeroes its CFL word and work counters, so
 * calls in sequence are independent, but calls that overlap on the GPU (on
 * different streams or threads) race on the array and give wrong results. */
#define GFX_FLUID_NOALLOC_SCRATCH_BYTES (4u << 20)
int gfx_fluid_step_noalloc(const gfx_fluid_config *cfg, double *U_dev, double dt,
                           int detect_features, double *fluence_dev, void *stream);

/* Scans the proper cells of U_dev: GFX_ERR_STATE (with the counts in the
 * error message) if any holds a non-finite value; the number of cells at the
 * density floor is reported alongside.  The reference checks nothing here
 * (its floors in Fluid_P__Kernel.f90:94-192 are silent).  Synchronises the
 * stream. */
int gfx_fluid_check_state(gfx_fluid *h, const double *U_dev, void *stream);

/* Restart (Integrator_Template.f90:476-502, 658-764): U_dev holds a state
 * written by a step of this library (a checkpoint read back); the next step
 * or evolve continues from it as an uninterrupted run would, detecting the
 * shock features of U_dev first.  No device work. */
int gfx_fluid_resume(gfx_fluid *h, double *U_dev);

/* Volume integrals of the six conserved fields of U_dev over the proper
 * cells, sum U dV (the conservation tallies of Current_ASC__Template.f90:
 * 203-349 and VolumeIntegral_Form.f90:25-117, on the device): totals_host[6].
 * Partial sums are added in a fixed order, so repeated calls agree bit for
 * bit.  Synchronises the stream. */
int gfx_fluid_totals(gfx_fluid *h, const double *U_dev, double *totals_host, void *stream);

/* Speed knobs (set by genasis_b200/autotune.py).  The step's results do not
 * depend on them, bit for bit; the adjoint's change only by the rounding of
 * its atomic additions, whose order is not fixed in any case:
 * z_chunk = z length of the cell pencils a CTA marches in the stage kernel
 * (0 = default: enough items for 16 per SM; a batch created afterwards takes
 * it per brick, default 32); adjoint_segment = faces per thread in the
 * adjoint's reverse sweep (0 = 8); tile_rows = rows of the 32-wide tile of a
 * CTA, 8 (256 threads, 2 CTAs per SM) or 16 (512 threads, 1 CTA per SM; 0 =
 * 16; PARABOLIC runs on 16 only; the bricks of a batch must agree).  No
 * counterpart in the reference. */
int gfx_fluid_set_tuning(gfx_fluid *h, int z_chunk, int adjoint_segment, int tile_rows);

int gfx_fluid_last_error(char *buf, size_t len);

/* Fault injection for tests, on the host: the nth device allocation that the
 * library makes on the calling thread from now on (0 = the next one) fails as
 * if the device were out of memory, once; a negative nth turns it off.  The
 * call that meets it returns GFX_ERR_NO_MEMORY, frees what it had allocated
 * (a create) or keeps the buffers it had (a handle's lazily allocated
 * workspaces), and the next call allocates again.  The reference aborts on
 * an allocation failure and has no counterpart. */
int gfx_fluid_debug_fail_allocation(int nth);

#ifdef __cplusplus
}
#endif
#endif

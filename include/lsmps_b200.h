/*
 * lsmps_b200.h - C ABI of the B200-native LSMPS per-step particle hot path.
 *
 * Every entry point below replaces one function or method of the lsmps3D C++
 * module API (paths are relative to the lsmps-3D project root).  The POD view
 * structs are layout-identical to the reference's views when the reference is
 * built with LSMPS3D_USE_DOUBLE (real = double, index_t = int32_t,
 * size_type = size_t), so a reference view can be passed by address.
 *
 * Memory: every device pointer in a view is owned by the caller.  The opaque
 * context owns only scratch (radix-sort ping-pong buffers, scan partials, the
 * device status word) and the CUDA stream the work is queued on.
 *
 * Errors: no entry point exits the process.  Each returns an lsmps_status; a
 * human-readable message for the last failure is available from
 * lsmps_ctx_last_error().  In synchronous mode (the default) each call waits
 * for its kernels and folds the device-side status (CSR capacity overflow,
 * non-SPD moment matrices, non-finite coordinates) into the return value.
 */
#ifndef LSMPS_B200_H
#define LSMPS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------- */
/* Status codes                                                              */
/* ------------------------------------------------------------------------- */
typedef enum lsmps_status {
  LSMPS_OK = 0,
  /* CSR (or PPE) capacity smaller than required; lsmps_ctx_required() gives
   * the required entry count.  Reference: std::exit in
   * src/neighbor/neighbor_search.cu:22-30. */
  LSMPS_CAPACITY_EXCEEDED = 1,
  /* Invalid grid, null buffer, size mismatch, radius > cell size, ...
   * Reference: std::exit in neighbor_search.cu:257-273, 354-361 and the
   * validate_* helpers of every module. */
  LSMPS_INVALID_ARGUMENT = 2,
  /* A consumer was given a moment view that was never prepared.
   * Reference: moment_matrix.cu:571-576. */
  LSMPS_NOT_PREPARED = 3,
  /* At least one moment matrix failed the Cholesky factorisation (its info
   * entry is > 0).  The reference never checks potrf info
   * (moment_matrix.cu:438-439); this status is informational and only
   * returned when the context asks for strict SPD checking. */
  LSMPS_NON_SPD = 4,
  LSMPS_CUDA_ERROR = 5,
  /* A count exceeds the 32-bit index range (reference: neighbor_search.cu:270). */
  LSMPS_INDEX_OVERFLOW = 6,
  /* A particle coordinate is NaN or infinite. */
  LSMPS_NON_FINITE = 7
} lsmps_status;

typedef enum lsmps_precision {
  /* Every floating operation in double, the reference's real type. */
  LSMPS_PRECISION_PLAIN = 0,
  /* FP32 neighbour geometry and compensated FP32 moment assembly with FP64
   * refinement; FP64 kept for ill-conditioned matrices and the PPE RHS. */
  LSMPS_PRECISION_MIXED = 1
} lsmps_precision;

/* Surface labels: include/lsmps3d/surface/surface_type.cuh:5-10. */
enum {
  LSMPS_SURFACE_INNER = 0,
  LSMPS_SURFACE_NEAR_SURFACE = 1,
  LSMPS_SURFACE_SURFACE = 2,
  LSMPS_SURFACE_SPLASH = 3
};

/* Moment matrix kinds: include/lsmps3d/moment_matrix/moment_matrix.cuh:39-44. */
typedef enum lsmps_moment_kind {
  LSMPS_MOMENT_VELOCITY_WALL_DIRICHLET_A = 0,
  LSMPS_MOMENT_PRESSURE_WALL_NEUMANN_A = 1,
  LSMPS_MOMENT_PRESSURE_WALL_NEUMANN_B = 2,
  LSMPS_MOMENT_FLUID_ONLY_A = 3
} lsmps_moment_kind;

/* ------------------------------------------------------------------------- */
/* Views (caller-owned device memory)                                        */
/* ------------------------------------------------------------------------- */

/* lsmps3d::FluidParticleSoA, include/lsmps3d/particle/particle_data.cuh:7-17. */
typedef struct lsmps_fluid {
  size_t count;
  double* x;
  double* y;
  double* z;
  double* vx;
  double* vy;
  double* vz;
  double* pressure;
  int32_t* surface_type;
} lsmps_fluid;

/* lsmps3d::WallParticleSoA, particle_data.cuh:19-30. */
typedef struct lsmps_walls {
  size_t count;
  double* x;
  double* y;
  double* z;
  double* vx;
  double* vy;
  double* vz;
  double* normal_x;
  double* normal_y;
  double* normal_z;
} lsmps_walls;

/* lsmps3d::CellGrid, include/lsmps3d/neighbor/cell_list.cuh:7-15. */
typedef struct lsmps_grid {
  double origin[3];
  double cell_size;
  int32_t dims[3];
} lsmps_grid;

/* lsmps3d::CellListView, cell_list.cuh:17-24.  particle_count and
 * cell_count are capacities; cell_ids holds the SORTED cell id of each sorted
 * position, sorted_indices the particle index at that position, and
 * cell_begin/cell_end the [first, last+1) sorted range of each cell or -1. */
typedef struct lsmps_cells {
  size_t particle_count;
  size_t cell_count;
  int32_t* cell_ids;
  int32_t* sorted_indices;
  int32_t* cell_begin;
  int32_t* cell_end;
} lsmps_cells;

/* lsmps3d::NeighborListView, include/lsmps3d/particle/neighbor_list.cuh:7-12.
 * neighbor_count is the capacity of indices. */
typedef struct lsmps_csr {
  size_t particle_count;
  size_t neighbor_count;
  int32_t* offsets;
  int32_t* indices;
} lsmps_csr;

/* lsmps3d::ProvisionVelocityView (include/lsmps3d/provision/explicit_update.cuh:11-16)
 * and lsmps3d::CorrectionVectorView
 * (include/lsmps3d/correction/pressure_correction.cuh:11-16) share this layout. */
typedef struct lsmps_vector {
  size_t count;
  double* x;
  double* y;
  double* z;
} lsmps_vector;

/* lsmps3d::SurfaceDetectionDiagnosticsView,
 * include/lsmps3d/surface/surface_detection.cuh:10-21.  Any pointer may be NULL. */
typedef struct lsmps_surface_diagnostics {
  int32_t* fluid_neighbor_count;
  int32_t* wall_neighbor_count;
  double* number_density;
  double* number_density_ratio;
  double* anisotropy;
  double* air_open_ratio;
  double* air_anisotropy;
  double* surface_normal_x;
  double* surface_normal_y;
  double* surface_normal_z;
} lsmps_surface_diagnostics;

/* Output buffers and metadata of one moment-matrix kind: the device side of
 * lsmps3d::MomentMatrixView (moment_matrix.cuh:46-60).  inverse_matrices holds
 * particle_count blocks of matrix_size^2 doubles, column-major
 * ([row + col * n]), full symmetric storage.  moment_trace is the trace
 * before regularisation, regularization_added the lambda*tr/n added to the
 * diagonal, info the Cholesky status (0 = SPD, k = leading minor k failed).
 * inversion_count is a single device int incremented once per build. */
typedef struct lsmps_moment {
  size_t particle_count;
  int32_t matrix_size;
  int32_t kind;
  double support_radius;
  double wall_weight_scale;
  double* inverse_matrices;
  double* moment_trace;
  double* regularization_added;
  int32_t* info;
  int32_t* inversion_count;
} lsmps_moment;

/* lsmps3d::CsrMatrixView, include/lsmps3d/ppe/ppe_matrix.cuh:15-22. */
typedef struct lsmps_csr_matrix {
  size_t rows;
  size_t cols;
  size_t nnz;
  int32_t* row_offsets;
  int32_t* col_indices;
  double* values;
} lsmps_csr_matrix;

/* lsmps3d::PpeWorkspaceView, ppe_matrix.cuh:24-30. */
typedef struct lsmps_ppe {
  lsmps_csr_matrix matrix;
  double* rhs;
  double* pressure;
  double* divergence;
  double* pressure_laplacian;
} lsmps_ppe;

/* The scalar fields of lsmps3d::SimulationConfig (include/lsmps3d/core/config.hpp:12-82)
 * that hot-path kernels read.  File paths, the INI layer and the time-step
 * controller fields stay on the host side of the reference and are omitted. */
typedef struct lsmps_params {
  double particle_spacing;
  double support_radius;
  double near_surface_radius;
  lsmps_grid grid;
  double time_step;
  double density;
  double kinematic_viscosity;
  double gravity[3];
  int32_t splash_neighbor_threshold;
  int32_t include_wall_neighbors;
  double number_density_ratio_threshold;
  double air_open_ratio_threshold;
  double air_anisotropy_threshold;
  double wall_normal_independence_threshold;
  double virtual_light_cone_cosine;
  double lsmps_regularization;
  double lsmps_wall_weight_scale;
  double ps_displacement_scale;
  double ps_min_distance_ratio;
  double ps_max_displacement_ratio;
  double wall_clearance_ratio;
  double velocity_smoothing_strength;
} lsmps_params;

/* Every buffer one time step touches.  The step runs, in the reference
 * driver's order (src/app/simulation_driver.cu:346-383):
 *   provision -> PPE assembly -> pressure correction -> neighbour rebuild ->
 *   surface classification,
 * where the pressure handed to the correction is `pressure` (the PPE solve
 * is outside this path). */
typedef struct lsmps_step_state {
  lsmps_fluid fluid;
  lsmps_walls walls;
  lsmps_cells fluid_cells;
  lsmps_cells wall_cells;
  lsmps_csr fluid_neighbors;
  lsmps_csr wall_neighbors;
  lsmps_fluid temporary_velocity;
  lsmps_walls temporary_wall_velocity;
  lsmps_vector velocity_laplacian;
  lsmps_moment velocity_moment;
  lsmps_moment pressure_moment;
  lsmps_ppe ppe;
  lsmps_vector pressure_gradient;
  lsmps_vector ps_displacement;
  lsmps_vector smoothed_velocity;
  double* pressure;
} lsmps_step_state;

typedef struct lsmps_ctx lsmps_ctx;

/* ------------------------------------------------------------------------- */
/* Context                                                                   */
/* ------------------------------------------------------------------------- */
lsmps_status lsmps_ctx_create(int device, lsmps_ctx** out);
void lsmps_ctx_destroy(lsmps_ctx* ctx);
/* Queue all further work of this context on `stream` (a cudaStream_t; NULL =
 * the legacy default stream).  A new context starts on its own non-blocking
 * stream. */
lsmps_status lsmps_ctx_set_stream(lsmps_ctx* ctx, void* stream);
void* lsmps_ctx_stream(lsmps_ctx* ctx);
lsmps_status lsmps_ctx_set_precision(lsmps_ctx* ctx, int precision);
/* 1 (default): every call waits for its kernels and returns the device status.
 * 0: calls only queue work; lsmps_ctx_synchronize() returns the folded status. */
lsmps_status lsmps_ctx_set_synchronous(lsmps_ctx* ctx, int synchronous);
/* Pre-size scratch so that no call of this size allocates (needed before
 * graph capture). */
lsmps_status lsmps_ctx_reserve(lsmps_ctx* ctx, size_t fluid_capacity, size_t wall_capacity,
                               size_t cell_capacity);
lsmps_status lsmps_ctx_synchronize(lsmps_ctx* ctx);
/* Required entry count recorded by the last LSMPS_CAPACITY_EXCEEDED. */
uint64_t lsmps_ctx_required(lsmps_ctx* ctx);
/* Number of kernel launches this context has queued since creation. */
uint64_t lsmps_ctx_launch_count(lsmps_ctx* ctx);
/* Mixed form (no counterpart in the reference, which has one precision):
 * moment matrices whose FP32 Cholesky factor failed or whose condition
 * estimate (max L_ii / min L_ii)^2 exceeded the threshold are factorised in
 * FP64 instead.  The threshold defaults to 1e4 (one FP64 refinement of an
 * FP32 factor leaves a relative error of about (kappa 2^-24)^2: ~4e-7 at 1e4,
 * ~4e-3 at 1e6); the count accumulates over the context's life (read back at
 * each status fold). */
lsmps_status lsmps_ctx_set_condition_threshold(lsmps_ctx* ctx, double threshold);
/* lsmps_step's gather kernels visit the fluid in the order of the state's
 * fluid cell list (particles of one cell on adjacent threads, sharing their
 * neighbours' records in cache) when this context built that list last
 * (1, the default), or in index order (0).  Results are identical either way. */
lsmps_status lsmps_ctx_set_cell_order(lsmps_ctx* ctx, int on);
/* Cell-sorted rows (1, the default): this context's builds of the fluid table
 * also write, beside every entry's neighbour index, the neighbour's position in
 * the fluid cell list (context memory, 4 bytes per entry of the table's
 * capacity), and while lsmps_step visits the fluid in cell order its gather
 * kernels read those rows and neighbour records packed in cell order, so the
 * records of a home cell's neighbours lie in a few contiguous runs whatever
 * the caller's particle numbering.  The tables, and every result, are the
 * same either way; 0 reads the rows' indices and records in index order.  The
 * kept rows describe the table as this context built it: a caller that edits
 * the fluid table's indices before the next step sets 0. */
lsmps_status lsmps_ctx_set_sorted_rows(lsmps_ctx* ctx, int on);
/* Copy the first `count` entries of the cell-sorted rows this context holds
 * (of its last build of the fluid table) to device memory `dst`, on the
 * context's stream; LSMPS_NOT_PREPARED when none are held. */
lsmps_status lsmps_ctx_copy_sorted_rows(lsmps_ctx* ctx, int32_t* dst, size_t count);
uint64_t lsmps_ctx_fp64_fallbacks(lsmps_ctx* ctx);
/* Launch-shape knobs (no counterpart in the reference, whose kernels all use
 * one thread per particle in 128-thread blocks).  Values are indices into each
 * knob's variant list; lsmps_autotune() picks them by timing. */
typedef enum lsmps_knob {
  /* plain-form moment kernel: 0 = compiler's register choice, 1 = capped for
   * 8 blocks per SM (default), 2 = the two kinds on two warps sharing each
   * row */
  LSMPS_KNOB_MOMENT_OCCUPANCY = 0,
  /* lanes cooperating on one PPE row: 0 -> 1, 1 -> 4 (default), 2 -> 8,
   * 3 -> 16 */
  LSMPS_KNOB_PPE_LANES = 1,
  /* lanes cooperating on one particle in the velocity-Laplacian, pressure
   * gradient/shifting and smoothing passes: 0 -> 1, 1 -> 2, 2 -> 4 (default) */
  LSMPS_KNOB_GATHER_LANES = 2,
  LSMPS_KNOB_COUNT = 3
} lsmps_knob;
lsmps_status lsmps_ctx_set_knob(lsmps_ctx* ctx, int knob, int value);
int lsmps_ctx_knob(lsmps_ctx* ctx, int knob);
/* Number of variants of a knob (0 for an unknown knob). */
int lsmps_knob_variants(int knob);
/* Project autotuner (no counterpart in the reference): times every variant of
 * every knob on the caller's state with CUDA events (`repeats` timed launches
 * after one untimed launch each) and leaves the fastest set on the context.
 * Only stages that are pure functions of the state are run (the moment stage
 * and the PPE assembly), so the simulation does not advance; the state's
 * temporary velocity should hold u* (it does after any lsmps_step).  If
 * best_ms is not NULL it receives LSMPS_KNOB_COUNT mean times (ms) of the
 * chosen variants.  Synchronous. */
lsmps_status lsmps_autotune(lsmps_ctx* ctx, const lsmps_params* params, const lsmps_step_state* state,
                            int repeats, double* best_ms);
/* Per-kernel device timing (no counterpart in the reference, which has no
 * tracing): while on, every launch is bracketed by CUDA events.  Turning it
 * on clears the records. */
lsmps_status lsmps_ctx_set_profiling(lsmps_ctx* ctx, int on);
/* Waits for the stream, aggregates the records by kernel name in order of
 * first launch, writes the names '\n'-separated into `names`, the summed
 * milliseconds and launch counts into the arrays, clears the records and
 * returns the number of entries (-1 on error). */
int lsmps_ctx_profile_report(lsmps_ctx* ctx, char* names, size_t names_len, double* total_ms,
                             uint64_t* launches, int max_entries);
const char* lsmps_ctx_last_error(lsmps_ctx* ctx);
const char* lsmps_status_string(int status);
/* SimulationConfig defaults (include/lsmps3d/core/config.hpp:12-60). */
void lsmps_params_default(lsmps_params* out);

/* ------------------------------------------------------------------------- */
/* Neighbour search: include/lsmps3d/neighbor/neighbor_search.cuh            */
/* ------------------------------------------------------------------------- */
/* build_cell_list(FluidParticleSoA|WallParticleSoA, CellGrid, CellListView),
 * neighbor_search.cuh:10-16.  Stable: particles of one cell keep ascending
 * index order, as Thrust's stable radix sort_by_key does in the reference. */
lsmps_status lsmps_build_cell_list(lsmps_ctx* ctx, const double* x, const double* y,
                                   const double* z, size_t count, const lsmps_grid* grid,
                                   const lsmps_cells* cells);

/* The same cell list, bit-identical to lsmps_build_cell_list's, from a call
 * that allocates no memory and needs no context.  No counterpart in the
 * reference, whose build_cell_list sorts through Thrust's allocator.
 *
 * For callers that must not allocate device memory while they run: a process
 * whose device memory is all handed out by its own pool allocator, or a loop
 * that must not meet the device-wide synchronisation of cudaFree.  The
 * context entry point grows its scratch with cudaMalloc on demand; this one
 * sorts in a fixed scratch array compiled into the library (about 4.1 MiB of
 * device memory per device, loaded with the library's device code).
 *
 * - count above LSMPS_NOALLOC_MAX_PARTICLES returns LSMPS_CAPACITY_EXCEEDED
 *   before any device work; other argument errors return
 *   LSMPS_INVALID_ARGUMENT (LSMPS_INDEX_OVERFLOW for more than 2^31-1 cells).
 * - Runs on the calling thread's current device, on `stream` (a
 *   cudaStream_t; NULL is the legacy default stream), and waits for it before
 *   returning.  A NaN or infinite coordinate returns LSMPS_NON_FINITE.
 * - The first call on a device does its set-up: it looks up the scratch
 *   array's device address and loads the device code of the sort kernels on
 *   that device (the CUDA runtime loads code lazily by default, and loading
 *   can allocate), so later calls load nothing.  Make that first call (any
 *   count, 0 included) before capturing any stream.
 * - An error already pending on the calling thread (from earlier CUDA work)
 *   is reported as LSMPS_CUDA_ERROR without being cleared and without any
 *   device work queued.
 * - Nothing has to be zeroed beforehand: each call clears its own status
 *   word and writes every scratch entry before reading it.
 * - There is one scratch array per device, so two calls in flight at once on
 *   one device would race on it.  Calls are therefore serialised per device
 *   by a lock held until the call's kernels finish: a second host thread
 *   calling on the same device waits.  (Each process has its own array.) */
#define LSMPS_NOALLOC_MAX_PARTICLES 524288
lsmps_status lsmps_build_cell_list_noalloc(void* stream, const double* x, const double* y, const double* z,
                                           size_t count, const lsmps_grid* grid, const lsmps_cells* cells);

/* Renumbers the fluid particles in the order of fluid_cells (cell id
 * ascending, stable), as last built for the current positions (by
 * lsmps_build_neighbor_lists or lsmps_step): x, y, z, vx, vy, vz, pressure
 * and surface_type are permuted in place and, when permutation is not NULL,
 * permutation[k] receives the previous index of the particle now at k (a
 * device array of fluid->count).  No counterpart in the reference; it keeps
 * the gathers of later steps local when the input numbering does not follow
 * space.  Afterwards the neighbour lists (and anything else the caller keeps
 * per fluid particle) are stale: rebuild them with lsmps_build_neighbor_lists
 * before the next step.  The rebuilt rows list the same neighbours in the same
 * order, so the next step's results are the renumbered results of the step
 * without renumbering, bit for bit. */
lsmps_status lsmps_reorder_fluid(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_cells* fluid_cells,
                                 int32_t* permutation);

/* build_neighbor_lists(...), neighbor_search.cuh:18-24.  Rows follow the
 * reference traversal order (27 cells dz -> dy -> dx, ascending sorted
 * position inside each cell); fluid rows exclude the particle itself. */
lsmps_status lsmps_build_neighbor_lists(lsmps_ctx* ctx, const lsmps_fluid* fluid,
                                        const lsmps_walls* walls, const lsmps_params* params,
                                        const lsmps_cells* fluid_cells,
                                        const lsmps_cells* wall_cells,
                                        const lsmps_csr* fluid_neighbors,
                                        const lsmps_csr* wall_neighbors);

/* ------------------------------------------------------------------------- */
/* Surface detection: include/lsmps3d/surface/surface_detection.cuh          */
/* ------------------------------------------------------------------------- */
/* compute_uniform_reference_number_density(real, real), surface_detection.cuh:28
 * (host loop, surface_detection.cu:494-520).  Returns a negative value on
 * invalid input. */
double lsmps_reference_number_density(double particle_spacing, double support_radius);

/* classify_surface_particles(...), surface_detection.cuh:31-36.
 * diagnostics may be NULL. */
lsmps_status lsmps_classify_surface(lsmps_ctx* ctx, const lsmps_fluid* fluid,
                                    const lsmps_walls* walls, const lsmps_csr* fluid_neighbors,
                                    const lsmps_csr* wall_neighbors, const lsmps_params* params,
                                    const lsmps_surface_diagnostics* diagnostics);

/* compute_virtual_light_diagnostics(...), surface_detection.cuh:38-43
 * (src/surface/surface_detection.cu:350-475, 555-578).  For each fluid
 * particle, how many of the reference's 14 fixed light directions (the six
 * axes and eight diagonals in the coordinate planes) stay open: a direction
 * is blocked when a fluid neighbour (and, with include_wall_neighbors, a wall
 * neighbour) within the support radius lies inside the cone of
 * virtual_light_cone_cosine around it.  open_direction_count[i] gets the
 * count, open_fraction[i] the count / 14; either may be NULL, not both. */
lsmps_status lsmps_virtual_light(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_walls* walls,
                                 const lsmps_csr* fluid_neighbors, const lsmps_csr* wall_neighbors,
                                 const lsmps_params* params, int32_t* open_direction_count,
                                 double* open_fraction);

/* ------------------------------------------------------------------------- */
/* Moment matrices: include/lsmps3d/moment_matrix/moment_matrix.cuh          */
/* ------------------------------------------------------------------------- */
/* Build and invert the moment matrices of `count` kinds at once
 * (DeviceMomentMatrix::prepare_matrices, moment_matrix.cuh:80-84, without the
 * host-side generation cache, which the C++/Python owners keep).  Kinds that
 * share the Type-A fluid sum are assembled in one pass over the rows.  Each
 * inversion_count is incremented once. */
lsmps_status lsmps_prepare_moments(lsmps_ctx* ctx, const lsmps_fluid* fluid,
                                   const lsmps_walls* walls, const lsmps_csr* fluid_neighbors,
                                   const lsmps_csr* wall_neighbors, const lsmps_params* params,
                                   const lsmps_moment* kinds, int count);

/* ------------------------------------------------------------------------- */
/* Provision: include/lsmps3d/provision/explicit_update.cuh                  */
/* ------------------------------------------------------------------------- */
/* compute_velocity_laplacian_kernel launch inside
 * DeviceProvisionExplicitUpdate::compute_temporary_velocity
 * (src/provision/explicit_update.cu:178-248, 391-395). */
lsmps_status lsmps_velocity_laplacian(lsmps_ctx* ctx, const lsmps_fluid* fluid,
                                      const lsmps_walls* walls, const lsmps_csr* fluid_neighbors,
                                      const lsmps_csr* wall_neighbors,
                                      const lsmps_moment* velocity_moment,
                                      const lsmps_vector* laplacian);
/* compute_provision_temporary_velocity(...), explicit_update.cuh:84-87. */
lsmps_status lsmps_temporary_velocity(lsmps_ctx* ctx, const lsmps_fluid* fluid,
                                      const lsmps_params* params, const lsmps_vector* laplacian,
                                      const lsmps_fluid* temporary_velocity);
/* compute_provision_temporary_wall_velocity(...), explicit_update.cuh:89-91. */
lsmps_status lsmps_temporary_wall_velocity(lsmps_ctx* ctx, const lsmps_walls* walls,
                                           const lsmps_params* params,
                                           const lsmps_walls* temporary_wall_velocity);

/* ------------------------------------------------------------------------- */
/* PPE assembly: include/lsmps3d/ppe/ppe_matrix.cuh                          */
/* ------------------------------------------------------------------------- */
/* assemble_ppe_matrix_and_rhs(...), ppe_matrix.cuh:120-129.  Row i starts at
 * i + fluid_offsets[i]; the diagonal comes first, then one slot per fluid
 * neighbour in CSR order.  Surface and Splash rows are Dirichlet rows. */
lsmps_status lsmps_assemble_ppe(lsmps_ctx* ctx, const lsmps_fluid* fluid,
                                const lsmps_walls* walls, const lsmps_params* params,
                                const lsmps_csr* fluid_neighbors, const lsmps_csr* wall_neighbors,
                                const lsmps_fluid* temporary_velocity,
                                const lsmps_walls* temporary_wall_velocity,
                                const lsmps_moment* velocity_moment,
                                const lsmps_moment* pressure_moment, const lsmps_ppe* workspace);

/* ------------------------------------------------------------------------- */
/* PPE solve: AmgxPpeSolver::solve, include/lsmps3d/ppe/ppe_matrix.cuh:88-110 */
/* ------------------------------------------------------------------------- */
/* The reference solves the assembled system with AMGX (src/ppe/ppe_matrix.cu:
 * 586-679; a third-party library, used only when found at build time) in
 * AMGX's GMRES configuration (:604-610).  lsmps_solve_ppe solves it on the
 * device with restarted GMRES (Saad & Schultz), keeping the reference's
 * semantics: initial guess zero, stop at max_iters or when the residual's L2
 * norm reaches tolerance x the initial one, then clamp negative values to
 * zero (:662).  Works on any square CSR matrix (row_offsets[rows] entries
 * used; nnz is not read). */
enum {
  LSMPS_CONVERGENCE_RELATIVE_INITIAL = 0, /* AMGX "RELATIVE_INI": |r| <= tol |r0| */
  LSMPS_CONVERGENCE_ABSOLUTE = 1          /* AMGX "ABSOLUTE": |r| <= tol */
};
enum {
  LSMPS_PRECONDITIONER_NONE = 0,  /* AMGX "NOSOLVER" (the reference's configuration) */
  LSMPS_PRECONDITIONER_JACOBI = 1 /* right preconditioning with diag(A) */
};
typedef struct lsmps_solver_options {
  int32_t max_iters;         /* total Arnoldi steps over all restarts; 100 */
  int32_t restart;           /* Krylov dimension per cycle, 1..64; 20 */
  double tolerance;          /* 1e-6 */
  int32_t convergence;       /* LSMPS_CONVERGENCE_* */
  int32_t preconditioner;    /* LSMPS_PRECONDITIONER_* */
  int32_t clamp_negative;    /* 1: pressure = max(pressure, 0) afterwards */
  int32_t use_initial_guess; /* 0: start from zero, as the reference */
} lsmps_solver_options;
typedef struct lsmps_solver_report {
  int32_t iterations;      /* Arnoldi steps taken */
  int32_t converged;       /* 1 if the final true residual met the criterion */
  double initial_residual; /* |b - A x0| */
  double final_residual;   /* |b - A x| before the clamp */
} lsmps_solver_report;
void lsmps_solver_options_default(lsmps_solver_options* options);
/* options may be NULL (defaults); report may be NULL.  Not capturable in a
 * CUDA graph: each Arnoldi step reads 17 bytes back to the host. */
lsmps_status lsmps_solve_ppe(lsmps_ctx* ctx, const lsmps_csr_matrix* matrix, const double* rhs,
                             double* pressure, const lsmps_solver_options* options,
                             lsmps_solver_report* report);

/* ------------------------------------------------------------------------- */
/* Pressure correction: include/lsmps3d/correction/pressure_correction.cuh   */
/* ------------------------------------------------------------------------- */
/* clamp_particle_pressure(...), pressure_correction.cuh:91. */
lsmps_status lsmps_clamp_particle_pressure(lsmps_ctx* ctx, const lsmps_fluid* fluid,
                                           double* pressure);
/* compute_pressure_gradient(...), pressure_correction.cuh:93-100. */
lsmps_status lsmps_pressure_gradient(lsmps_ctx* ctx, const lsmps_fluid* fluid,
                                     const lsmps_walls* walls, const lsmps_csr* fluid_neighbors,
                                     const lsmps_csr* wall_neighbors, const double* pressure,
                                     const lsmps_params* params,
                                     const lsmps_moment* pressure_moment,
                                     const lsmps_vector* gradient);
/* compute_particle_shifting_displacement(...), pressure_correction.cuh:102-107. */
lsmps_status lsmps_particle_shifting(lsmps_ctx* ctx, const lsmps_fluid* fluid,
                                     const lsmps_walls* walls, const lsmps_csr* fluid_neighbors,
                                     const lsmps_csr* wall_neighbors, const lsmps_params* params,
                                     const lsmps_vector* displacement);
/* update_velocity_and_position(...), pressure_correction.cuh:109-113. */
lsmps_status lsmps_update_velocity_position(lsmps_ctx* ctx, const lsmps_fluid* fluid,
                                            const lsmps_fluid* temporary_velocity,
                                            const lsmps_params* params,
                                            const lsmps_vector* gradient,
                                            const lsmps_vector* displacement);
/* anti_penetration_kernel launch in DevicePressureCorrection::apply
 * (src/correction/pressure_correction.cu:404-444, 639-643). */
lsmps_status lsmps_anti_penetration(lsmps_ctx* ctx, const lsmps_fluid* fluid,
                                    const lsmps_walls* walls, const lsmps_csr* wall_neighbors,
                                    const lsmps_params* params);
/* smooth_particle_velocity(...), pressure_correction.cuh:115-118. */
lsmps_status lsmps_smooth_particle_velocity(lsmps_ctx* ctx, const lsmps_fluid* fluid,
                                            const lsmps_csr* fluid_neighbors,
                                            const lsmps_params* params,
                                            const lsmps_vector* smoothed_velocity);
/* DevicePressureCorrection::apply(...) after prepare_matrices,
 * pressure_correction.cuh:69-76 (src/correction/pressure_correction.cu:598-645):
 * clamp -> gradient -> shifting -> update -> anti-penetration -> smoothing. */
lsmps_status lsmps_pressure_correction(lsmps_ctx* ctx, const lsmps_fluid* fluid,
                                       const lsmps_walls* walls,
                                       const lsmps_csr* fluid_neighbors,
                                       const lsmps_csr* wall_neighbors,
                                       const lsmps_fluid* temporary_velocity, double* pressure,
                                       const lsmps_params* params,
                                       const lsmps_moment* pressure_moment,
                                       const lsmps_vector* gradient,
                                       const lsmps_vector* displacement,
                                       const lsmps_vector* smoothed_velocity);

/* ------------------------------------------------------------------------- */
/* Time-step control on the device (simulation_driver.cu:110-143, 337-338;    */
/* SimulationTimeManager, include/lsmps3d/core/time_step.hpp)                */
/* ------------------------------------------------------------------------- */
/* TimeStepLimits (time_step.hpp:9-18) without the output interval (output
 * scheduling is host I/O). */
typedef struct lsmps_time_limits {
  double min_time_step;
  double max_time_step;
  double growth_factor;   /* >= 1 */
  double cfl;
  double particle_spacing;
  double final_time;
} lsmps_time_limits;
/* The time manager's state, kept in DEVICE memory by the caller. */
typedef struct lsmps_time_state {
  double current_time;
  double time_step;      /* dt of the step just advanced (the config's time_step) */
  double cfl_time_step;
  double max_velocity;   /* largest finite |u| at the start of the step */
  uint64_t step_index;
} lsmps_time_state;
/* SimulationTimeManager::reset (time_step.cpp:85-94): time 0, time step
 * clamped to [min, max].  Host-only; copy the result to device memory. */
void lsmps_time_state_init(const lsmps_time_limits* limits, double time_step, lsmps_time_state* host_state);
/* max_velocity (the largest finite |u| over the fluid) followed by
 * SimulationTimeManager::advance (time_step.cpp:104-132) on *device_state:
 * dt = clamp(min(dt_prev * growth, cfl * l0 / |u|max), min, max), cut to the
 * remaining time; time += dt.  No host round trip (capturable). */
lsmps_status lsmps_advance_time(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_time_limits* limits,
                                lsmps_time_state* device_state);
/* While set, every kernel of the step that uses the time step (u* combine,
 * PPE right-hand side, velocity/position update) reads it from this device
 * address (e.g. &device_state->time_step) instead of lsmps_params.time_step;
 * NULL restores lsmps_params.time_step. */
lsmps_status lsmps_ctx_set_device_time_step(lsmps_ctx* ctx, const double* device_time_step);

/* ------------------------------------------------------------------------- */
/* Whole step (src/app/simulation_driver.cu:346-383 minus the solve and I/O) */
/* ------------------------------------------------------------------------- */
/* One time step on the state's buffers: moments (velocity and pressure
 * Type-A, once per geometry) -> provision -> PPE assembly -> correction with
 * `pressure` -> neighbour rebuild -> surface labels.  Uses the context's
 * precision mode. */
lsmps_status lsmps_step(lsmps_ctx* ctx, const lsmps_params* params, const lsmps_step_state* state);
/* Copy/compute overlap for a caller whose particle state lives in host memory
 * (no counterpart in the reference, whose state stays on the device).  All
 * are cudaEvent_t handles (NULL: not used), used by every following lsmps_step
 * of this context while its stream is not being captured; only the fluid
 * positions must be in place when the step is queued:
 *   wall_event   - the step waits for it before it first reads the walls'
 *                  positions and normals (in the mixed form after the fluid
 *                  moment sums, in the plain form before the moment stage);
 *   input_event  - the step waits for it after its moment stage and before the
 *                  provision stage: the fluid velocities, pressure and labels
 *                  and the wall velocities may still be arriving while the
 *                  moments are built;
 *   output_event - the step records it once the pressure correction is done:
 *                  the fluid positions, velocities and pressure are final and
 *                  can be copied out while the neighbour rebuild and the labels
 *                  run (the labels are final only at the end of the step). */
lsmps_status lsmps_ctx_set_step_events(lsmps_ctx* ctx, void* wall_event, void* input_event, void* output_event);

/* ------------------------------------------------------------------------- */
/* Batched boxes in one CUDA graph (no counterpart in the reference)          */
/* ------------------------------------------------------------------------- */
/* Many independent boxes (each its own params and step state, of any size)
 * stepped by one captured CUDA graph.  The batch owns `streams` worker
 * streams, each with its own context; box b runs on stream b mod streams, so
 * boxes on different streams overlap on the GPU.
 *   create -> add every box -> capture(precision) -> launch (repeatedly) ->
 *   synchronize (folds every worker context's device status) -> destroy.
 * capture reserves each worker context for its largest box, optionally runs
 * lsmps_autotune on that box (autotune_repeats > 0; 0 keeps the defaults),
 * then records one lsmps_step per box between a fork and a join on the
 * batch's origin stream.  Each launch advances every box by one step; the
 * boxes' buffers must stay valid and keep their sizes while the graph
 * exists. */
typedef struct lsmps_batch lsmps_batch;
lsmps_status lsmps_batch_create(int device, int streams, lsmps_batch** out);
void lsmps_batch_destroy(lsmps_batch* batch);
lsmps_status lsmps_batch_add(lsmps_batch* batch, const lsmps_params* params, const lsmps_step_state* state);
int lsmps_batch_size(lsmps_batch* batch);
lsmps_status lsmps_batch_capture(lsmps_batch* batch, int precision, int autotune_repeats);
/* Form of the graph, chosen before capture (no counterpart in the reference).
 * 1 (default): merged -- when the boxes differ only in their cell grids
 * (origin, dims), all boxes are stepped as one particle set: each launch
 * gathers the boxes' particle state (fluid SoA, labels, pressure input,
 * walls) into the batch's merged buffers, runs one lsmps_step on the merged
 * set (every kernel one grid-wide launch over all boxes; the cell hash and
 * the neighbour search keep each particle on its own box's grid), and
 * scatters every output back into the boxes' views.  The merged neighbour
 * tables and cell lists stay the batch's own between launches (capture builds
 * them from the boxes' positions; each launch ends with their rebuild): the
 * boxes' copies are outputs, and changes a caller makes to them are not read.
 * Boxes whose other parameters differ fall back to form 0.
 * 0: one lsmps_step per box on the worker streams.
 * Either way each box's results equal its own lsmps_step bit for bit.
 * lsmps_batch_merged reports the form the last capture used. */
lsmps_status lsmps_batch_set_merged(lsmps_batch* batch, int on);
int lsmps_batch_merged(lsmps_batch* batch);
/* stream: where the graph is launched (NULL: the batch's origin stream). */
lsmps_status lsmps_batch_launch(lsmps_batch* batch, void* stream);
lsmps_status lsmps_batch_synchronize(lsmps_batch* batch);
void* lsmps_batch_stream(lsmps_batch* batch);
const char* lsmps_batch_last_error(lsmps_batch* batch);

/* ------------------------------------------------------------------------- */
/* Differentiable operators (no counterpart in the reference)                */
/* ------------------------------------------------------------------------- */
/* Outputs of lsmps_operators_forward, or (to lsmps_operators_backward) the
 * cotangents dL/d(output) of a loss L.  Per fluid particle, over its fluid CSR
 * row, with the fluid-only Type-A moment matrix (kind FLUID_ONLY_A):
 *   grad_*      LSMPS gradient of the scalar field f
 *   laplacian   LSMPS Laplacian of f (2/r_e^2 times rows 3..5)
 *   divergence  LSMPS divergence of the vector field v
 *   ppe_*       optional fluid-only PPE rows in the reference's layout
 *               (diagonal first, then the CSR row; ppe_matrix.cu:243-370
 *               without wall terms): row_offsets[count + 1], col_indices and
 *               values[count + K]; ppe_rhs = divergence / dt.
 * Any pointer may be NULL: the output is not written (forward) or its
 * cotangent is zero (backward; ppe_row_offsets / ppe_col_indices are not
 * read). */
typedef struct lsmps_operator_out {
  size_t count;
  double* grad_x;
  double* grad_y;
  double* grad_z;
  double* laplacian;
  double* divergence;
  int32_t* ppe_row_offsets;
  int32_t* ppe_col_indices;
  double* ppe_values;
  double* ppe_rhs;
} lsmps_operator_out;

/* fluid: positions (x, y, z, count; other fields unused); fn: its fluid CSR
 * (the topology is an input: it is held fixed under differentiation).  If
 * inverse_out is not NULL it receives the count x 81 inverses (column-major),
 * which lsmps_operators_backward can reuse instead of recomputing them. */
lsmps_status lsmps_operators_forward(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_csr* fn,
                                     const lsmps_params* params, const double* f, const lsmps_vector* v,
                                     const lsmps_operator_out* out, double* inverse_out);
/* Gradients of L with respect to f (f_bar), v (v_bar) and the positions
 * (x_bar), each optional (NULL: not computed) and overwritten.  inverse: the
 * forward's inverse_out, or NULL to recompute the inverses from the positions
 * (the memory-lean choice: nothing of the forward has to be kept). */
lsmps_status lsmps_operators_backward(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_csr* fn,
                                      const lsmps_params* params, const double* f, const lsmps_vector* v,
                                      const lsmps_operator_out* cotangent, const double* inverse, double* f_bar,
                                      const lsmps_vector* v_bar, const lsmps_vector* x_bar);
/* The step's operators with their wall terms, as a differentiable pair (no
 * counterpart in the reference).  Per fluid particle i over its fluid and
 * wall CSR rows, with the velocity Dirichlet-A moment matrix M_v (wall
 * samples lambda_w w b b^T) and the pressure Neumann-A matrix M_p (wall
 * terms lambda_w w q q^T with the Neumann vector q), both regularised as
 * the step does (moment_matrix.cu:177-201, 254-309):
 *   lap_*        velocity Laplacian of u, wall samples lambda_w w b (u_w - u_i)
 *                (explicit_update.cu:178-248)
 *   divergence   divergence of u with M_v (ppe_matrix.cu:355-361); 0 on the
 *                Dirichlet rows (Surface and Splash)
 *   grad_*       pressure gradient of p with M_p and the wall source
 *                lambda_w w q (r_e rho g.n) (pressure_correction.cu:200-276);
 *                0 for Splash
 *   ppe_*        the PPE rows of the pressure Laplacian row of M_p, Dirichlet
 *                rows for Surface and Splash (ppe_matrix.cu:243-370);
 *                ppe_rhs = divergence / dt - wall_rhs
 *   wall_rhs     the wall Neumann term sum 2 lambda_w w (g.n) (L.q) / r_e
 * Inputs: fluid x, y, z, vx, vy, vz (u), pressure (p) and surface_type
 * (NULL: all Inner); walls x, y, z, vx, vy, vz (u_w) and normals.  Labels,
 * walls and both CSR tables are held fixed under differentiation.  Any
 * output pointer may be NULL (not written; in the backward: zero cotangent;
 * ppe_row_offsets / ppe_col_indices are not read). */
typedef struct lsmps_step_operator_out {
  size_t count;
  double* lap_x;
  double* lap_y;
  double* lap_z;
  double* divergence;
  double* grad_x;
  double* grad_y;
  double* grad_z;
  int32_t* ppe_row_offsets;
  int32_t* ppe_col_indices;
  double* ppe_values;
  double* ppe_rhs;
  double* wall_rhs;
} lsmps_step_operator_out;
lsmps_status lsmps_step_operators_forward(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_walls* walls,
                                          const lsmps_csr* fn, const lsmps_csr* wn, const lsmps_params* params,
                                          const lsmps_step_operator_out* out);
/* Gradients of L with respect to u (u_bar), p (p_bar) and the fluid
 * positions (x_bar), each optional and overwritten; the inverses are
 * recomputed from the positions.  Deterministic or atomic as set by
 * lsmps_ctx_set_adjoint_atomic (the wall terms are the owner's own and need
 * neither). */
lsmps_status lsmps_step_operators_backward(lsmps_ctx* ctx, const lsmps_fluid* fluid, const lsmps_walls* walls,
                                           const lsmps_csr* fn, const lsmps_csr* wn, const lsmps_params* params,
                                           const lsmps_step_operator_out* cotangent, const lsmps_vector* u_bar,
                                           double* p_bar, const lsmps_vector* x_bar);
/* Form of lsmps_operators_backward (no counterpart in the reference).
 * 0 (default): deterministic -- the CSR is transposed (entries sorted stably
 * by neighbour) and every particle gathers the terms of its own row and of
 * the rows that list it in a fixed order, with no atomics; repeated calls give
 * the same bits.  Costs a sort of the K entries and 20 bytes of scratch per
 * entry.  1: each row scatters its terms into its neighbours with FP64
 * atomics (no transpose; the sums' order, and so the last bits, may vary
 * between calls). */
lsmps_status lsmps_ctx_set_adjoint_atomic(lsmps_ctx* ctx, int on);

#ifdef __cplusplus
}
#endif

#endif /* LSMPS_B200_H */

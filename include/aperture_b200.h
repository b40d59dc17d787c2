/*
 * aperture_b200.h -- C ABI of the B200 particle update for Aperture3 labs.
 *
 * Replaces the CUDA implementations behind the reference's algorithm
 * classes (src/algorithms/ptc_updater.h, field_solver.h) for Cartesian 1D
 * and 2D grids: the Vay push fused with charge-conserving (Esirkepov)
 * current deposition, the periodic guard exchange of a single rank, and
 * the Yee FDTD field update. All arrays are device memory owned by the
 * caller (sim_data in the reference); the library owns only its scratch.
 *
 * Conventions
 *  - Every function returns an ap_status (0 == AP_OK).
 *  - Field arrays are pitched like cudaMalloc3D arrays (pitch in bytes,
 *    dims[1] * dims[2] rows of dims[0] floats), as multi_array
 *    (src/core/multi_array.h) stores them.
 *  - Particles use the reference SoA members (src/data/particle_data.h:50-61).
 *    cell == AP_MAX_CELL marks an empty slot.
 *  - By default each call synchronises its stream before returning, as the
 *    reference calls cudaDeviceSynchronize after each kernel
 *    (ptc_updater.cu:776-777); ap_set_sync(ctx, 0) makes calls asynchronous.
 */
#ifndef APERTURE_B200_H_
#define APERTURE_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define AP_API __attribute__((visibility("default")))
#else
#define AP_API
#endif

#define AP_MAX_CELL 0xFFFFFFFFu
#define AP_MAX_SPECIES 8

typedef enum {
  AP_OK = 0,
  AP_ERR_INVALID = 1,      /* bad argument, or a call made in the wrong state */
  AP_ERR_CUDA = 2,         /* a CUDA runtime call failed                       */
  AP_ERR_NAN = 3,          /* NaN momentum met by the push (reference: trap)   */
  AP_ERR_MOVED_FAR = 4,    /* a particle moved more than one cell in a step    */
  AP_ERR_CAPACITY = 5,     /* a size exceeds a fixed limit                     */
  AP_ERR_TIMEOUT = 6,      /* a bounded device-side wait gave up               */
  AP_ERR_UNSUPPORTED = 7,  /* grid dimension / option not implemented          */
  AP_ERR_NOMEM = 8,        /* device allocation failed                         */
  AP_ERR_TILE = 9          /* a particle was found outside its sort tile       */
} ap_status;

/* Same members and layout as Quadmesh (src/core/quadmesh.h:16-29). */
typedef struct {
  int dims[3];
  int guard[3];
  float delta[3];
  float inv_delta[3];
  float lower[3];
  float sizes[3];
  int dimension;
} ap_mesh;

/* The SimParams fields the particle update and field solver read
 * (src/sim_params.h:17-123) plus the per-species charges and masses
 * (sim_environment_impl.hpp:90-101), and the device tile shape. */
typedef struct {
  int num_species;           /* Rho arrays present (1..8)                   */
  int data_interval;         /* Rho is deposited when (step+1) % it == 0   */
  int current_smoothing;     /* binomial filter passes over J per step     */
  int periodic[3];           /* periodic_boundary                          */
  float charges[AP_MAX_SPECIES];
  float masses[AP_MAX_SPECIES];
  int tile[2];               /* sort tile in cells; 0 picks a default       */
  int chunk;                 /* particles staged per pass in the 2D kernel:
                                256, 512, 1024 or 2048; 0 picks a default   */
} ap_params;

typedef struct {
  float *ptr;
  size_t pitch; /* bytes between rows */
} ap_array;

/* The sim_data members used by the update (src/sim_data.h:14-70). */
typedef struct {
  ap_array E[3], B[3], Ebg[3], Bbg[3], J[3];
  ap_array Rho[AP_MAX_SPECIES];
  ap_array divE, divB;
} ap_fields;

/* particle_data (src/data/particle_data.h:50-61). */
typedef struct {
  float *x1, *x2, *x3;
  float *p1, *p2, *p3;
  float *E, *weight;
  uint32_t *cell;
  uint64_t *id;
  uint32_t *flag;
} ap_particles;

/* Counters of the last update, read back from the device status word. */
typedef struct {
  uint64_t nan_momenta;  /* particles skipped for NaN momentum            */
  uint64_t moved_far;    /* particles with |dc| > 1 (deposit skipped)     */
  uint64_t lost;         /* particles that left through a non-periodic side */
  uint64_t tile_faults;  /* particles found outside their tile            */
  uint64_t live;         /* particles in the tile order after the update  */
} ap_step_stats;

/* FP64 diagnostics: the reductions are done on the device in double. */
typedef struct {
  double kinetic;        /* sum w * m * (gamma - 1) over live particles      */
  double charge;         /* sum q * w over live particles                    */
  double field_energy;   /* 0.5 * sum (E^2 + B^2) * cell volume over the bulk */
  double max_abs_rho;    /* max |rho_total| over the bulk                    */
  double gauss_residual; /* max |divE - sum rho| over the bulk               */
  double max_abs_j;      /* max |J| over the bulk, all components            */
  double continuity_residual; /* max |rho(t+1) - rho(t) + div J| over the bulk,
                               * from the last update (ap_set_continuity_check);
                               * NaN when it was not recorded               */
} ap_diag;

typedef struct ap_ctx ap_ctx;

/* Library version string. */
AP_API const char *ap_version(void);
/* Human-readable name of an ap_status. */
AP_API const char *ap_status_string(int status);

/* Creates a context for one rank's grid. Replaces the constructors
 * ptc_updater(sim_environment&) (ptc_updater.cu:742-744) and
 * field_solver(sim_environment&) (field_solver.cu:330), and the
 * __constant__ mesh/params upload of setup_env_extra
 * (cuda/sim_environment.cpp:129-157). Uses the current CUDA device. */
AP_API int ap_ctx_create(const ap_mesh *mesh, const ap_params *params,
                         ap_ctx **out);
AP_API int ap_ctx_destroy(ap_ctx *ctx);

/* Stream used by every launch of this context (default: a private
 * non-blocking stream). */
AP_API int ap_set_stream(ap_ctx *ctx, void *cuda_stream);
/* 1 (default): every call synchronises before returning and reports device
 * status; 0: calls only enqueue work, ap_sync() reports status. */
AP_API int ap_set_sync(ap_ctx *ctx, int sync);
AP_API int ap_sync(ap_ctx *ctx);

/* Binds the field arrays (get_data_ptrs, cuda/sim_data.cu:295). */
AP_API int ap_bind_fields(ap_ctx *ctx, const ap_fields *fields);
/* Binds the particle arrays: slots [0, number) are in use, capacity is the
 * allocated length (particles_t, core/particle_base.h). */
AP_API int ap_bind_particles(ap_ctx *ctx, const ap_particles *ptc,
                             size_t number, size_t capacity);
/* Tells the context that the caller changed particle slots (cells, counts)
 * since the last update; the tile order is rebuilt at the next update. */
AP_API int ap_particles_modified(ap_ctx *ctx, size_t number);
AP_API int ap_get_number(const ap_ctx *ctx, size_t *number);
/* Slots [*first, *end) hold every particle (holes included); first is 0
 * unless a compaction wrote the store into the upper half of the capacity
 * (ap_set_compaction), end is the particle number. */
AP_API int ap_get_slot_range(const ap_ctx *ctx, size_t *first, size_t *end);

/* ptc_updater::update_particles(sim_data&, double dt, uint32_t step)
 * (ptc_updater.cu:748-841): zero J (and Rho), push, deposit + move, fold
 * the guard current, smooth, and wrap particles through periodic sides. */
AP_API int ap_update_particles(ap_ctx *ctx, double dt, uint32_t step);
/* ptc_updater::smooth_current(sim_data&, uint32_t) (ptc_updater.cu:852-873). */
AP_API int ap_smooth_current(ap_ctx *ctx, uint32_t step);
/* ptc_updater::smooth_current(multi_array<Scalar>&) (ptc_updater.cu:875-912):
 * one filter pass over one array (no guard refresh). */
AP_API int ap_smooth_array(ap_ctx *ctx, ap_array a);

/* field_solver::update_fields(sim_data&, double dt, uint32_t step)
 * (field_solver.cu:334-358). */
AP_API int ap_update_fields(ap_ctx *ctx, double dt, uint32_t step);
/* field_solver::update_e_field / update_b_field / compute_divs
 * (field_solver.cu:404-449, 360-402, 454-504). These write the bulk and,
 * in periodic dims, the guard images of the updated cells. */
AP_API int ap_update_e_field(ap_ctx *ctx, double dt);
AP_API int ap_update_b_field(ap_ctx *ctx, double dt);
AP_API int ap_compute_divs(ap_ctx *ctx);

/* sim_environment::send_guard_cells / send_add_guard_cells for one array on
 * one rank (sim_environment_impl.hpp:274-317, cuda/sim_environment.cpp:
 * 9-127): periodic copy / fold of the guard strips. */
AP_API int ap_send_guard_cells(ap_ctx *ctx, ap_array a);
AP_API int ap_send_add_guard_cells(ap_ctx *ctx, ap_array a);

/* 2D: every `interval` updates (0 = never, the default), rewrite the
 * particle arrays in tile order before the push, so that each tile's
 * particles sit in consecutive slots again (new; between sorts the
 * reference keeps every particle in its slot). Particles change slots, not
 * values; slots after the live ones become empty (cell == AP_MAX_CELL).
 * This bounds the scatter of the particle accesses that grows as particles
 * cross tiles. */
AP_API int ap_set_compaction(ap_ctx *ctx, int interval);
/* FP64 continuity check (new; derived from the deposit of
 * ptc_updater.cu:295-386 and the divergence of compute_divs_2d,
 * field_solver.cu:237-288). While on (1), every Cartesian update_particles
 * that deposits Rho right after an update that also deposited it records,
 * on the device and in FP64, max |sum_s Rho_s(t+1) - sum_s Rho_s(t) +
 * J1(i+1) - J1(i) + J2(j+1) - J2(j)| over the bulk cells (the face past the
 * last bulk cell is the first one's periodic image on periodic sides), in
 * the deposit's own units; ap_diagnostics reports it as
 * continuity_residual. Other updates report NaN. Off by default; costs one
 * FP64 copy of the charge density per output step while on. */
AP_API int ap_set_continuity_check(ap_ctx *ctx, int on);

/* sim_data::sort_particles -> particle_base::sort_by_cell
 * (sim_data_impl.hpp:78-89, cuda/core/particle_base_impl.cu:435-487):
 * stable sort of all SoA members by cell, empty slots last and trimmed;
 * bound photons are sorted the same way. */
AP_API int ap_sort_by_cell(ap_ctx *ctx);

/* The device tile order maintained by the per-step counting sort: order has
 * `live` entries (particle slot indices grouped by tile, stable), and
 * tile_start has ntiles + 1 entries. Pointers stay valid until the next
 * update. */
AP_API int ap_get_tile_order(ap_ctx *ctx, const uint32_t **order,
                             const uint32_t **tile_start, uint32_t *ntiles,
                             size_t *live);

/* Counters of the last update (waits for the stream). */
AP_API int ap_get_stats(ap_ctx *ctx, ap_step_stats *stats);
/* FP64 energy / charge / Gauss-law diagnostics (new; the reference only
 * computes per-particle gamma, cuda/core/particles.cu:10-22). */
AP_API int ap_diagnostics(ap_ctx *ctx, ap_diag *out);
/* The same reductions without waiting: the seven values (in ap_diag's member
 * order) are copied to host_out, which should be pinned host memory, on the
 * context's stream; they are there after the next ap_sync. A 1D context
 * whose particle count moved on the device (pair injection) must be synced
 * first. */
AP_API int ap_diagnostics_async(ap_ctx *ctx, double *host_out);
/* Failure-detection self-test: waits, with the bounded wait the 2D kernel
 * uses for its field tiles and a short limit, on a barrier that nothing
 * completes, and returns the status the give-up produces (AP_ERR_TIMEOUT).
 * Nothing is left running; the context stays usable. */
AP_API int ap_selftest_wait_timeout(ap_ctx *ctx);

/* ---------------------------------------------------------------------
 * Log-spherical (ln r, theta) grids: ptc_updater_logsph and
 * field_solver_logsph (src/algorithms/ptc_updater_logsph.h:13-28,
 * field_solver_logsph.h:10-20). Dimension 0 is ln r, dimension 1 is
 * theta in [lower, lower + size]; both dims non-periodic.
 *
 * The dev_params members these kernels read (src/sim_params.h:31-48):
 * user_push_2d_logsph.cuh:14-114 (gravity, rad_cooling_*, B0),
 * field_solver_logsph.cu:16-26 (compactness, omega in beta_phi),
 * ptc_updater_logsph.cu:440-455 and field_solver_logsph.cu:322-345
 * (damping_length, damping_coef). */
typedef struct {
  float compactness;
  float omega;
  float gravity;          /* applied every push, as the reference does */
  float rad_cooling_coef;
  float B0;
  float damping_coef;
  int rad_cooling_on;
  int damping_length;
} ap_logsph_params;

/* Coefficient arrays of Grid_LogSph (grid_log_sph.h:45-47). */
enum {
  AP_COEF_L1E = 0, AP_COEF_L2E, AP_COEF_L3E, AP_COEF_L1B, AP_COEF_L2B,
  AP_COEF_L3B, AP_COEF_A1E, AP_COEF_A2E, AP_COEF_A3E, AP_COEF_A1B,
  AP_COEF_A2B, AP_COEF_A3B, AP_COEF_DV, AP_NUM_COEF
};

/* Creates a log-spherical context: ap_ctx_create plus Grid_LogSph::
 * compute_coef (grid_log_sph.cpp:11-126), evaluated on the host in the
 * reference's float / double arithmetic and kept on the device. With such
 * a context ap_update_particles runs ptc_updater_logsph::update_particles
 * followed by its apply_boundary (ptc_updater_logsph.cu:681-836),
 * ap_update_fields runs field_solver_logsph::update_fields
 * (field_solver_logsph.cu:354-398; its step argument is unused) and
 * ap_compute_divs runs compute_divs_logsph. */
AP_API int ap_ctx_create_logsph(const ap_mesh *mesh, const ap_params *params,
                                const ap_logsph_params *lsp, ap_ctx **out);
/* Device view of one coefficient array (mesh_ptrs_log_sph,
 * cuda/grids/grid_log_sph_ptrs.h:8-17); which is an AP_COEF_* value. */
AP_API int ap_logsph_coef(ap_ctx *ctx, int which, ap_array *out);
/* field_solver_logsph::apply_boundary(data, omega, time)
 * (field_solver_logsph.cu:403-428) on one rank: stellar surface, outflow
 * damping, and both axes. */
AP_API int ap_logsph_field_boundary(ap_ctx *ctx, double omega);
/* ptc_updater_logsph::inject_ptc (ptc_updater_logsph.cu:301-393, 441-490,
 * 849-870): measures the electron and ion densities next to the stellar
 * surface and, in every theta row but the outermost whose density times
 * q_e stays below 1.5 sin(theta) / dtheta^2, adds inj_per_cell e-/e+ pairs
 * in cell (guard0 + 2, row): x1 = 0.5, x2 uniform, p1' = 2 p1 |cos theta|,
 * p2' = p1 sin theta sgn(cos theta), p3' = 0, E = sqrt(1 + p1^2), weight
 * w sin theta, flag primary. The particle number grows by 2 inj_per_cell
 * per bulk theta row (rows without injection leave empty slots); x2 is
 * drawn from Philox4x32-10 keyed by seed with the call count as counter,
 * in place of the reference's cuRAND states. p2, p3 and omega are accepted
 * and, as in the reference's kernel, unused. */
AP_API int ap_logsph_inject(ap_ctx *ctx, int inj_per_cell, float p1, float p2, float p3,
                            float w, float omega, uint64_t seed);

/* 1D gap lab (labs/1dgap; src/algorithms/ptc_updater_1dgap.h,
 * field_solver_1dgap.h). A context made here runs, in ap_update_particles,
 * ptc_updater_1dgap::update_particles (ptc_updater_1dgap.cu:219-272): E3 is
 * set to E1 smoothed current_smoothing times (E2 is the scratch), the gap
 * pusher with beta_phi(x) = x moves the particles (no wrap; a particle
 * outside the bulk is emptied at the next update), J1 (times delta / dt)
 * and every species' Rho are deposited on every step and smoothed; and in
 * ap_update_fields field_solver_1dgap::update_fields (field_solver_1dgap.cu:
 * 28-40): E1 += (j0 - J1) dt on the bulk cells but the outermost, with
 * j0 = 1.6 B0. */
typedef struct {
  float B0;                  /* SimParams::B0                               */
} ap_gap_params;
AP_API int ap_ctx_create_1dgap(const ap_mesh *mesh, const ap_params *params,
                               const ap_gap_params *gap, ap_ctx **out);

/* 1D GR lab (labs/1dgr; src/algorithms/ptc_updater_1dgr.h,
 * field_solver_1dgr.h, src/grids/grid_1dgr.h). A context made here holds
 * the metric coefficients of Grid_1dGR::compute_coef (grid_1dgr.cpp:21-187),
 * computed on the host as the reference does from the tabulated field-line
 * data it reads from coef.h5 (radius r, B^1, B^3, j^1, rho, theta and
 * dpsi/dtheta, table.n entries each, r increasing), so no HDF5 is needed.
 * ap_update_particles then runs ptc_updater_1dgr::update_particles
 * (ptc_updater_1dgr.cu:418-473): E3 = E1 smoothed current_smoothing times
 * by the K1_j-weighted filter (E2 is the scratch), the GR pusher
 * (update_ptc_1dgr, :137-300; tracked particles get the lower u_0 in p2
 * every data_interval steps), J1 through K1_j times delta / dt and every
 * species' Rho through K1 on every step, then J1 and Rho smoothed; and
 * ap_update_fields field_solver_1dgr::update_fields (field_solver_1dgr.cu:
 * 14-44): E1 += (j0 - J1) dt on cells [guard + 1, dims - guard - 5). A
 * particle that would move more than one cell (which the reference reports
 * and follows past the coefficient arrays) is emptied and counted as
 * AP_ERR_MOVED_FAR. */
typedef struct {
  float a;      /* SimParams::a, the black hole's spin */
  float omega;  /* SimParams::omega, the field line's angular velocity */
  float B0;     /* SimParams::B0 */
} ap_gr_params;
typedef struct {
  const float *r, *B1, *B3, *jr, *rho, *theta, *dpsidth; /* host arrays of n floats */
  size_t n;
} ap_gr_table;
/* Coefficient arrays of Grid_1dGR, in the order of its mesh_ptrs
 * (grid_1dgr.h:16-20); theta and agrf stay zero, as compute_coef leaves
 * them. */
#define AP_GR_D1 0
#define AP_GR_D2 1
#define AP_GR_D3 2
#define AP_GR_ALPHA 3
#define AP_GR_THETA 4
#define AP_GR_K1 5
#define AP_GR_K1_J 6
#define AP_GR_J0 7
#define AP_GR_AGRR 8
#define AP_GR_AGRF 9
#define AP_GR_RHO0 10
#define AP_GR_GAMMA_RR 11
#define AP_GR_GAMMA_FF 12
#define AP_GR_BETA_PHI 13
#define AP_GR_B3B1 14
#define AP_GR_NCOEF 15
AP_API int ap_ctx_create_1dgr(const ap_mesh *mesh, const ap_params *params,
                              const ap_gr_params *gr, const ap_gr_table *table, ap_ctx **out);
/* Device array of one coefficient (which = AP_GR_*). */
AP_API int ap_gr_coef(ap_ctx *ctx, int which, ap_array *out);

/* ---------------------------------------------------------------------
 * Batched mode (new; the reference runs one simulation per process).
 * A batch advances many independent 2D Cartesian runs, each an ordinary
 * context with bound fields and particles, with ONE persistent
 * push / deposit launch per tile shape over all runs' tiles, the small
 * per-run kernels enqueued on one stream, and no host synchronisation
 * between steps. Every run gives the same particles, bit for bit, as when
 * it is advanced alone through ap_update_particles. Runs may be 1D or 2D
 * Cartesian and each has its own time step and step counter. The batch
 * takes over the runs' streams and sets them asynchronous (ap_set_sync 0). */
typedef struct ap_batch ap_batch;

AP_API int ap_batch_create(ap_ctx *const *runs, int nruns, ap_batch **out);
/* Destroy a batch before its runs; the runs go back to synchronous calls
 * on the default stream. */
AP_API int ap_batch_destroy(ap_batch *batch);
/* Adds a run to / removes a run from a batch (continuous batching: runs join
 * and leave between steps); a removed run goes back to synchronous calls on
 * the default stream. ap_batch_create accepts nruns == 0. */
AP_API int ap_batch_add(ap_batch *batch, ap_ctx *run);
AP_API int ap_batch_remove(ap_batch *batch, ap_ctx *run);
AP_API int ap_batch_size(const ap_batch *batch, int *nruns);
/* Stream of the batch (default: a private non-blocking stream). */
AP_API int ap_batch_set_stream(ap_batch *batch, void *cuda_stream);
/* ap_update_particles for every run: dt[r] and steps[r] are the time step
 * and step number of run r. */
AP_API int ap_batch_update_particles(ap_batch *batch, const double *dt,
                                     const uint32_t *steps);
/* ap_update_fields for every run, dt and steps as above. */
AP_API int ap_batch_update_fields(ap_batch *batch, const double *dt, const uint32_t *steps);
/* ap_sort_by_cell for every run. */
AP_API int ap_batch_sort_by_cell(ap_batch *batch);
/* Waits for the batch and returns the first non-OK device status of a run
 * (run index in *failed_run, -1 if none; may be NULL). */
AP_API int ap_batch_sync(ap_batch *batch, int *failed_run);
/* nsteps steps of the lab loop for every run without returning between
 * steps (new; the loop of labs/box/src/main.cpp:69-92 and
 * labs/1dgap/src/main.cpp:61-98 over a batch): step s calls
 * ap_batch_update_particles, ap_batch_update_fields and, when inject is
 * nonzero, ap_batch_inject_pairs with run r at step steps0[r] + s, then
 * sorts each run whose step is a positive multiple of sort_interval (0:
 * never). Exactly the calls a caller would make step by step, so every run
 * computes the same; what it saves is the caller's per-step work on the
 * host. Nothing waits for the device unless a 2D run sorts. */
AP_API int ap_batch_advance(ap_batch *batch, const double *dt, const uint32_t *steps0,
                            int nsteps, int sort_interval, int inject);
/* Graph capture. While on, every batched call stages its launch
 * descriptors in host / device blocks of its own, kept until the mode is
 * turned off, and waits for nothing on the host, so that a sequence of
 * ap_batch_update_particles / _update_fields / _inject_pairs calls can be
 * captured into a CUDA graph on the batch's stream (stream capture in
 * relaxed mode; the first step after adding runs or changing tile shapes
 * allocates, so run it before capturing) and the graph replayed. The host
 * side of the captured calls runs once, at capture: a replay repeats those
 * steps' parameters, so capture whole cycles (an even number of steps;
 * compaction intervals and charge-deposition steps that repeat). Turning
 * the mode off (after the graphs are destroyed) frees the blocks. */
AP_API int ap_batch_set_capture(ap_batch *batch, int on);
/* Project autotuner: advances the batch by *steps_used complete steps
 * (particle update, then field update; 5 per candidate) starting at
 * steps[r], timing the push / deposit of each class of runs (same grid
 * size) over the last three steps of each candidate -- every tile shape
 * (16x16, 32x16, 16x8, 8x8, 4x4) with 256-particle chunks, and 16x16 and
 * 32x16 with 512-particle chunks -- and keeps the fastest per class.
 * Particle results do not depend on the shape or chunk; J can differ in
 * the last bits (the fixed-point scale follows the largest tile
 * population). */
AP_API int ap_batch_autotune(ap_batch *batch, const double *dt, const uint32_t *steps,
                             int *steps_used);
/* Tile shape of one run (16x16, 32x16, 16x8, 8x8 or 4x4); rebuilds its
 * tile order at the next update. */
AP_API int ap_set_tile_shape(ap_ctx *ctx, int tx, int ty);
AP_API int ap_get_tile_shape(const ap_ctx *ctx, int *tx, int *ty);

/* ---------------------------------------------------------------------
 * Pair injection (the served 1D gap runs; the reference's analogue is
 * radiative_transfer::produce_pairs, src/cuda/radiation/
 * radiative_transfer.cu:99-177, 252-301, and the 1D gap lab's
 * produce_pair, labs/1dgap/src/cuda/radiation/user_radiative_functions.cuh:
 * 80-131). A live particle with gamma > gamma_thr travels ds = |v| dt per
 * step and emits with probability 1 - exp(-ds / free_path), the uniform
 * number drawn from Philox4x32-10 keyed on (seed) with counter (step,
 * particle id); the photon energy pair_energy leaves the parent (its
 * momentum is rescaled to gamma - pair_energy) and becomes an e-/e+ pair at
 * the parent's position, each member with p1 = sgn(p1_parent) *
 * sqrt(pair_energy^2 / 4 - 1), the parent's weight and the secondary flag.
 * New particles are appended after the live slots in slot order of their
 * parents; ids are first_id, first_id + 1, ... in that order. Emissions
 * beyond the particle capacity are dropped (counted). */
typedef struct {
  float gamma_thr;     /* 1e6 in the served workload                      */
  float free_path;     /* mean free path, in the units of x (0.05)        */
  float pair_energy;   /* photon energy converted into one pair           */
  int enabled;
  uint64_t seed;       /* per-run key of the random stream                */
  uint64_t first_id;   /* id given to the next created particle           */
} ap_pair_params;

/* Enables (or changes) pair injection. From then on the context keeps its
 * live particle count on the device: the 1D update, the injection and the
 * 1D sort read and write it there without host synchronisation, and calls
 * that report the count (ap_get_number, ap_sync, ...) read it back. */
AP_API int ap_set_pair_params(ap_ctx *ctx, const ap_pair_params *params);
/* Running totals since ap_set_pair_params: particle-steps (live slots summed
 * over injection passes), pairs created, pairs dropped over capacity
 * (waits for the stream). */
AP_API int ap_get_pair_stats(ap_ctx *ctx, uint64_t *particle_steps, uint64_t *emitted_total,
                             uint64_t *dropped_total);
/* One injection pass over the live particles (after the particle update of
 * `step`, with that step's dt); waits for the stream. *emitted (may be
 * NULL) receives the number of pairs created; *dropped (may be NULL) those
 * over capacity. */
AP_API int ap_inject_pairs(ap_ctx *ctx, double dt, uint32_t step, uint64_t *emitted,
                           uint64_t *dropped);
/* The same for every run of a batch that has pair injection enabled (dt[r]
 * and steps[r] per run). 1D runs are served by three batched launches and
 * no host synchronisation: their counts stay on the device until
 * ap_get_number or another call that needs them reads them back. */
AP_API int ap_batch_inject_pairs(ap_batch *batch, const double *dt, const uint32_t *steps);

/* ---------------------------------------------------------------------
 * Photons and pair production: radiative_transfer (src/radiation/
 * radiative_transfer.h:11-29, src/cuda/radiation/radiative_transfer.cu)
 * with the user radiative functions of the framework
 * (src/cuda/radiation/user_radiative_functions.cu, AP_RAD_DEFAULT), of
 * the pulsar lab (labs/pulsar/src/cuda/radiation/
 * user_radiative_functions.cu, AP_RAD_PULSAR), of the 1D GR lab
 * (labs/1dgr/src/cuda/radiation/user_radiative_functions.cuh, AP_RAD_GR1D)
 * or of the 1D gap lab (labs/1dgap/.../user_radiative_functions.cuh,
 * AP_RAD_GAP1D) -- the last two sample inverse-Compton emission and
 * gamma-gamma conversion from the tables of ap_ic_init -- and the photon
 * movers of the particle updaters (ptc_updater.cu:627-690,
 * ptc_updater_logsph.cu:58-131, ptc_updater_1dgr.cu:301-400,
 * ptc_updater_1dgap.cu:163-192), which ap_update_particles runs after the
 * particles when photons are bound, followed by the exchange: photons
 * leaving the bulk wrap through periodic sides (Cartesian) or are removed
 * (the 1D GR and gap movers remove photons outside the bulk before moving
 * them, as the reference's do).
 *
 * Each pass ranks its emitters in slot order and appends: photon k of an
 * emit_photons call at slot number + k (the photon count then grows by the
 * emitters + 1, the reference's padding), pair k of a produce_pairs call at
 * particle slots number + 20 + 2k and + 1 (the count grows by 2 x the
 * converted photons + 50). Random numbers: each particle (photon) draws
 * four uniforms in (0, 1] from Philox4x32-10 keyed on `seed` with counter
 * (call, id, 1) for emission (2 for conversion), call counting the passes
 * of its kind since ap_set_rad_params (the reference draws cuRAND XORWOW in
 * thread order). Every new photon and particle gets an id (photons from
 * first_photon_id, particles from first_particle_id, in rank order); the
 * tracked flag keeps the reference's meaning (a draw below track_percent).
 * An emission past the photon capacity leaves its parent unchanged and a
 * pair whose second slot is past the particle capacity removes its photon;
 * both are counted as dropped. Empty slots that a pass leaves in its range
 * (a photon the model does not keep) have cell = MAX_CELL. */
#define AP_RAD_DEFAULT 0
#define AP_RAD_PULSAR 1
#define AP_RAD_GR1D 2
#define AP_RAD_GAP1D 3
typedef struct {
  float *x1, *x2, *x3;
  float *p1, *p2, *p3;
  float *E, *weight, *path_left;
  uint32_t *cell;
  uint64_t *id;
  uint32_t *flag;
} ap_photons; /* photon_data (src/data/particle_data.h:68-80) */
typedef struct {
  int model;            /* AP_RAD_DEFAULT or AP_RAD_PULSAR                 */
  float delta_t;        /* SimParams::delta_t (the pulsar emission rate)   */
  float gamma_thr;      /* default model: emission threshold               */
  float E_secondary;    /* default model: photon energy scale              */
  float photon_path;    /* default model: free path scale                  */
  float r_cutoff;       /* default: longest path; log-spherical mover:
                           photons beyond this radius are removed          */
  float track_percent;  /* fraction of new photons / pairs flagged tracked */
  float e_curv, l_curv; /* pulsar model: curvature photon energy and rate  */
  float BQ;             /* pulsar model: critical field                    */
  float omega;          /* pulsar model: emission only inside 0.6 / omega  */
  uint64_t seed;
  uint64_t first_photon_id;
  uint64_t first_particle_id;
  /* AP_RAD_GR1D and AP_RAD_GAP1D (user_rt_init of either lab, e.g.
     labs/1dgr/src/cuda/radiation/user_radiative_functions.cuh:191-203):
     tables of n_gamma x n_ep entries for the background
     broken_power_law(1.25, 1.1, e_min, 1e-10, 0.1) with photon density
     1.5e24 / ic_path; the gap lab keeps photons above 0.001 / e_min; the
     spin and omega are the 1D GR context's (ap_gr_params).                  */
  float e_min;          /* SimParams::e_min (default 1e-3)                 */
  float ic_path;        /* SimParams::ic_path (default 1)                  */
  int n_gamma, n_ep;    /* SimParams::n_gamma, n_ep (default 600, 600)     */
} ap_rad_params;
typedef struct {
  uint64_t marked;   /* particles (photons) that passed the model's check  */
  uint64_t written;  /* appended within the capacity                      */
  uint64_t dropped;  /* over the capacity                                 */
} ap_rad_counts;

/* Background photon spectra of inverse_compton::init (src/radiation/
 * spectra.h); p[] holds the constructor's arguments in order. */
#define AP_SPEC_POWER_LAW_HARD 0   /* delta, emin, emax                 */
#define AP_SPEC_POWER_LAW_SOFT 1   /* alpha, emin, emax                 */
#define AP_SPEC_BROKEN_POWER_LAW 2 /* alpha, delta, epeak, emin, emax   */
#define AP_SPEC_BLACK_BODY 3       /* kT                                */
#define AP_SPEC_MONO_ENERGETIC 4   /* e0, de                            */
typedef struct {
  int kind;
  float p[5];
} ap_spectrum;

/* inverse_compton's constructor and init(n_e, emin, emax, n0)
 * (src/cuda/radiation/rt_ic.cu:207-435): for n_gamma Lorentz factors
 * log-spaced over [1.01, 1e15], the scattering rate and the gamma-gamma
 * pair rate in the background n0 * n_e, and the cumulative, normalised
 * distributions of the scattered photon energy over n_ep linear (dNde) and
 * n_ep log-spaced (dNde_thomson) fractions of gamma. The reference
 * integrates on the host (100 angles x 800 energies per entry, one entry
 * after the other); here one GPU pass per table, with the same integrands
 * in double and the same float rounding of the stored values and of the
 * cumulative sums. The tables stay on the device for AP_RAD_GR1D. */
AP_API int ap_ic_init(ap_ctx *ctx, const ap_spectrum *spectrum, double emin, double emax,
                      double n0, int n_gamma, int n_ep);
/* Copies the tables to host arrays (each may be NULL): ic_rate, gg_rate,
 * gammas of n_gamma floats; dNde, dNde_thomson of n_gamma x n_ep floats,
 * row n for gammas[n]; steps = {dep, dg, dlep}. */
AP_API int ap_ic_tables(ap_ctx *ctx, float *ic_rate, float *gg_rate, float *gammas,
                        float *dNde, float *dNde_thomson, float *steps);

/* Binds caller-owned photon arrays of `capacity` slots, `number` in use. */
AP_API int ap_bind_photons(ap_ctx *ctx, const ap_photons *ph, size_t number, size_t capacity);
AP_API int ap_get_photon_number(const ap_ctx *ctx, size_t *number);
/* Sets the model and its parameters; resets the pass counters. */
AP_API int ap_set_rad_params(ap_ctx *ctx, const ap_rad_params *params);
/* radiative_transfer::emit_photons (radiative_transfer.cu:196-243):
 * particles in the bulk (ions excepted) that pass check_emit_photon emit
 * one photon each; photon_produced (ptr may be NULL; a 2D field array)
 * accumulates their weights per cell. Waits for the stream. */
AP_API int ap_emit_photons(ap_ctx *ctx, ap_array photon_produced, ap_rad_counts *out);
/* radiative_transfer::produce_pairs (radiative_transfer.cu:245-301):
 * photons in the bulk that pass check_produce_pair become an e-/e+ pair;
 * pair_produced (ptr may be NULL) accumulates their weights per cell.
 * Waits for the stream. */
AP_API int ap_produce_pairs(ap_ctx *ctx, ap_array pair_produced, ap_rad_counts *out);
/* The photon move of one update (also run by ap_update_particles when
 * photons are bound; the 1D GR mover records the lower u_0 of tracked
 * photons as on step 0 when called here). */
AP_API int ap_move_photons(ap_ctx *ctx, double dt);

/* Device time per phase of the update, from CUDA events recorded on the
 * context's stream around each phase while profiling is on. */
typedef struct {
  double push_deposit_ms; /* fused push + deposit kernel                  */
  double order_ms;        /* per-step tile counting sort (scan + scatter) */
  double rebuild_ms;      /* full tile-order rebuild                      */
  double finalize_ms;     /* current/charge zeroing, fold and rounding    */
  double fields_ms;       /* Yee update of E and B and divergences        */
  double sort_ms;         /* sort_by_cell                                 */
  uint64_t push_deposit_launches;
} ap_phase_times;

/* Turns per-phase event timing on (1) or off (0); new for measurement. */
AP_API int ap_set_profiling(ap_ctx *ctx, int on);
/* Sums the recorded phase times (waits for the stream); reset != 0 clears
 * them afterwards. */
AP_API int ap_get_phase_times(ap_ctx *ctx, ap_phase_times *out, int reset);

/* Limits of ap_update_particles_1d_noalloc. */
#define AP_NOALLOC_MAX_CELLS 16392   /* dims[0], guard cells included */
#define AP_NOALLOC_MAX_SPECIES 3

/* No counterpart in the reference. The 1D particle update of
 * ap_update_particles (push, deposit, periodic fold, rounding of J and Rho,
 * wrap) for callers that cannot allocate device memory when they call it --
 * for example a process whose device memory is fully reserved by another
 * allocator, where a cudaMalloc would fail or fragment that pool. It needs
 * no context and allocates nothing: the caller passes the particle and
 * field arrays, and the library's only other device memory is a fixed
 * file-scope array of (3 + AP_NOALLOC_MAX_SPECIES) * AP_NOALLOC_MAX_CELLS
 * 64-bit words (about 770 KB), which every GPU that loads the library holds
 * until the process exits. Grids with more than AP_NOALLOC_MAX_CELLS cells
 * (AP_ERR_CAPACITY), more than AP_NOALLOC_MAX_SPECIES species
 * (AP_ERR_CAPACITY), current smoothing (AP_ERR_UNSUPPORTED) or other than
 * 1D (AP_ERR_UNSUPPORTED) are rejected. The first call in each CUDA
 * context (normally once per device: the device's primary context) looks
 * up the array's device address with cudaGetSymbolAddress and caches it
 * under that context's id, so make that first call before any stream
 * capture; a context that is destroyed and re-created is looked up afresh.
 * All calls share the array and clear it at their start: calls that
 * overlap on the GPU (on different streams, or from different threads)
 * race and must not be issued. The call enqueues its work on cuda_stream
 * (0 = legacy default stream) and synchronises that stream before
 * returning, also when it fails after enqueueing work. */
AP_API int ap_update_particles_1d_noalloc(const ap_mesh *mesh, const ap_params *params,
                                          const ap_particles *ptc, size_t number,
                                          const ap_fields *fields, double dt,
                                          uint32_t step, void *cuda_stream);

/* Status of the last failing call on this context. */
AP_API int ap_last_error(const ap_ctx *ctx);

/* Number of kernels this context has launched (for launch accounting). */
AP_API uint64_t ap_launch_count(const ap_ctx *ctx);

#ifdef __cplusplus
}
#endif

#endif /* APERTURE_B200_H_ */

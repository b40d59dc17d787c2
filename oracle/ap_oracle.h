/*
 * CPU oracle for the Aperture3 particle update (TEST INFRASTRUCTURE ONLY).
 *
 * This is a plain-C restatement of the reference algorithm, used by the
 * tests, by __graft_entry__.smoke() and by the cpu_baseline leg of bench.py
 * as the checker. The product library never links, loads or calls it.
 *
 * Arithmetic is FP32 literal: every expression keeps the operation order of
 * the reference kernels and the file is compiled with -ffp-contract=off, so
 * each result is the correctly rounded IEEE value of the same expression
 * sequence the reference evaluates. Current and charge can also be
 * accumulated in FP64 (the *_f64 deposit variants) to state the FP32
 * summation error.
 *
 * Parity pin: oracle/ref_build compiles the reference's own kernel bodies
 * (src/cuda/algorithms/ptc_updater.cu, field_solver.cu) as host C++ behind a
 * shim of the CUDA built-ins; tests/test_oracle_pin.py checks this file
 * against that build and against the committed fixtures in tests/golden/.
 *
 * Field arrays are row-major without padding: element (i, j) of a 2D array
 * lives at [i + j * dims[0]]; 1D arrays have dims[1] == 1.
 */
#ifndef AP_ORACLE_H_
#define AP_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_MAX_CELL 0xFFFFFFFFu

/* Mirrors Quadmesh (src/core/quadmesh.h:16-29). */
typedef struct {
  int dims[3];
  int guard[3];
  float delta[3];
  float inv_delta[3];
  float lower[3];
  float sizes[3];
  int dimension;
} or_mesh;

/* Mirrors particle_data (src/data/particle_data.h:50-61). */
typedef struct {
  float *x1, *x2, *x3;
  float *p1, *p2, *p3;
  float *E, *weight;
  uint32_t *cell;
  uint64_t *id;
  uint32_t *flag;
} or_ptc;

/* Field pointers in the reference's component order. */
typedef struct {
  float *E[3], *B[3], *Ebg[3], *Bbg[3], *J[3];
  float *Rho[8];
  float *divE, *divB;
} or_fields;

/* Push (ptc_updater.cu:21-76 for 1D, :78-141 for 2D). Returns the number
 * of particles whose momentum was NaN on entry (the reference traps). */
uint64_t or_push_cart_1d(const or_mesh *m, or_ptc *p, size_t num, float dt,
                         float *const F[6], const float charges[8],
                         const float masses[8]);
uint64_t or_push_cart_2d(const or_mesh *m, or_ptc *p, size_t num, float dt,
                         float *const F[6], const float charges[8],
                         const float masses[8]);

/* Deposit + move (ptc_updater.cu:220-293 for 1D, :295-386 for 2D).
 * Rho[sp] is written only when (step + 1) % data_interval == 0.
 * Returns the number of particles that moved more than one cell. */
uint64_t or_deposit_cart_1d(const or_mesh *m, or_ptc *p, size_t num, float dt,
                            uint32_t step, int data_interval,
                            float *const J[3], float *const Rho[8],
                            const float charges[8]);
uint64_t or_deposit_cart_2d(const or_mesh *m, or_ptc *p, size_t num, float dt,
                            uint32_t step, int data_interval,
                            float *const J[3], float *const Rho[8],
                            const float charges[8]);
/* Same arithmetic with FP64 accumulators. */
uint64_t or_deposit_cart_1d_f64(const or_mesh *m, or_ptc *p, size_t num,
                                float dt, uint32_t step, int data_interval,
                                double *const J[3], double *const Rho[8],
                                const float charges[8]);
uint64_t or_deposit_cart_2d_f64(const or_mesh *m, or_ptc *p, size_t num,
                                float dt, uint32_t step, int data_interval,
                                double *const J[3], double *const Rho[8],
                                const float charges[8]);

/* Guard exchange on one rank (sim_environment_impl.hpp:286-305,
 * cuda/sim_environment.cpp:9-127): copy interior strips into the opposite
 * guards / add guard strips into the opposite interior, for every dim whose
 * periodic flag is set (a non-periodic dim has no neighbour on one rank). */
void or_send_guard_cells(const or_mesh *m, float *a, const int periodic[3]);
void or_send_add_guard_cells(const or_mesh *m, float *a, const int periodic[3]);
void or_send_add_guard_cells_f64(const or_mesh *m, double *a,
                                 const int periodic[3]);

/* Particle communication on one rank (sim_environment_impl.hpp:319-412,
 * kernels.cu:95-148, quadmesh.h:264-273). Particles outside the bulk are
 * shifted by -/+ reduced_dim in every dim they left; they are kept when all
 * of those dims are periodic and appended at the end of the array, and
 * their old slot becomes MAX_CELL. Returns the new number (<= cap). */
size_t or_send_particles(const or_mesh *m, or_ptc *p, size_t num, size_t cap,
                         const int periodic[3]);
/* Same per-particle outcome, in place: kept particles get the shifted cell
 * in their own slot, lost ones get MAX_CELL. Returns the number lost. */
uint64_t or_wrap_particles(const or_mesh *m, or_ptc *p, size_t num,
                           const int periodic[3]);

/* Yee FDTD (field_solver.cu:14-84, :133-193, :237-288), bulk cells only. */
void or_update_e_1d(const or_mesh *m, or_fields *f, float dt);
void or_update_b_1d(const or_mesh *m, or_fields *f, float dt);
void or_compute_divs_1d(const or_mesh *m, or_fields *f);
void or_update_e_2d(const or_mesh *m, or_fields *f, float dt);
void or_update_b_2d(const or_mesh *m, or_fields *f, float dt);
void or_compute_divs_2d(const or_mesh *m, or_fields *f);
/* field_solver::update_fields (field_solver.cu:334-358). */
void or_update_fields(const or_mesh *m, or_fields *f, double dt, uint32_t step,
                      const int periodic[3]);

/* Binomial current filter (ptc_updater.cu:501-560), writes tmp (bulk only),
 * then copies the bulk back into j. bnd = {lower0, upper0, lower1, upper1}
 * (true where the dim is not periodic). */
void or_filter_1d(const or_mesh *m, float *j, float *tmp, const int bnd[4]);
void or_filter_2d(const or_mesh *m, float *j, float *tmp, const int bnd[4]);

/* ptc_updater::update_particles (ptc_updater.cu:748-841) on one rank with
 * the in-place particle wrap (or_wrap_particles) instead of hole+append.
 * nthreads > 1 runs push and deposit with OpenMP (private current buffers
 * reduced in thread order). Returns NaN + lost counters packed as
 * (nan << 32) | lost, saturated. */
uint64_t or_update_particles(const or_mesh *m, or_ptc *p, size_t num,
                             or_fields *f, double dt, uint32_t step,
                             int data_interval, int num_species,
                             int current_smoothing, const float charges[8],
                             const float masses[8], const int periodic[3],
                             int nthreads);

/* Stable counting sort (core/particle_base_impl.hpp:250-305): perm[r] is the
 * input index that lands at rank r; keys >= nkeys must not occur. */
void or_stable_counting_sort(const uint32_t *keys, size_t n, uint32_t nkeys,
                             uint32_t *perm);
/* particle_base::sort_by_cell on the CPU (core/particle_base_impl.hpp:
 * 250-332): stable by cell, MAX_CELL last, then trimmed. Returns number. */
size_t or_sort_by_cell(const or_mesh *m, or_ptc *p, size_t num);

/* Tile key of a bulk cell: tiles of tile[0] x tile[1] cells tile the bulk
 * row-major; returns ntiles for MAX_CELL / non-bulk cells. */
uint32_t or_tile_key(const or_mesh *m, const int tile[2], uint32_t cell);
/* One step of the tile order: stable counting sort of the sequence
 * order_in[0..n) by or_tile_key(cell[order_in[r]]), dropping particles
 * whose key is ntiles. Writes order_out and tile_start[ntiles + 1];
 * returns the new length. */
size_t or_tile_order(const or_mesh *m, const int tile[2], const uint32_t *cell,
                     const uint32_t *order_in, size_t n, uint32_t *order_out,
                     uint32_t *tile_start);

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC 2011). */
void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Pair injection of the served 1D gap runs (the library's build semantics;
 * the reference analogue is radiative_transfer::produce_pairs and the 1D
 * gap lab's produce_pair, user_radiative_functions.cuh:80-131): in slot
 * order, a live particle with E > gamma_thr emits with probability
 * 1 - exp(-(|p| / E) dt / free_path), the uniform number being
 * ((out0 >> 8) + 0.5) / 2^24 of Philox4x32-10 with counter (step, id_lo,
 * id_hi, 0) and key (seed_lo, seed_hi); emitter k (k < free slots / 2)
 * loses pair_energy and appends an e- and an e+ at slots num + 2k,
 * num + 2k + 1 with ids first_id + 2k, + 1. Returns the new number;
 * *emitted / *dropped get the counts. */
size_t or_inject_pairs(or_ptc *p, size_t num, size_t cap, float dt, uint32_t step,
                       float gamma_thr, float free_path, float pair_energy,
                       uint64_t seed, uint64_t first_id, uint64_t *emitted,
                       uint64_t *dropped);

/* 1D gap pusher (ptc_updater_1dgap.cu:75-161, the 1dgap lab's
 * update_particles): per live particle in slot order, the E_parallel
 * interpolation from E3 (the smoothed copy of E1), the push with
 * beta_phi(x) = x in the reference's float / double mix, the move, and the
 * deposit of J1 (times delta / dt) and Rho[sp] (every step) with plain
 * float adds in the reference's order (f64 = 1: into double arrays). A
 * particle outside the bulk is emptied (cell = MAX_CELL). Returns the
 * number of moves of more than one cell. */
uint64_t or_update_ptc_1dgap(const or_mesh *m, or_ptc *p, size_t num, float dt,
                             const float *E3, float *J1, float *const Rho[8],
                             const float charges[8], const float masses[8]);
uint64_t or_update_ptc_1dgap_f64(const or_mesh *m, or_ptc *p, size_t num, float dt,
                                 const float *E3, double *J1, double *const Rho[8],
                                 const float charges[8], const float masses[8]);
/* filter_current1d (ptc_updater_1dgap.cu:196-213): one 1-2-1 pass over all
 * cells [0, dims0) from j into tmp, with the end cells of the bulk clamped
 * on boundary sides (bnd[0] lower, bnd[1] upper); a neighbour outside the
 * array (the reference reads past the row there) counts as 0. */
void or_filter_gap(const or_mesh *m, const float *j, float *tmp, const int bnd[2]);
/* ptc_updater_1dgap::update_particles (ptc_updater_1dgap.cu:219-272):
 * E3 = E1, smoothed `smoothing` times through E2; J1 and Rho zeroed; the
 * push / deposit; then J1 and each Rho smoothed `smoothing` times through
 * tmp. Returns the number of moves of more than one cell. */
uint64_t or_update_particles_1dgap(const or_mesh *m, or_ptc *p, size_t num, or_fields *f,
                                   float dt, int smoothing, int num_species,
                                   const float charges[8], const float masses[8],
                                   const int bnd[2]);
/* field_solver_1dgap::update_fields (field_solver_1dgap.cu:14-40):
 * E1 += (j0 - J1) dt on cells [guard + 1, dims0 - guard - 1), j0 = B0 1.6. */
void or_update_fields_1dgap(const or_mesh *m, float *E1, const float *J1, float B0, float dt);

/* ptc_updater_logsph::inject_ptc (ptc_updater_logsph.cu:301-393 inject_ptc,
 * 441-490 measure_surface_density, 849-870) with the library's build
 * semantics: the surface densities of electrons and ions in the cells
 * guard0 + 1 .. guard0 + 4 (1-4-6-4-1 spread over theta rows, w / 3 / 16
 * each, summed in double); for every theta row i in [guard1 + 1,
 * dims1 - guard1 - 1) whose max density times q_e stays below
 * 1.5 sin(theta_c) / dtheta^2, inj e-/e+ pairs at cell (guard0 + 2, i):
 * x1 = 0.5, x2 = ((out0 >> 8) + 0.5) / 2^24 of Philox4x32-10 with counter
 * (call, i, n, 0) and key (seed), p1' = p1 2 |cos th|, p2' = p1 sin th
 * sgn(cos th), p3 = 0, E = sqrt(1 + p1^2), weight w sin th, flag primary.
 * Pair n of bulk row r = i - guard1 takes slots num + 2 (r inj + n) and
 * + 1 (ids first_id + the same offsets); the slots of rows without
 * injection are empty. Returns num + 2 inj (dims1 - 2 guard1), or num when
 * that exceeds cap. */
size_t or_ls_inject(const or_mesh *m, or_ptc *p, size_t num, size_t cap, int inj, float p1,
                    float w, float q_e, uint64_t seed, uint32_t call, uint64_t first_id);
/* measure_surface_density (ptc_updater_logsph.cu:441-490) summed in double:
 * se / sp get dims1 - 2 guard1 values (electrons, ions). */
void or_ls_surface_density(const or_mesh *m, const or_ptc *p, size_t num, double *se,
                           double *sp);

#ifdef __cplusplus
}
#endif

#endif /* AP_ORACLE_H_ */

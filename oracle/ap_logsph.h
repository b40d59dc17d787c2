/*
 * CPU oracle for the log-spherical (ln r, theta) particle update and field
 * solver (TEST INFRASTRUCTURE ONLY; the product never links or calls it).
 *
 * ap_logsph.c is compiled twice into liboracle.so:
 *   *_f32  FP32-literal restatement: the expression order and the mixed
 *          float / double types of the reference, with the C library's float
 *          transcendentals (expf, sinf, ...). Pinned bit for bit against the
 *          reference's own kernel bodies run on the host (oracle/ref_build).
 *   *_f64  the same algorithm with every quantity in FP64 (positions
 *          included): the truth that FP32 results state their error against.
 *
 * Reference sources restated:
 *   src/grids/grid_log_sph.cpp:11-126, grid_log_sph.h:23-38   (coefficients)
 *   src/cuda/algorithms/user_push_2d_logsph.cuh:14-114          (push)
 *   src/cuda/algorithms/gravity.cuh:12-26, sync_cooling.cuh:59-86
 *   src/cuda/algorithms/ptc_updater_logsph.cu:26-44             (basis change)
 *   src/cuda/algorithms/ptc_updater_logsph.cu:134-299,414-438,440-455,
 *                                              616-666,681-836 (deposit,
 *                                              process_j, axis, outflow,
 *                                              filter, orchestration)
 *   src/cuda/algorithms/field_solver_logsph.cu:16-345,354-428  (fields)
 *
 * Arrays are row-major without padding, element (i, j) at [i + j * dims[0]].
 */
#ifndef AP_LOGSPH_ORACLE_H_
#define AP_LOGSPH_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#include "ap_oracle.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Physics parameters the log-spherical kernels read from dev_params. */
typedef struct {
  float compactness;      /* r_g / R_*, enters beta_phi and omega_LT */
  float omega;            /* dev_params.omega (beta_phi uses this one) */
  float gravity;          /* artificial gravity strength */
  float rad_cooling_coef;
  float B0;
  float damping_coef;
  int rad_cooling_on;
  int damping_length;
} or_ls_params;

/* Coefficient array order (Grid_LogSph members). */
enum {
  OR_L1E = 0, OR_L2E, OR_L3E, OR_L1B, OR_L2B, OR_L3B,
  OR_A1E, OR_A2E, OR_A3E, OR_A1B, OR_A2B, OR_A3B, OR_DV, OR_NCOEF
};

/* FP64 particle record (positions in FP64 too). */
typedef struct {
  double *x1, *x2, *x3;
  double *p1, *p2, *p3;
  double *E, *weight;
  uint32_t *cell;
  uint64_t *id;
  uint32_t *flag;
} or_ptc_d;

typedef struct {
  double *E[3], *B[3], *Ebg[3], *Bbg[3], *J[3];
  double *Rho[8];
  double *divE, *divB;
} or_fields_d;

/* ---- FP32-literal ---- */
void or_ls_coef_f32(const or_mesh *m, float *const c[OR_NCOEF]);
uint64_t or_ls_push_f32(const or_mesh *m, const or_ls_params *lp, or_ptc *p,
                        size_t num, float dt, float *const F[6],
                        const float charges[8], const float masses[8]);
/* J / Rho are float arrays (acc64 = 0) or double accumulators (acc64 = 1);
 * the contributions are FP32 either way. Returns |dc| > 1 count. */
uint64_t or_ls_deposit_f32(const or_mesh *m, const or_ls_params *lp,
                           or_ptc *p, size_t num, float dt, uint32_t step,
                           int data_interval, void *const J[3],
                           void *const Rho[8], int acc64, const float *dV,
                           const float charges[8]);
void or_ls_process_j_f32(const or_mesh *m, float *const J[3],
                         float *const Rho[8], int num_species,
                         const float *A1e, const float *A2e, const float *dV,
                         float dt);
void or_ls_axis_rho_f32(const or_mesh *m, float *J3);
void or_ls_ptc_outflow_f32(const or_mesh *m, const or_ls_params *lp,
                           or_ptc *p, size_t num);
void or_ls_filter_f32(const or_mesh *m, float *j, float *tmp, const float *A,
                      const int bnd[4]);
void or_ls_update_b_f32(const or_mesh *m, const or_ls_params *lp,
                        or_fields *f, float *const c[OR_NCOEF], float dt);
void or_ls_update_e_f32(const or_mesh *m, const or_ls_params *lp,
                        or_fields *f, float *const c[OR_NCOEF], float dt);
void or_ls_divs_f32(const or_mesh *m, or_fields *f, float *const c[OR_NCOEF]);
void or_ls_field_boundary_f32(const or_mesh *m, const or_ls_params *lp,
                              or_fields *f, float omega);
/* ptc_updater_logsph::update_particles (+ apply_boundary) on one rank,
 * non-periodic: particles leaving the bulk get MAX_CELL in place.
 * Returns (nan << 32) | lost, saturated. acc64 selects FP64 current sums,
 * rounded to FP32 before process_j. */
uint64_t or_ls_update_particles_f32(const or_mesh *m, const or_ls_params *lp,
                                    or_ptc *p, size_t num, or_fields *f,
                                    float *const c[OR_NCOEF], double dt,
                                    uint32_t step, int data_interval,
                                    int num_species, int current_smoothing,
                                    const float charges[8],
                                    const float masses[8], int acc64);
/* field_solver_logsph::update_fields: B, then E, then divE / divB. */
void or_ls_update_fields_f32(const or_mesh *m, const or_ls_params *lp,
                             or_fields *f, float *const c[OR_NCOEF], double dt);

/* ---- FP64 ---- */
void or_ls_coef_f64(const or_mesh *m, double *const c[OR_NCOEF]);
uint64_t or_ls_update_particles_f64(const or_mesh *m, const or_ls_params *lp,
                                    or_ptc_d *p, size_t num, or_fields_d *f,
                                    double *const c[OR_NCOEF], double dt,
                                    uint32_t step, int data_interval,
                                    int num_species, int current_smoothing,
                                    const float charges[8],
                                    const float masses[8], int acc64);
void or_ls_update_fields_f64(const or_mesh *m, const or_ls_params *lp,
                             or_fields_d *f, double *const c[OR_NCOEF],
                             double dt);
void or_ls_field_boundary_f64(const or_mesh *m, const or_ls_params *lp,
                              or_fields_d *f, float omega);

#ifdef __cplusplus
}
#endif

#endif /* AP_LOGSPH_ORACLE_H_ */

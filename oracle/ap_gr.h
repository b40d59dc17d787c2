/*
 * CPU oracle, 1D GR lab (TEST INFRASTRUCTURE ONLY); see ap_gr.c for the
 * reference lines each function restates. Arrays are 1D of dims[0] floats.
 */
#ifndef AP_GR_H_
#define AP_GR_H_

#include "ap_oracle.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Coefficient arrays of Grid_1dGR, in the order of its mesh_ptrs
 * (src/grids/grid_1dgr.h:16-20). THETA and AGRF stay zero, as
 * compute_coef leaves them. */
enum {
  OR_GR_D1, OR_GR_D2, OR_GR_D3, OR_GR_ALPHA, OR_GR_THETA, OR_GR_K1, OR_GR_K1_J, OR_GR_J0,
  OR_GR_AGRR, OR_GR_AGRF, OR_GR_RHO0, OR_GR_GAMMA_RR, OR_GR_GAMMA_FF, OR_GR_BETA_PHI,
  OR_GR_B3B1, OR_GR_NCOEF
};

/* Grid_1dGR::compute_coef (grid_1dgr.cpp:21-187) from the seven tabulated
 * arrays of length ntab the reference reads from coef.h5. */
void or_gr_coef(const or_mesh *m, float a, float omega, float B0, const float *v_r,
                const float *v_B1, const float *v_B3, const float *v_jr, const float *v_rho,
                const float *v_theta, const float *v_dpsidth, size_t ntab,
                float *const co[OR_GR_NCOEF]);
/* update_ptc_1dgr (ptc_updater_1dgr.cu:137-300) over slots [0, num) in
 * order; float adds into J1 / Rho (the reference's atomics in slot order),
 * or double adds of the same float contributions (_f64). Returns the number
 * of moves of more than one cell. */
uint64_t or_update_ptc_1dgr(const or_mesh *m, or_ptc *p, size_t num, float dt, uint32_t step,
                            int data_interval, float a, float omega, const float *E3,
                            const float *const co[OR_GR_NCOEF], float *J1, float *const Rho[8],
                            const float charges[8], const float masses[8]);
uint64_t or_update_ptc_1dgr_f64(const or_mesh *m, or_ptc *p, size_t num, float dt,
                                uint32_t step, int data_interval, float a, float omega,
                                const float *E3, const float *const co[OR_GR_NCOEF], double *J1,
                                double *const Rho[8], const float charges[8],
                                const float masses[8]);
/* filter_current1d of the GR lab (ptc_updater_1dgr.cu:388-404). */
void or_filter_gr(const or_mesh *m, const float *j, float *tmp, const float *k1,
                  const int bnd[2]);
/* ptc_updater_1dgr::update_particles (ptc_updater_1dgr.cu:418-473). */
uint64_t or_update_particles_1dgr(const or_mesh *m, or_ptc *p, size_t num, or_fields *f,
                                  float dt, uint32_t step, int data_interval, int smoothing,
                                  int num_species, float a, float omega,
                                  const float *const co[OR_GR_NCOEF], const float charges[8],
                                  const float masses[8], const int bnd[2]);
/* update_e_1dgr (field_solver_1dgr.cu:14-24). */
void or_update_e_1dgr(const or_mesh *m, float *E1, const float *J1, const float *j0, float dt);

#ifdef __cplusplus
}
#endif

#endif /* AP_GR_H_ */

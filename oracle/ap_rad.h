/*
 * CPU oracle, photons and pair production (TEST INFRASTRUCTURE ONLY); see
 * ap_rad.c for the reference lines each function restates. 2D arrays are
 * row-major without padding, as in ap_oracle.h.
 */
#ifndef AP_RAD_H_
#define AP_RAD_H_

#include "ap_ic.h"
#include "ap_oracle.h"

#ifdef __cplusplus
extern "C" {
#endif

/* photon_data (src/data/particle_data.h:68-80). */
typedef struct {
  float *x1, *x2, *x3;
  float *p1, *p2, *p3;
  float *E, *weight, *path_left;
  uint32_t *cell;
  uint64_t *id;
  uint32_t *flag;
} or_photons;

/* The emission / conversion models: the framework's default
 * (src/cuda/radiation/user_radiative_functions.cu), the pulsar lab's
 * (labs/pulsar/src/cuda/radiation/user_radiative_functions.cu), the 1D GR
 * lab's (labs/1dgr/src/cuda/radiation/user_radiative_functions.cuh) and the
 * 1D gap lab's (labs/1dgap/src/cuda/radiation/user_radiative_functions.cuh;
 * of or_rad_gr it reads only the tables). */
enum { OR_RAD_DEFAULT = 0, OR_RAD_PULSAR = 1, OR_RAD_GR1D = 2, OR_RAD_GAP1D = 3 };

/* What the 1D GR lab's functions read besides SimParams: Grid_1dGR's
 * per-cell arrays (grid_1dgr.h mesh_ptrs), the spin a, omega, and the
 * inverse-Compton tables. */
typedef struct {
  const float *alpha, *D1, *D2, *D3, *B3B1, *gamma_rr, *gamma_ff, *beta_phi, *theta;
  float a, omega;
  const or_ic_tables *ic;
} or_rad_gr;

/* The SimParams members the radiation functions read (src/sim_params.h:
 * 17-123), the random key and the id counters. */
typedef struct {
  int model;
  float delta_t, gamma_thr, E_secondary, photon_path, r_cutoff, track_percent;
  float e_curv, l_curv, BQ, omega;
  uint64_t seed;
  const or_rad_gr *gr; /* OR_RAD_GR1D, OR_RAD_GAP1D */
  float e_min;         /* OR_RAD_GAP1D: photons below 0.001 / e_min not kept */
} or_rad_params;

/* Counts of one emission or conversion pass. */
typedef struct {
  uint64_t marked;   /* particles (photons) that passed the check          */
  uint64_t written;  /* of those, appended within the capacity             */
  uint64_t dropped;  /* over the capacity (parent / photon left unchanged /
                        photon removed)                                    */
} or_rad_counts;

/* The four uniforms in (0, 1] of one particle (tag 1) or photon (tag 2)
 * for pass `call`: Philox4x32-10 keyed on the seed, counter (call, id,
 * tag). */
void or_rad_uniforms(uint64_t seed, uint32_t tag, uint32_t call, uint64_t id, float u[4]);

/* move_photons_cart_1d / _2d (src/cuda/algorithms/ptc_updater.cu:627-690)
 * followed by send_particles (sim_environment_impl.hpp:319-448): photons
 * leaving the bulk are wrapped through periodic sides or removed. */
void or_move_photons_cart(const or_mesh *m, or_photons *ph, size_t num, float dt,
                          const int periodic[3]);
/* move_photons (src/cuda/algorithms/ptc_updater_logsph.cu:58-131),
 * send_particles and clear_guard_cells for the non-periodic log-spherical
 * grid: photons outside the bulk are removed. */
void or_move_photons_logsph(const or_mesh *m, const or_rad_params *rp, or_photons *ph,
                            size_t num, float dt);

/* update_photon_1dgr (src/cuda/algorithms/ptc_updater_1dgr.cu:301-400):
 * photons outside the bulk are removed, the others get the GR force on p1
 * and move in x1; tracked photons keep the lower u_0 in p2 on steps with
 * step % data_interval == 0. */
void or_move_photons_gr(const or_mesh *m, const or_rad_gr *g, or_photons *ph, size_t num,
                        float dt, uint32_t step, int data_interval);

/* update_photon_1dgap (src/cuda/algorithms/ptc_updater_1dgap.cu:163-192):
 * photons outside the bulk are removed, the others move dt along the sign
 * of p1. */
void or_move_photons_gap(const or_mesh *m, or_photons *ph, size_t num, float dt);

/* radiative_transfer::emit_photons (src/cuda/radiation/radiative_transfer.cu:
 * 28-97, 196-243) with the model's check_emit_photon / emit_photon: parents
 * in slot order, photon k at slot ph_num + k; *ph_num becomes ph_num +
 * marked + 1 (the reference's padding), capped at ph_cap. photon_produced
 * (may be NULL) accumulates the parents' weights per cell. Photon ids are
 * first_id, first_id + 1, ... in that order. */
void or_emit_photons(const or_mesh *m, const or_rad_params *rp, or_ptc *p, size_t ptc_num,
                     or_photons *ph, size_t *ph_num, size_t ph_cap, const or_fields *f,
                     float *photon_produced, uint32_t call, uint64_t first_id,
                     or_rad_counts *out);
/* radiative_transfer::produce_pairs (radiative_transfer.cu:99-177, 245-301)
 * with the model's check_produce_pair / produce_pair: photons in slot
 * order, pair k at slots ptc_num + 20 + 2k and + 1; *ptc_num becomes
 * ptc_num + 2 marked + 50, capped at ptc_cap. Pair ids first_id + 2k,
 * + 1. */
void or_produce_pairs(const or_mesh *m, const or_rad_params *rp, or_photons *ph, size_t ph_num,
                      or_ptc *p, size_t *ptc_num, size_t ptc_cap, const or_fields *f,
                      float *pair_produced, uint32_t call, uint64_t first_id,
                      or_rad_counts *out);

#ifdef __cplusplus
}
#endif

#endif /* AP_RAD_H_ */

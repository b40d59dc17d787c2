/* Oracle pin build: host globals standing in for the reference's
 * __constant__ state (src/cuda/constant_mem.h:11-25). */
#ifndef AP_REF_CONSTANT_MEM_H_
#define AP_REF_CONSTANT_MEM_H_
#include "cuda_builtins_host.h"
#include "core/quadmesh.h"
namespace Aperture {
/* The SimParams members the kernels read (src/sim_params.h:17-73). */
struct ap_ref_params {
  int data_interval;
  int num_species;
  float compactness, omega, gravity, rad_cooling_coef, B0, damping_coef;
  bool rad_cooling_on;
  int damping_length;
  float q_e, r_cutoff, track_percent;
  float a;  /* 1D GR lab: spin */
  bool inject_ions;
  /* radiative transfer (user_radiative_functions.cu of src/ and of the
   * pulsar lab) */
  float delta_t, gamma_thr, E_secondary, photon_path, l_curv, e_curv, BQ;
  int n_gamma;  /* inverse-Compton table size (rt_ic.cu find_n_gamma) */
  float e_min;  /* 1D gap lab: photons below 0.001 / e_min not kept */
};
extern Quadmesh dev_mesh;
extern ap_ref_params dev_params;
extern float dev_charges[8];
extern float dev_masses[8];
extern int dev_rank;
extern unsigned long long dev_ptc_id;
}  // namespace Aperture
#endif

// SimParams: the fields of src/sim_params.h:17-123 the particle update and
// the field solver read, with the reference's names and defaults. Labs fill
// it directly (the reference parses a TOML file with cpptoml).
#ifndef APERTURE_DROPIN_SIM_PARAMS_H_
#define APERTURE_DROPIN_SIM_PARAMS_H_

#include <cstddef>
#include <cstdint>

#include "ap_common.h"

namespace Aperture {

struct SimParams {
  Scalar delta_t = 0.01;
  Scalar q_e = 1.0;
  Scalar ion_mass = 1.0;
  int num_species = 3;
  bool periodic_boundary[3] = {false, false, false};
  int current_smoothing = 0;
  size_t data_interval = 100;
  int sort_interval = 20;
  uint32_t max_steps = 10000;
  uint64_t max_ptc_number = 100;
  Scalar B0 = 1.0;
  int N[3] = {1, 1, 1};
  int guard[3] = {0, 0, 0};
  float lower[3] = {0.0, 0.0, 0.0};
  float size[3] = {1.0, 1.0, 1.0};
  int tile_size[3] = {1, 1, 1};
  // log-spherical grids (src/sim_params.h:31-48, 110)
  const char *coord_system = "Cartesian";
  Scalar compactness = 0.5;
  float omega = 0.2;
  Scalar gravity = 0.0;
  bool rad_cooling_on = false;
  Scalar rad_cooling_coef = 1.0;
  int damping_length = 30;
  float damping_coef = 0.002;
  // 1D GR lab: black hole spin (src/sim_params.h:63)
  float a = 0.0;
  // photons and pair production (src/sim_params.h:23, 50-83)
  uint64_t max_photon_number = 100;
  bool create_pairs = false;
  float gamma_thr = 20.0;
  float track_percent = 0.2;
  float BQ = 1.0;
  float photon_path = 1.0;
  float E_secondary = 4.0;
  float r_cutoff = 4.0;
  float l_curv = 6.0;
  float e_curv = 6.4e-9;
  // background photons and table sizes of the 1D GR and gap labs'
  // inverse-Compton tables (src/sim_params.h:69-88)
  float e_min = 1.0e-3;
  float ic_path = 1.0;
  int n_gamma = 600;
  int n_ep = 600;
  // which user radiative functions (AP_RAD_DEFAULT: src/cuda/radiation/
  // user_radiative_functions.cu; AP_RAD_PULSAR: the pulsar lab's;
  // AP_RAD_GR1D: the 1D GR lab's; AP_RAD_GAP1D: the 1D gap lab's; the
  // reference picks them at build time by lab shadowing) and the key of the counter-based random stream that
  // replaces cuRAND
  int rad_model = 0;
  uint64_t rad_seed = 1;
};

}  // namespace Aperture

#endif

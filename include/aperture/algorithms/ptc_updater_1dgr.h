// ptc_updater_1dgr (src/algorithms/ptc_updater_1dgr.h:11-30) on
// libaperture_b200.so. The environment must have been created with
// coord_system = "1DGR" and the field-line table (sim_environment).
#ifndef APERTURE_DROPIN_PTC_UPDATER_1DGR_H_
#define APERTURE_DROPIN_PTC_UPDATER_1DGR_H_

#include "../sim_data.h"

namespace Aperture {

class ptc_updater_1dgr {
 public:
  explicit ptc_updater_1dgr(sim_environment &env) : m_env(env) {}
  ~ptc_updater_1dgr() {}

  // ptc_updater_1dgr::update_particles (ptc_updater_1dgr.cu:418-473):
  // E3 = E1 smoothed current_smoothing times with the K1_j weights, the GR
  // push along the field line, J1 (through K1_j) and Rho (through K1)
  // deposited and smoothed. Particles outside the bulk become empty slots
  // at the next update. Photons are not part of this library.
  void update_particles(sim_data &data, double dt, uint32_t step = 0) {
    ap_check(ap_update_particles(m_env.ctx(), dt, step), "update_particles");
    size_t n = 0;
    ap_check(ap_get_number(m_env.ctx(), &n), "get_number");
    data.particles.set_num(n);
  }

 private:
  sim_environment &m_env;
};

}  // namespace Aperture

#endif

// ptc_updater_1dgap (src/algorithms/ptc_updater_1dgap.h:11-27) on
// libaperture_b200.so. The environment must have been created with
// coord_system = "1DGap".
#ifndef APERTURE_DROPIN_PTC_UPDATER_1DGAP_H_
#define APERTURE_DROPIN_PTC_UPDATER_1DGAP_H_

#include "../sim_data.h"

namespace Aperture {

class ptc_updater_1dgap {
 public:
  explicit ptc_updater_1dgap(sim_environment &env) : m_env(env) {}
  ~ptc_updater_1dgap() {}

  // ptc_updater_1dgap::update_particles (ptc_updater_1dgap.cu:219-272):
  // E3 = E1 smoothed current_smoothing times, the gap push (beta_phi(x) =
  // x), J1 and Rho deposited and smoothed; particles are not wrapped, one
  // outside the bulk becomes an empty slot at the next update. Photons are
  // not part of this library.
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

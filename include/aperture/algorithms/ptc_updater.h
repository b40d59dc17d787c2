// ptc_updater (src/algorithms/ptc_updater.h:11-24) on libaperture_b200.so.
#ifndef APERTURE_DROPIN_PTC_UPDATER_H_
#define APERTURE_DROPIN_PTC_UPDATER_H_

#include "../sim_data.h"

namespace Aperture {

class ptc_updater {
 public:
  explicit ptc_updater(sim_environment &env) : m_env(env) {}
  ~ptc_updater() {}

  // ptc_updater::update_particles (ptc_updater.cu:748-841).
  void update_particles(sim_data &data, double dt, uint32_t step = 0) {
    ap_check(ap_update_particles(m_env.ctx(), dt, step), "update_particles");
    size_t n = 0;
    ap_check(ap_get_number(m_env.ctx(), &n), "get_number");
    data.particles.set_num(n);
  }
  // No-op in the reference (ptc_updater.cu:843-850).
  void apply_boundary(sim_data &, double, uint32_t = 0) {}
  // ptc_updater::smooth_current (ptc_updater.cu:852-912).
  void smooth_current(sim_data &, uint32_t step = 0) {
    ap_check(ap_smooth_current(m_env.ctx(), step), "smooth_current");
  }
  void smooth_current(multi_array<Scalar> &array) {
    ap_check(ap_smooth_array(m_env.ctx(), array.view()), "smooth_current");
  }

 protected:
  sim_environment &m_env;
};

}  // namespace Aperture

#endif

// ptc_updater_logsph (src/algorithms/ptc_updater_logsph.h:13-28) on
// libaperture_b200.so. The environment must have been created with
// coord_system = "LogSpherical".
#ifndef APERTURE_DROPIN_PTC_UPDATER_LOGSPH_H_
#define APERTURE_DROPIN_PTC_UPDATER_LOGSPH_H_

#include "../sim_data.h"

namespace Aperture {

class ptc_updater_logsph {
 public:
  explicit ptc_updater_logsph(sim_environment &env) : m_env(env) {}
  ~ptc_updater_logsph() {}

  // update_particles followed by apply_boundary (ptc_updater_logsph.cu:
  // 681-836): push, move, deposit, process_j, smoothing, axis current,
  // outflow flags; particles that leave the grid become empty slots.
  void update_particles(sim_data &data, double dt, uint32_t step = 0) {
    ap_check(ap_update_particles(m_env.ctx(), dt, step), "update_particles");
    size_t n = 0;
    ap_check(ap_get_number(m_env.ctx(), &n), "get_number");
    data.particles.set_num(n);
  }
  // Already run by update_particles, as in the reference.
  void apply_boundary(sim_data &, double, uint32_t = 0) {}
  // inject_ptc (ptc_updater_logsph.cu:849-870): pairs at the stellar
  // surface where it is not yet dense; see ap_logsph_inject.
  void inject_ptc(sim_data &data, int inj_per_cell, Scalar p1, Scalar p2, Scalar p3, Scalar w,
                  Scalar omega) {
    ap_check(ap_logsph_inject(m_env.ctx(), inj_per_cell, p1, p2, p3, w, omega,
                              0x5EEDull + inject_calls_++),
             "inject_ptc");
    size_t n = 0;
    ap_check(ap_get_number(m_env.ctx(), &n), "get_number");
    data.particles.set_num(n);
  }

 private:
  sim_environment &m_env;
  uint64_t inject_calls_ = 0;
};

}  // namespace Aperture

#endif

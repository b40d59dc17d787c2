// field_solver_logsph (src/algorithms/field_solver_logsph.h:10-20) on
// libaperture_b200.so. The environment must have been created with
// coord_system = "LogSpherical".
#ifndef APERTURE_DROPIN_FIELD_SOLVER_LOGSPH_H_
#define APERTURE_DROPIN_FIELD_SOLVER_LOGSPH_H_

#include "../sim_data.h"

namespace Aperture {

class field_solver_logsph {
 public:
  explicit field_solver_logsph(sim_environment &env) : m_env(env) {}
  ~field_solver_logsph() {}

  // field_solver_logsph::update_fields (field_solver_logsph.cu:354-398).
  void update_fields(sim_data &, double dt, double time = 0.0) {
    (void)time;
    ap_check(ap_update_fields(m_env.ctx(), dt, 0), "update_fields");
  }
  // field_solver_logsph::apply_boundary (field_solver_logsph.cu:403-428).
  void apply_boundary(sim_data &, double omega, double time = 0.0) {
    (void)time;
    ap_check(ap_logsph_field_boundary(m_env.ctx(), omega), "apply_boundary");
  }

 private:
  sim_environment &m_env;
};

}  // namespace Aperture

#endif

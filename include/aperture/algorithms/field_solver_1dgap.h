// field_solver_1dgap (src/algorithms/field_solver_1dgap.h:9-20) on
// libaperture_b200.so. The environment must have been created with
// coord_system = "1DGap".
#ifndef APERTURE_DROPIN_FIELD_SOLVER_1DGAP_H_
#define APERTURE_DROPIN_FIELD_SOLVER_1DGAP_H_

#include "../sim_data.h"

namespace Aperture {

class field_solver_1dgap {
 public:
  explicit field_solver_1dgap(sim_environment &env) : m_env(env) {}
  ~field_solver_1dgap() {}

  // field_solver_1dgap::update_fields (field_solver_1dgap.cu:28-40):
  // E1 += (1.6 B0 - J1) dt on the bulk cells but the outermost.
  void update_fields(sim_data &data, double dt, double time = 0.0) {
    (void)data;
    (void)time;
    ap_check(ap_update_fields(m_env.ctx(), dt, 0), "update_fields");
  }

 private:
  sim_environment &m_env;
};

}  // namespace Aperture

#endif

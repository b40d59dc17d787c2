// field_solver_1dgr (src/algorithms/field_solver_1dgr.h:11-22) on
// libaperture_b200.so: E1 += (j0 - J1) dt (field_solver_1dgr.cu:14-44).
#ifndef APERTURE_DROPIN_FIELD_SOLVER_1DGR_H_
#define APERTURE_DROPIN_FIELD_SOLVER_1DGR_H_

#include "../sim_data.h"

namespace Aperture {

class field_solver_1dgr {
 public:
  explicit field_solver_1dgr(sim_environment &env) : m_env(env) {}
  ~field_solver_1dgr() {}

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

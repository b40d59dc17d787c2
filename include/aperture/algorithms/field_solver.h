// field_solver (src/algorithms/field_solver.h:11-25) on libaperture_b200.so.
#ifndef APERTURE_DROPIN_FIELD_SOLVER_H_
#define APERTURE_DROPIN_FIELD_SOLVER_H_

#include "../sim_data.h"

namespace Aperture {

class field_solver {
 public:
  explicit field_solver(sim_environment &env) : m_env(env) {}
  ~field_solver() {}

  // field_solver::update_fields (field_solver.cu:334-358).
  void update_fields(sim_data &, double dt, uint32_t step = 0) {
    ap_check(ap_update_fields(m_env.ctx(), dt, step), "update_fields");
  }
  // No-op in the reference (field_solver.cu:451-452).
  void apply_outflow_boundary(sim_data &, double = 0.0) {}
  void compute_divs(sim_data &) { ap_check(ap_compute_divs(m_env.ctx()), "compute_divs"); }
  void update_e_field(sim_data &, double dt) {
    ap_check(ap_update_e_field(m_env.ctx(), dt), "update_e_field");
  }
  void update_b_field(sim_data &, double dt) {
    ap_check(ap_update_b_field(m_env.ctx(), dt), "update_b_field");
  }

 private:
  sim_environment &m_env;
};

}  // namespace Aperture

#endif

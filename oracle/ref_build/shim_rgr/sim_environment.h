/* Oracle pin build, 1D GR radiation: the sim_environment that the lab's
 * user_rt_init takes (src/sim_environment.h), reduced to the members it
 * names. The pin never calls user_rt_init. */
#ifndef AP_REF_RGR_SIM_ENVIRONMENT_H_
#define AP_REF_RGR_SIM_ENVIRONMENT_H_
#include "core/grid.h"
namespace Aperture {
struct sim_environment {
  const SimParams &params() const { return m_params; }
  Grid &local_grid();
  SimParams m_params;
};
}  // namespace Aperture
#endif

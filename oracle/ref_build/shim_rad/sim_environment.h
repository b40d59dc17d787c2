/* Oracle pin build, radiation part: the sim_environment that the
 * reference's user radiative functions take in user_rt_init
 * (src/sim_environment.h), reduced to the one member the pulsar lab's
 * version names. The pin never calls user_rt_init. */
#ifndef AP_REF_RAD_SIM_ENVIRONMENT_H_
#define AP_REF_RAD_SIM_ENVIRONMENT_H_
namespace Aperture {
class Grid;
struct sim_environment {
  Grid &local_grid();
};
}  // namespace Aperture
#endif

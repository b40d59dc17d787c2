/* Oracle pin build: mesh_ptrs_log_sph with the members of
 * src/cuda/grids/grid_log_sph_ptrs.h:8-17. */
#ifndef AP_REF_GRID_LOG_SPH_PTRS_H_
#define AP_REF_GRID_LOG_SPH_PTRS_H_
#include "cuda/utils/pitchptr.h"
namespace Aperture {
struct mesh_ptrs_log_sph {
  pitchptr<Scalar> l1_e, l2_e, l3_e;
  pitchptr<Scalar> l1_b, l2_b, l3_b;
  pitchptr<Scalar> A1_e, A2_e, A3_e;
  pitchptr<Scalar> A1_b, A2_b, A3_b;
  pitchptr<Scalar> dV;
};
}  // namespace Aperture
#endif

/* Oracle pin build: host globals standing in for the reference's
 * __constant__ state (src/cuda/constant_mem.h:11-25). */
#ifndef AP_REF_CONSTANT_MEM_H_
#define AP_REF_CONSTANT_MEM_H_
#include "cuda_builtins_host.h"
#include "core/quadmesh.h"
namespace Aperture {
struct ap_ref_params { int data_interval; };
extern Quadmesh dev_mesh;
extern ap_ref_params dev_params;
extern float dev_charges[8];
extern float dev_masses[8];
}  // namespace Aperture
#endif

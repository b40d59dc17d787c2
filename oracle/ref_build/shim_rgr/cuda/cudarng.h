/* Oracle pin build, 1D GR radiation: CudaRng of src/cuda/cudarng.h:10-27
 * with its m_local_state member (the 1D GR lab's emit_photon hands it to
 * gen_photon_e), handing out the uniforms the pin driver queued; the
 * photon-energy draw of gen_photon_e (curand_uniform of that state) comes
 * from the same queue (rgr_host_math.h). */
#ifndef AP_REF_RGR_CUDARNG_H_
#define AP_REF_RGR_CUDARNG_H_
#include "rgr_host_math.h"
namespace Aperture {
namespace Kernels {
struct CudaRng {
  explicit CudaRng(curandState *s) : m_local_state(*s) {}
  float operator()() { return ap_ref_next_uniform(); }
  curandState m_local_state;
};
}  // namespace Kernels
}  // namespace Aperture
#endif

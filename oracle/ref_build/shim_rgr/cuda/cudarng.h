/* Oracle pin build, 1D GR radiation: CudaRng of src/cuda/cudarng.h:10-27
 * with its m_local_state member (the 1D GR lab's emit_photon hands it to
 * gen_photon_e), handing out the uniforms the pin driver queued; the
 * photon-energy draw of gen_photon_e comes from the same queue. */
#ifndef AP_REF_RGR_CUDARNG_H_
#define AP_REF_RGR_CUDARNG_H_
#include "ls_host_math.h"
namespace Aperture {
namespace Kernels {
extern const float *ap_ref_rng_queue;
extern int ap_ref_rng_left;
extern int ap_ref_rng_underflow; /* set when a function draws more than queued */
inline float ap_ref_next_uniform() {
  if (ap_ref_rng_left <= 0) {
    ap_ref_rng_underflow = 1;
    return 0.5f;
  }
  --ap_ref_rng_left;
  return *ap_ref_rng_queue++;
}
struct CudaRng {
  explicit CudaRng(curandState *s) : m_local_state(*s) {}
  float operator()() { return ap_ref_next_uniform(); }
  curandState m_local_state;
};
}  // namespace Kernels
}  // namespace Aperture
#endif

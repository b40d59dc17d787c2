/* Oracle pin build, radiation part: CudaRng of src/cuda/cudarng.h:10-27
 * with the same interface, handing out the uniforms the pin driver queued
 * (the reference draws them from cuRAND XORWOW). */
#ifndef AP_REF_RAD_CUDARNG_H_
#define AP_REF_RAD_CUDARNG_H_
#include "ls_host_math.h"
namespace Aperture {
namespace Kernels {
extern const float *ap_ref_rng_queue;
extern int ap_ref_rng_left;
extern int ap_ref_rng_underflow;  /* set when a function draws more than queued */
struct CudaRng {
  explicit CudaRng(curandState *) {}
  float operator()() {
    if (ap_ref_rng_left <= 0) {
      ap_ref_rng_underflow = 1;
      return 0.5f;
    }
    --ap_ref_rng_left;
    return *ap_ref_rng_queue++;
  }
};
}  // namespace Kernels
}  // namespace Aperture
#endif

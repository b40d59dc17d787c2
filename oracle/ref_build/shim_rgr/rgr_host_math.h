/* Oracle pin build, 1D GR radiation: the float overload set of
 * ls_host_math.h (unqualified log, exp, sqrt, ... of float arguments are
 * the float functions, as in the reference's device code), with a
 * curand_uniform that hands out the uniforms the pin driver queued: the
 * reference's gen_photon_e draws its photon energy from the CudaRng's
 * state. */
#ifndef AP_REF_RGR_HOST_MATH_H_
#define AP_REF_RGR_HOST_MATH_H_
#include <cmath>
using std::sqrt;
using std::acos;
using std::log;
using std::atan2;
using std::sin;
using std::cos;
using std::exp;
using std::floor;
using std::abs;
using std::pow;
/* CUDA's device min / max of floating-point values: fmin / fmax */
inline double min(double a, double b) { return std::fmin(a, b); }
inline double max(double a, double b) { return std::fmax(a, b); }
inline float min(float a, float b) { return std::fmin(a, b); }
inline float max(float a, float b) { return std::fmax(a, b); }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
struct curandState { unsigned long long s; };
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
}  // namespace Kernels
}  // namespace Aperture
inline float curand_uniform(curandState *) { return Aperture::Kernels::ap_ref_next_uniform(); }
#define __syncthreads() ((void)0)
inline unsigned long long atomicAdd(unsigned long long *a, int v) {
  unsigned long long old = *a;
  *a += (unsigned long long)v;
  return old;
}
#endif

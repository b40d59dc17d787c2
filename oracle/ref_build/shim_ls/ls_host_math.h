/* Oracle pin build, log-spherical part: the device code of the reference
 * calls unqualified sqrt, acos, log, atan2, sin, cos, floor on float
 * arguments, which CUDA resolves to the float functions (sqrtf, acosf, ...).
 * These using-declarations give the host build the same overload set, so
 * the host run evaluates the C library's float functions. Also host
 * stand-ins for curand (only the injection kernel draws numbers; the pin
 * never calls it) and for __syncthreads (the emulated launches run one
 * thread at a time, and no thread of these kernels reads a cell that
 * another thread writes before the barrier). */
#ifndef AP_REF_LS_HOST_MATH_H_
#define AP_REF_LS_HOST_MATH_H_
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
struct curandState { unsigned long long s; };
inline float curand_uniform(curandState *st) {
  st->s = st->s * 6364136223846793005ull + 1442695040888963407ull;
  return (float)((st->s >> 40) + 1) / 16777217.0f;
}
#define __syncthreads() ((void)0)
/* atomicAdd(&dev_ptc_id, 1) in the injection kernel: CUDA converts the int. */
inline unsigned long long atomicAdd(unsigned long long *a, int v) {
  unsigned long long old = *a;
  *a = old + (unsigned long long)v;
  return old;
}
#endif

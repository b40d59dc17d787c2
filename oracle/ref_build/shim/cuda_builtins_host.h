/* Host stand-ins for the CUDA built-ins the reference kernels use, so their
 * bodies run as sequential host code (one thread, one block): every
 * grid-stride loop then visits all elements in index order and atomicAdd is
 * a plain add. Part of the oracle pin build; never part of the product. */
#ifndef AP_REF_CUDA_BUILTINS_HOST_H_
#define AP_REF_CUDA_BUILTINS_HOST_H_
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstddef>
using std::max;
using std::min;

struct ap_ref_dim3 { unsigned x, y, z; };
#ifdef AP_REF_MT
/* multi-threaded timing build: every host thread emulates its own launch */
extern thread_local ap_ref_dim3 blockIdx, blockDim, threadIdx, gridDim;
#else
extern ap_ref_dim3 blockIdx, blockDim, threadIdx, gridDim;
#endif

#define __global__
#define __device__
#define __host__
#define __constant__
#define __forceinline__ inline
#define __launch_bounds__(...)

template <typename T> inline T atomicAdd(T *addr, T v) {
  T old = *addr;
  *addr = old + v;
  return old;
}
/* The reference traps on NaN momenta; the pin build never feeds NaN. */
#define asm(...) ((void)0)
#endif

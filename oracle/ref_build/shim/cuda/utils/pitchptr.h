/* Oracle pin build: the pitched-pointer accessor the reference kernels use
 * (same member names and byte-offset semantics as src/cuda/utils/pitchptr.h). */
#ifndef AP_REF_PITCHPTR_H_
#define AP_REF_PITCHPTR_H_
#include "cuda_builtins_host.h"
struct cudaPitchedPtr { void *ptr; size_t pitch, xsize, ysize; };
namespace Aperture {
template <typename T> struct pitchptr {
  cudaPitchedPtr p;
  T &operator[](size_t off) { return *(T *)((char *)p.ptr + off); }
  const T &operator[](size_t off) const { return *(T *)((char *)p.ptr + off); }
  T &operator()(int i, int j = 0) { return *((T *)((char *)p.ptr + j * p.pitch) + i); }
  const T &operator()(int i, int j = 0) const { return *((T *)((char *)p.ptr + j * p.pitch) + i); }
  T &operator()(int i, int j, int k) { return *((T *)((char *)p.ptr + (j + k * p.ysize) * p.pitch) + i); }
  size_t compute_offset(int i, int j = 0) const { return j * p.pitch + i * sizeof(T); }
  size_t compute_offset(int i, int j, int k) const { return (j + k * p.ysize) * p.pitch + i * sizeof(T); }
};
}  // namespace Aperture
#endif

// Shared pieces of the C++ drop-in layer over libaperture_b200.so: the
// Scalar type, the mesh (Quadmesh layout, src/core/quadmesh.h:16-29), the
// error type and the status check. Host code only.
#ifndef APERTURE_DROPIN_COMMON_H_
#define APERTURE_DROPIN_COMMON_H_

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "../aperture_b200.h"

namespace Aperture {

typedef float Scalar;  // src/core/typedefs.h:11-18 (single precision build)
typedef float Pos_t;

// The reference throws from CudaSafeCall (src/cuda/cudaUtility.h:61-74);
// every failing call of this layer throws ap_error.
class ap_error : public std::runtime_error {
 public:
  ap_error(int status, const std::string &what)
      : std::runtime_error(what + ": " + ap_status_string(status)), status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

inline void ap_check(int status, const char *what) {
  if (status != AP_OK) throw ap_error(status, what);
}

inline void cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess)
    throw ap_error(AP_ERR_CUDA, std::string(what) + " (" + cudaGetErrorString(e) + ")");
}

// Quadmesh: same members and index helpers as src/core/quadmesh.h:16-364.
struct Quadmesh : public ap_mesh {
  int reduced_dim(int i) const { return dims[i] - 2 * guard[i]; }
  int dim() const {
    if (dims[1] <= 1 && dims[2] <= 1) return 1;
    if (dims[2] <= 1) return 2;
    return 3;
  }
  Scalar pos(int i, int n, Scalar pos_in_cell) const {
    return i < dimension ? lower[i] + delta[i] * (n - guard[i] + pos_in_cell)
                         : pos_in_cell * delta[i];
  }
  Scalar pos(int i, int n, int stagger) const { return pos(i, n, (Scalar)(stagger * 0.5 + 0.5)); }
  int get_idx(int c1, int c2 = 0, int c3 = 0) const {
    return c1 + c2 * dims[0] + c3 * dims[0] * dims[1];
  }
  int size() const { return dims[0] * dims[1] * dims[2]; }
  uint32_t get_c1(uint32_t idx) const { return idx % dims[0]; }
  uint32_t get_c2(uint32_t idx) const { return (idx / dims[0]) % dims[1]; }
};

}  // namespace Aperture

#endif

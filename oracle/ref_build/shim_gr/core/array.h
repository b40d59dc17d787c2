/* Oracle pin build: a host array standing in for the reference's
 * array<T> (src/core/array.h) in Grid_1dGR: zero-filled storage, element
 * access, and a device copy that is the host storage itself. */
#ifndef AP_REF_GR_ARRAY_H_
#define AP_REF_GR_ARRAY_H_
#include <cstddef>
#include <vector>
namespace Aperture {
template <typename T>
class array {
 public:
  array() {}
  explicit array(size_t n) : v_(n, T(0)) {}
  T &operator[](size_t i) { return v_[i]; }
  const T &operator[](size_t i) const { return v_[i]; }
  size_t size() const { return v_.size(); }
  T *data() { return v_.data(); }
  const T *data() const { return v_.data(); }
  void copy_to_device() {}
  // the host storage stands in for the device copy
  T *dev_ptr() { return v_.data(); }
  const T *dev_ptr() const { return v_.data(); }

 private:
  std::vector<T> v_;
};
}  // namespace Aperture
#endif

/* Oracle pin build: a host-only 2D array with the multi_array members that
 * Grid_LogSph::compute_coef uses (resize, element access, copy_to_device
 * as a no-op). */
#ifndef AP_REF_MULTI_ARRAY_H_
#define AP_REF_MULTI_ARRAY_H_
#include <vector>
namespace Aperture {
template <typename T> class multi_array {
 public:
  void resize(int w, int h) { m_w = w; m_h = h; m_v.assign((size_t)w * h, T(0)); }
  T &operator()(int i, int j) { return m_v[(size_t)i + (size_t)j * m_w]; }
  const T &operator()(int i, int j) const { return m_v[(size_t)i + (size_t)j * m_w]; }
  void copy_to_device() {}
  void copy_to_host() {}
  const T *data() const { return m_v.data(); }
  int m_w = 0, m_h = 0;
  std::vector<T> m_v;
};
}  // namespace Aperture
#endif

/* Oracle pin build: declarations that let Grid_LogSph::compute_flux
 * compile; the pin never calls it. */
#ifndef AP_REF_FIELDS_H_
#define AP_REF_FIELDS_H_
#include "core/grid.h"
namespace Aperture {
template <typename T> struct scalar_field {
  void initialize() {}
  void copy_to_host() {}
  const Grid &grid() const { return *m_grid; }
  T &operator()(int, int, int, int) { return m_v; }
  const Grid *m_grid = nullptr;
  T m_v = T(0);
};
template <typename T> struct vector_field : scalar_field<T> {};
}  // namespace Aperture
#endif

/* Oracle pin build: the Grid base that src/grids/grid_log_sph.h derives
 * from, reduced to what Grid_LogSph::compute_coef uses (a Quadmesh). */
#ifndef AP_REF_GRID_H_
#define AP_REF_GRID_H_
#include "core/quadmesh.h"
namespace Aperture {
struct SimParams {};
class Grid {
 public:
  virtual ~Grid() {}
  virtual void compute_coef(const SimParams &) {}
  const Quadmesh &mesh() const { return m_mesh; }
  Quadmesh m_mesh;
};
}  // namespace Aperture
#endif

/* Oracle pin build: the Grid base that src/grids/grid_1dgr.h derives from,
 * reduced to what Grid_1dGR::compute_coef uses (a Quadmesh), and the three
 * SimParams members it reads. */
#ifndef AP_REF_GR_GRID_H_
#define AP_REF_GR_GRID_H_
#include "core/quadmesh.h"
namespace Aperture {
struct SimParams {
  float omega, a, B0;
};
class Grid {
 public:
  Grid() {}
  Grid(int, int = 1, int = 1) {}
  virtual ~Grid() {}
  virtual void compute_coef(const SimParams &) {}
  const Quadmesh &mesh() const { return m_mesh; }
  Quadmesh m_mesh;
};
}  // namespace Aperture
#endif

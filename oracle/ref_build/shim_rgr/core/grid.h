/* Oracle pin build, 1D GR radiation: the Grid base of src/grids/grid_1dgr.h
 * as in shim_gr/core/grid.h, with the SimParams members that the lab's
 * user_rt_init also names (e_min, ic_path). */
#ifndef AP_REF_GR_GRID_H_
#define AP_REF_GR_GRID_H_
#include "core/quadmesh.h"
namespace Aperture {
struct SimParams {
  float omega, a, B0;
  float e_min, ic_path;
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

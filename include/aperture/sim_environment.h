// sim_environment for one rank without MPI (src/sim_environment.h,
// sim_environment_impl.hpp): the grid, the per-species charges and masses,
// and the guard exchange, which on one periodic rank is done by device
// kernels instead of MPI self-exchanges. Owns the library context.
#ifndef APERTURE_DROPIN_SIM_ENVIRONMENT_H_
#define APERTURE_DROPIN_SIM_ENVIRONMENT_H_

#include <cmath>
#include <cstring>

#include "multi_array.h"
#include "sim_params.h"

namespace Aperture {

class Grid {
 public:
  const Quadmesh &mesh() const { return mesh_; }
  Quadmesh &mesh() { return mesh_; }
  int dim() const { return mesh_.dim(); }

 private:
  Quadmesh mesh_{};
};

class sim_environment {
 public:
  // The reference constructor (int*, char***) initialises MPI and parses
  // the configuration file; this one takes the parsed parameters. A 1D GR
  // environment (coord_system "1DGR") also takes the field-line table the
  // reference's Grid_1dGR reads from coef.h5 (grid_1dgr.cpp:41-66).
  explicit sim_environment(const SimParams &params, int device = -1,
                           const ap_gr_table *gr_table = nullptr)
      : params_(params) {
    if (device >= 0) cuda_check(cudaSetDevice(device), "cudaSetDevice");
    // Grid::init (src/core/grid.cpp:31-48)
    Quadmesh &m = grid_.mesh();
    for (int i = 0; i < 3; ++i) {
      m.guard[i] = params.guard[i];
      m.sizes[i] = params.size[i];
      m.lower[i] = params.lower[i];
      m.dims[i] = params.N[i] + 2 * params.guard[i];
      m.delta[i] = params.size[i] / params.N[i];
      m.inv_delta[i] = (float)(1.0 / m.delta[i]);
    }
    m.dimension = m.dim();
    // setup_env (sim_environment_impl.hpp:90-101)
    for (int i = 0; i < AP_MAX_SPECIES; ++i) {
      charges_[i] = params.q_e;
      masses_[i] = params.q_e;
    }
    charges_[0] *= -1.0f;           // electron
    masses_[2] *= params.ion_mass;  // ion
    ap_params p{};
    p.num_species = params.num_species;
    p.data_interval = (int)params.data_interval;
    p.current_smoothing = params.current_smoothing;
    for (int i = 0; i < 3; ++i) p.periodic[i] = params.periodic_boundary[i] ? 1 : 0;
    for (int i = 0; i < AP_MAX_SPECIES; ++i) {
      p.charges[i] = charges_[i];
      p.masses[i] = masses_[i];
    }
    p.tile[0] = p.tile[1] = 0;
    p.chunk = 0;
    ap_params_ = p;
    if (std::strcmp(params.coord_system, "LogSpherical") == 0) {
      // Grid_LogSph (src/grids/grid_log_sph.cpp:11-126): the library
      // computes the coefficient arrays when the context is created
      ap_logsph_params lp{};
      lp.compactness = params.compactness;
      lp.omega = params.omega;
      lp.gravity = params.gravity;
      lp.rad_cooling_coef = params.rad_cooling_coef;
      lp.B0 = params.B0;
      lp.damping_coef = params.damping_coef;
      lp.rad_cooling_on = params.rad_cooling_on ? 1 : 0;
      lp.damping_length = params.damping_length;
      ap_check(ap_ctx_create_logsph(&m, &p, &lp, &ctx_), "ap_ctx_create_logsph");
    } else if (std::strcmp(params.coord_system, "1DGR") == 0) {
      // the 1D GR lab (labs/1dgr): ptc_updater_1dgr / field_solver_1dgr
      if (!gr_table) throw ap_error(AP_ERR_INVALID, "1DGR environment without a coef table");
      ap_gr_params gp{};
      gp.a = params.a;
      gp.omega = params.omega;
      gp.B0 = params.B0;
      ap_check(ap_ctx_create_1dgr(&m, &p, &gp, gr_table, &ctx_), "ap_ctx_create_1dgr");
    } else if (std::strcmp(params.coord_system, "1DGap") == 0) {
      // the 1D gap lab (labs/1dgap): ptc_updater_1dgap / field_solver_1dgap
      ap_gap_params gp{};
      gp.B0 = params.B0;
      ap_check(ap_ctx_create_1dgap(&m, &p, &gp, &ctx_), "ap_ctx_create_1dgap");
    } else {
      ap_check(ap_ctx_create(&m, &p, &ctx_), "ap_ctx_create");
    }
  }
  ~sim_environment() {
    if (ctx_) ap_ctx_destroy(ctx_);
  }
  sim_environment(const sim_environment &) = delete;
  sim_environment &operator=(const sim_environment &) = delete;

  SimParams &params() { return params_; }
  const SimParams &params() const { return params_; }
  const Grid &local_grid() const { return grid_; }
  const Grid &grid() const { return grid_; }
  const Quadmesh &mesh() const { return grid_.mesh(); }
  const float *charges() const { return charges_; }
  const float *masses() const { return masses_; }
  ap_ctx *ctx() const { return ctx_; }

  void send_array_guard_cells(multi_array<Scalar> &a) {
    ap_check(ap_send_guard_cells(ctx_, a.view()), "send_guard_cells");
  }
  void send_add_array_guard_cells(multi_array<Scalar> &a) {
    ap_check(ap_send_add_guard_cells(ctx_, a.view()), "send_add_guard_cells");
  }
  void send_guard_cells(vector_field<Scalar> &f) {
    for (int i = 0; i < 3; ++i) send_array_guard_cells(f.data(i));
  }
  void send_guard_cells(scalar_field<Scalar> &f) { send_array_guard_cells(f.data()); }
  void send_add_guard_cells(vector_field<Scalar> &f) {
    for (int i = 0; i < 3; ++i) send_add_array_guard_cells(f.data(i));
  }
  void send_add_guard_cells(scalar_field<Scalar> &f) { send_add_array_guard_cells(f.data()); }

 private:
  SimParams params_;
  Grid grid_;
  float charges_[AP_MAX_SPECIES];
  float masses_[AP_MAX_SPECIES];
  ap_params ap_params_{};
  ap_ctx *ctx_ = nullptr;
};

}  // namespace Aperture

#endif

// A 1D gap lab written against the drop-in C++ headers the way the
// reference's 1dgap lab uses its algorithm classes (labs/1dgap/src/
// main.cpp): a ramp in E1, pairs from fill_multiplicity, then
// update_particles / update_fields with a periodic sort. Exits 0 and
// prints "gap_lab ok" when the run is healthy.
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "aperture/algorithms/field_solver_1dgap.h"
#include "aperture/algorithms/ptc_updater_1dgap.h"
#include "aperture/radiation/radiative_transfer.h"

using namespace Aperture;

int main(int argc, char **argv) {
  int steps = argc > 1 ? atoi(argv[1]) : 8;
  SimParams params;
  params.coord_system = "1DGap";
  params.N[0] = 2048;
  params.guard[0] = 2;
  params.lower[0] = 0.0f;
  params.size[0] = 1.0f;
  params.delta_t = 0.5f / 2048;
  params.q_e = 1.0f;
  params.num_species = 2;
  params.current_smoothing = 1;
  params.sort_interval = 5;
  params.max_ptc_number = 2048 * 8;
  params.B0 = 1.0f;
  params.periodic_boundary[0] = false;
  // labs/1dgap/src/main.cpp: radiative_transfer with the lab's functions
  params.create_pairs = true;
  params.rad_model = AP_RAD_GAP1D;
  params.max_photon_number = 2048 * 8;
  params.ic_path = 1.0e-3f;
  params.n_gamma = 200;
  params.n_ep = 200;
  try {
    sim_environment env(params);
    sim_data data(env);
    field_solver_1dgap solver(env);
    ptc_updater_1dgap pusher(env);
    radiative_transfer rad(env);
    data.E.initialize(0, [](double x, double, double) { return 0.5 * x; });
    data.fill_multiplicity(1.0f, 2);
    const size_t n0 = data.particles.number();
    uint64_t emitters = 0;
    for (uint32_t step = 0; step < (uint32_t)steps; ++step) {
      pusher.update_particles(data, params.delta_t, step);  // and the photons
      solver.update_fields(data, params.delta_t, step * params.delta_t);
      if (params.create_pairs) {
        rad.emit_photons(data);
        emitters += rad.last_counts().marked;
        rad.produce_pairs(data);
      }
      if (step % params.sort_interval == 0 && step != 0) data.sort_particles();
    }
    ap_diag d{};
    ap_check(ap_diagnostics(env.ctx(), &d), "diagnostics");
    const bool ok = n0 == (size_t)2048 * 4 && data.particles.number() > n0 / 2 &&
                    std::isfinite(d.kinetic) && std::isfinite(d.field_energy) &&
                    d.field_energy > 0.0 && emitters > 0;
    std::printf("particles %zu of %zu kinetic %.6e field_energy %.6e emitters %llu\n",
                data.particles.number(), n0, d.kinetic, d.field_energy,
                (unsigned long long)emitters);
    std::printf(ok ? "gap_lab ok\n" : "gap_lab FAILED\n");
    return ok ? 0 : 1;
  } catch (const ap_error &e) {
    std::printf("gap_lab error: %s\n", e.what());
    return 2;
  }
}

// A 2D periodic box lab written against the drop-in C++ headers the way a
// reference lab's main.cpp uses the algorithm classes (construct the
// environment, the data, the solver and the pusher; set fields; fill
// particles; loop update_particles / update_fields / sort_particles).
// Exits 0 and prints "box_lab ok" when the run is healthy.
#include <cmath>
#include <cstdio>

#include "aperture/algorithms/field_solver.h"
#include "aperture/algorithms/ptc_updater.h"

using namespace Aperture;

int main(int argc, char **argv) {
  int steps = argc > 1 ? atoi(argv[1]) : 8;
  SimParams params;
  params.N[0] = params.N[1] = 64;
  params.guard[0] = params.guard[1] = 2;
  params.size[0] = params.size[1] = 1.0f;
  params.delta_t = 0.5f / 64;
  params.q_e = 1.0f;
  params.num_species = 2;
  params.periodic_boundary[0] = params.periodic_boundary[1] = true;
  params.data_interval = 4;
  params.sort_interval = 5;
  params.max_ptc_number = 64 * 64 * 8;
  params.B0 = 1.0f;
  try {
    sim_environment env(params);
    sim_data data(env);
    field_solver solver(env);
    ptc_updater pusher(env);
    // an electromagnetic wave along the diagonal on top of a guide field
    const double k = 2.0 * M_PI, amp = 0.2;
    data.E.initialize(0, [&](double x, double y, double) { return -amp * std::sin(k * (x + y)); });
    data.E.initialize(1, [&](double x, double y, double) { return amp * std::sin(k * (x + y)); });
    data.B.initialize(2, [&](double x, double y, double) {
      return params.B0 + amp * std::sqrt(2.0) * std::sin(k * (x + y));
    });
    env.send_guard_cells(data.E);
    env.send_guard_cells(data.B);
    data.fill_multiplicity(1.0f, 4);
    const size_t n0 = data.particles.number();
    for (uint32_t step = 0; step < (uint32_t)steps; ++step) {
      pusher.update_particles(data, params.delta_t, step);
      solver.update_fields(data, params.delta_t, step);
      if (step % params.sort_interval == 0 && step != 0) data.sort_particles();
    }
    ap_diag d{};
    ap_check(ap_diagnostics(env.ctx(), &d), "diagnostics");
    const bool ok = data.particles.number() == n0 && n0 == (size_t)64 * 64 * 8 &&
                    std::isfinite(d.kinetic) && std::fabs(d.charge) < 1e-6 &&
                    d.field_energy > 0.0;
    std::printf("particles %zu kinetic %.6e charge %.3e field_energy %.6e\n",
                data.particles.number(), d.kinetic, d.charge, d.field_energy);
    std::printf(ok ? "box_lab ok\n" : "box_lab FAILED\n");
    return ok ? 0 : 1;
  } catch (const ap_error &e) {
    std::printf("box_lab error: %s\n", e.what());
    return 2;
  }
}

// A log-spherical lab written against the drop-in C++ headers the way the
// reference's pulsar lab uses the algorithm classes: dipole background B
// through init_bg_B_field, pairs from fill_multiplicity, then
// update_particles / update_fields / apply_boundary with a spin-up of the
// star and a periodic sort. Exits 0 and prints "pulsar_lab ok" when the
// run is healthy.
#include <cmath>
#include <cstdio>

#include "aperture/algorithms/field_solver_logsph.h"
#include "aperture/algorithms/ptc_updater_logsph.h"

using namespace Aperture;

int main(int argc, char **argv) {
  int steps = argc > 1 ? atoi(argv[1]) : 8;
  SimParams params;
  params.coord_system = "LogSpherical";
  params.N[0] = 128;
  params.N[1] = 64;
  params.guard[0] = params.guard[1] = 2;
  params.lower[0] = 0.0f;
  params.size[0] = (float)std::log(50.0);
  params.size[1] = (float)M_PI;
  params.delta_t = 0.4f * (float)M_PI / 64;
  params.q_e = 1.0f;
  params.num_species = 3;
  params.data_interval = 4;
  params.sort_interval = 5;
  params.max_ptc_number = 128 * 64 * 8;
  params.B0 = 1.0f;
  params.omega = 0.1f;
  params.compactness = 0.0f;
  params.damping_length = 16;
  try {
    sim_environment env(params);
    sim_data data(env);
    field_solver_logsph solver(env);
    ptc_updater_logsph pusher(env);
    const Scalar B0 = params.B0;
    data.init_bg_B_field(0, [B0](Scalar x1, Scalar x2, Scalar) {
      Scalar r = std::exp(x1);
      return 2.0 * B0 * std::cos(x2) / (r * r * r);
    });
    data.init_bg_B_field(1, [B0](Scalar x1, Scalar x2, Scalar) {
      Scalar r = std::exp(x1);
      return B0 * std::sin(x2) / (r * r * r);
    });
    data.init_bg_fields();
    data.fill_multiplicity(1.0f, 2);
    const size_t n0 = data.particles.number();
    for (uint32_t step = 0; step < (uint32_t)steps; ++step) {
      const double time = step * params.delta_t;
      const double omega = params.omega * std::fmin(time / 0.05, 1.0);
      pusher.update_particles(data, params.delta_t, step);
      solver.update_fields(data, params.delta_t, time);
      solver.apply_boundary(data, omega, time);
      if (step % params.sort_interval == 0 && step != 0) data.sort_particles();
    }
    ap_diag d{};
    ap_check(ap_diagnostics(env.ctx(), &d), "diagnostics");
    const bool ok = n0 == (size_t)128 * 64 * 4 && data.particles.number() > n0 / 2 &&
                    std::isfinite(d.kinetic) && std::isfinite(d.field_energy) &&
                    d.field_energy > 0.0;
    std::printf("particles %zu of %zu kinetic %.6e field_energy %.6e\n",
                data.particles.number(), n0, d.kinetic, d.field_energy);
    std::printf(ok ? "pulsar_lab ok\n" : "pulsar_lab FAILED\n");
    return ok ? 0 : 1;
  } catch (const ap_error &e) {
    std::printf("pulsar_lab error: %s\n", e.what());
    return 2;
  }
}

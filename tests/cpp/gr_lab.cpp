// A 1D GR lab written against the drop-in C++ headers the way the
// reference's 1dgr lab uses its algorithm classes (labs/1dgr/src/main.cpp):
// the field-line table the reference reads from coef.h5 (a synthetic one
// here), pairs from fill_multiplicity, then update_particles /
// update_fields, the lab's radiative transfer (inverse-Compton emission and
// gamma-gamma conversion from its tables) and a periodic sort. Exits 0 and
// prints "gr_lab ok" when the run is healthy.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "aperture/algorithms/field_solver_1dgr.h"
#include "aperture/algorithms/ptc_updater_1dgr.h"
#include "aperture/radiation/radiative_transfer.h"

using namespace Aperture;

int main(int argc, char **argv) {
  int steps = argc > 1 ? atoi(argv[1]) : 8;
  SimParams params;
  params.coord_system = "1DGR";
  params.N[0] = 4096;
  params.guard[0] = 3;
  params.lower[0] = -6.273f;
  params.size[0] = 6.138f;
  params.delta_t = 1.0e-3f;
  params.q_e = 1.2f;
  params.num_species = 2;
  params.current_smoothing = 2;
  params.sort_interval = 5;
  params.data_interval = 4;
  params.max_ptc_number = 4096 * 8;
  params.B0 = 1.0f;
  params.a = 0.99f;
  params.omega = 0.211765f;
  params.periodic_boundary[0] = false;
  // labs/1dgr/src/main.cpp: radiative_transfer with the lab's functions
  params.create_pairs = true;
  params.rad_model = AP_RAD_GR1D;
  params.max_photon_number = 4096 * 8;
  params.ic_path = 1.0e-3f;
  params.n_gamma = 200;
  params.n_ep = 200;
  // a field-line table: B^3 / B^1 large enough near the horizon that u_0
  // is real everywhere
  const int nt = 600;
  std::vector<float> r(nt), B1(nt), B3(nt), jr(nt), rho(nt), th(nt), dpsi(nt);
  const double a = params.a, om = params.omega;
  for (int i = 0; i < nt; ++i) {
    const double ri = 1.15 * std::pow(14.0 / 1.15, i / (nt - 1.0));
    const double t = 0.3 + 0.2 / ri;
    const double Sigma = ri * ri + a * a * std::cos(t) * std::cos(t);
    const double Delta = ri * ri - 2 * ri + a * a;
    const double A = (ri * ri + a * a) * (ri * ri + a * a) - Delta * a * a * std::sin(t) * std::sin(t);
    const double w = 2 * a * ri / A;
    const double g11 = Sigma / Delta, g33 = A * std::sin(t) * std::sin(t) / Sigma;
    const double al2 = Delta * Sigma / A;
    const double need = g11 * (g33 * (om - w) * (om - w) - al2) / (g33 * al2);
    const double b31 = 1.5 * std::sqrt(need > 0 ? need : 0.0) + 0.1;
    r[i] = (float)ri;
    B1[i] = (float)(1.0 / (ri * ri));
    B3[i] = (float)(b31 / (ri * ri));
    jr[i] = (float)(0.5 / (ri * ri));
    rho[i] = (float)(0.2 / (ri * ri));
    th[i] = (float)t;
    dpsi[i] = (float)(0.5 * std::sin(t));
  }
  ap_gr_table tab{r.data(), B1.data(), B3.data(), jr.data(), rho.data(), th.data(),
                  dpsi.data(), (size_t)nt};
  try {
    sim_environment env(params, -1, &tab);
    sim_data data(env);
    field_solver_1dgr solver(env);
    ptc_updater_1dgr pusher(env);
    radiative_transfer rad(env);
    data.E.initialize(0, [](double x, double, double) { return 0.05 * std::sin(3.0 * x); });
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
    const bool ok = n0 == (size_t)4096 * 4 && data.particles.number() > n0 / 2 &&
                    std::isfinite(d.kinetic) && std::isfinite(d.field_energy) &&
                    std::isfinite(d.max_abs_j) && d.max_abs_j > 0.0 && emitters > 0;
    std::printf("particles %zu of %zu field_energy %.6e max|J| %.6e emitters %llu\n",
                data.particles.number(), n0, d.field_energy, d.max_abs_j,
                (unsigned long long)emitters);
    std::printf(ok ? "gr_lab ok\n" : "gr_lab FAILED\n");
    return ok ? 0 : 1;
  } catch (const ap_error &e) {
    std::printf("gr_lab error: %s\n", e.what());
    return 2;
  }
}

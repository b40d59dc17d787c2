// A log-spherical lab written against the drop-in C++ headers the way the
// reference's pulsar lab uses the algorithm classes (labs/pulsar/src/
// main.cpp:63-140): dipole background B through init_bg_B_field, pairs from
// fill_multiplicity (given an outward momentum here), then update_particles
// / update_fields / apply_boundary with a spin-up of the star, photon
// emission and pair production with the pulsar lab's radiative functions,
// and a periodic sort. Exits 0 and prints "pulsar_lab ok" when the run is
// healthy.
#include <cmath>
#include <cstdio>

#include <vector>

#include "aperture/algorithms/field_solver_logsph.h"
#include "aperture/algorithms/ptc_updater_logsph.h"
#include "aperture/radiation/radiative_transfer.h"

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
  // curvature photons and their conversion (pulsar lab functions), with
  // constants that make them frequent on this small grid
  params.create_pairs = true;
  params.rad_model = AP_RAD_PULSAR;
  params.max_photon_number = 200000;
  params.e_curv = 1.0f;
  params.l_curv = 0.05f;
  params.BQ = 0.1f;
  params.r_cutoff = 4.0f;
  params.track_percent = 0.1f;
  try {
    sim_environment env(params);
    sim_data data(env);
    field_solver_logsph solver(env);
    ptc_updater_logsph pusher(env);
    radiative_transfer rad(env);
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
    {  // every particle moves outwards with p1 = 8
      std::vector<float> p1(n0, 8.0f), E(n0, std::sqrt(65.0f));
      particle_data &d = data.particles.data();
      cuda_check(cudaMemcpy(d.p1, p1.data(), 4 * n0, cudaMemcpyHostToDevice), "p1");
      cuda_check(cudaMemcpy(d.E, E.data(), 4 * n0, cudaMemcpyHostToDevice), "E");
      data.particles_modified();
    }
    uint64_t photons = 0, pairs = 0;
    for (uint32_t step = 0; step < (uint32_t)steps; ++step) {
      const double time = step * params.delta_t;
      const double omega = params.omega * std::fmin(time / 0.05, 1.0);
      pusher.update_particles(data, params.delta_t, step);
      solver.update_fields(data, params.delta_t, time);
      solver.apply_boundary(data, omega, time);
      rad.emit_photons(data);
      photons += rad.last_counts().written;
      rad.produce_pairs(data);
      pairs += rad.last_counts().written;
      if (step % params.sort_interval == 0 && step != 0) data.sort_particles();
    }
    ap_diag d{};
    ap_check(ap_diagnostics(env.ctx(), &d), "diagnostics");
    const bool ok = n0 == (size_t)128 * 64 * 4 && data.particles.number() > n0 / 2 &&
                    std::isfinite(d.kinetic) && std::isfinite(d.field_energy) &&
                    d.field_energy > 0.0 && photons > 0 && pairs > 0;
    std::printf("particles %zu of %zu kinetic %.6e field_energy %.6e photons %llu pairs %llu\n",
                data.particles.number(), n0, d.kinetic, d.field_energy,
                (unsigned long long)photons, (unsigned long long)pairs);
    std::printf(ok ? "pulsar_lab ok\n" : "pulsar_lab FAILED\n");
    return ok ? 0 : 1;
  } catch (const ap_error &e) {
    std::printf("pulsar_lab error: %s\n", e.what());
    return 2;
  }
}

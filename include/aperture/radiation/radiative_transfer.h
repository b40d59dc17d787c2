// radiative_transfer (src/radiation/radiative_transfer.h:11-29) on
// libaperture_b200.so: photon emission and pair production with the user
// radiative functions SimParams::rad_model selects (the reference chooses
// them at build time by lab shadowing). The environment's sim_data must have
// been created with SimParams::create_pairs set, so that its photons are
// bound; the photon move is part of ptc_updater::update_particles, as in the
// reference.
#ifndef APERTURE_DROPIN_RADIATIVE_TRANSFER_H_
#define APERTURE_DROPIN_RADIATIVE_TRANSFER_H_

#include "../sim_data.h"

namespace Aperture {

class radiative_transfer {
 public:
  explicit radiative_transfer(sim_environment &env) : m_env(env) { initialize(); }
  ~radiative_transfer() {}

  // user_rt_init and the model's parameters.
  void initialize() {
    const SimParams &p = m_env.params();
    ap_rad_params rp{};
    rp.model = p.rad_model;
    rp.delta_t = p.delta_t;
    rp.gamma_thr = p.gamma_thr;
    rp.E_secondary = p.E_secondary;
    rp.photon_path = p.photon_path;
    rp.r_cutoff = p.r_cutoff;
    rp.track_percent = p.track_percent;
    rp.e_curv = p.e_curv;
    rp.l_curv = p.l_curv;
    rp.BQ = p.BQ;
    rp.omega = p.omega;
    rp.seed = p.rad_seed;
    rp.first_photon_id = 1ull << 60;
    rp.first_particle_id = (1ull << 60) + (1ull << 59);
    rp.e_min = p.e_min;
    rp.ic_path = p.ic_path;
    rp.n_gamma = p.n_gamma;
    rp.n_ep = p.n_ep;
    ap_check(ap_set_rad_params(m_env.ctx(), &rp), "radiative_transfer");
  }

  // radiative_transfer::emit_photons (radiative_transfer.cu:196-243).
  void emit_photons(sim_data &data) {
    ap_rad_counts c{};
    ap_check(ap_emit_photons(m_env.ctx(), data.photon_produced.data().view(), &c),
             "emit_photons");
    size_t n = 0;
    ap_check(ap_get_photon_number(m_env.ctx(), &n), "get_photon_number");
    data.photons.set_num(n);
    m_last = c;
  }

  // radiative_transfer::produce_pairs (radiative_transfer.cu:245-301).
  void produce_pairs(sim_data &data) {
    ap_rad_counts c{};
    ap_check(ap_produce_pairs(m_env.ctx(), data.pair_produced.data().view(), &c),
             "produce_pairs");
    size_t n = 0;
    ap_check(ap_get_number(m_env.ctx(), &n), "get_number");
    data.particles.set_num(n);
    m_last = c;
  }

  // Counts of the last pass (new; the reference logs them).
  const ap_rad_counts &last_counts() const { return m_last; }

 private:
  sim_environment &m_env;
  ap_rad_counts m_last{};
};

}  // namespace Aperture

#endif

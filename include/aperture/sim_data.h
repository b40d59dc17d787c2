// sim_data (src/sim_data.h:14-70): the field arrays and the particle store
// of one rank, bound to the library context of a sim_environment.
#ifndef APERTURE_DROPIN_SIM_DATA_H_
#define APERTURE_DROPIN_SIM_DATA_H_

#include <cstring>
#include <random>
#include <vector>

#include "sim_environment.h"

namespace Aperture {

// particle_data (src/data/particle_data.h:50-61): device SoA pointers.
struct particle_data {
  Pos_t *x1, *x2, *x3;
  Scalar *p1, *p2, *p3, *E, *weight;
  uint32_t *cell;
  uint64_t *id;
  uint32_t *flag;
};

// particles_t (src/core/particles.h): fixed-capacity device SoA.
class particles_t {
 public:
  explicit particles_t(size_t capacity) : cap_(capacity ? capacity : 1) {
    auto alloc = [&](void **p, size_t b) { cuda_check(cudaMalloc(p, b * cap_), "particles"); };
    alloc((void **)&d_.x1, 4);
    alloc((void **)&d_.x2, 4);
    alloc((void **)&d_.x3, 4);
    alloc((void **)&d_.p1, 4);
    alloc((void **)&d_.p2, 4);
    alloc((void **)&d_.p3, 4);
    alloc((void **)&d_.E, 4);
    alloc((void **)&d_.weight, 4);
    alloc((void **)&d_.cell, 4);
    alloc((void **)&d_.id, 8);
    alloc((void **)&d_.flag, 4);
    cuda_check(cudaMemset(d_.cell, 0xff, 4 * cap_), "particles");  // MAX_CELL
    cuda_check(cudaMemset(d_.id, 0, 8 * cap_), "particles");
  }
  ~particles_t() {
    void *ps[] = {d_.x1, d_.x2, d_.x3, d_.p1, d_.p2, d_.p3, d_.E, d_.weight, d_.cell, d_.id, d_.flag};
    for (void *p : ps) cudaFree(p);
  }
  particles_t(const particles_t &) = delete;
  particles_t &operator=(const particles_t &) = delete;
  particle_data &data() { return d_; }
  size_t number() const { return num_; }
  size_t size() const { return cap_; }
  void set_num(size_t n) { num_ = n; }
  ap_particles view() const {
    return ap_particles{d_.x1, d_.x2, d_.x3, d_.p1, d_.p2, d_.p3, d_.E, d_.weight,
                        d_.cell, d_.id, d_.flag};
  }

 private:
  particle_data d_{};
  size_t num_ = 0, cap_;
};

// photon_data (src/data/particle_data.h:68-80): device SoA pointers.
struct photon_data {
  Pos_t *x1, *x2, *x3;
  Scalar *p1, *p2, *p3, *E, *weight, *path_left;
  uint32_t *cell;
  uint64_t *id;
  uint32_t *flag;
};

// photons_t (src/core/photons.h): fixed-capacity device SoA.
class photons_t {
 public:
  explicit photons_t(size_t capacity) : cap_(capacity ? capacity : 1) {
    auto alloc = [&](void **p, size_t b) { cuda_check(cudaMalloc(p, b * cap_), "photons"); };
    void **f[] = {(void **)&d_.x1, (void **)&d_.x2, (void **)&d_.x3, (void **)&d_.p1,
                  (void **)&d_.p2, (void **)&d_.p3, (void **)&d_.E, (void **)&d_.weight,
                  (void **)&d_.path_left, (void **)&d_.cell, (void **)&d_.flag};
    for (void **p : f) alloc(p, 4);
    alloc((void **)&d_.id, 8);
    cuda_check(cudaMemset(d_.cell, 0xff, 4 * cap_), "photons");  // MAX_CELL
  }
  ~photons_t() {
    void *ps[] = {d_.x1, d_.x2, d_.x3, d_.p1, d_.p2, d_.p3, d_.E, d_.weight, d_.path_left,
                  d_.cell, d_.id, d_.flag};
    for (void *p : ps) cudaFree(p);
  }
  photons_t(const photons_t &) = delete;
  photons_t &operator=(const photons_t &) = delete;
  photon_data &data() { return d_; }
  size_t number() const { return num_; }
  size_t size() const { return cap_; }
  void set_num(size_t n) { num_ = n; }
  ap_photons view() const {
    return ap_photons{d_.x1, d_.x2, d_.x3, d_.p1, d_.p2, d_.p3, d_.E, d_.weight, d_.path_left,
                      d_.cell, d_.id, d_.flag};
  }

 private:
  photon_data d_{};
  size_t num_ = 0, cap_;
};

struct sim_data {
  explicit sim_data(sim_environment &e)
      : env(e),
        particles((size_t)e.params().max_ptc_number),
        photons(e.params().create_pairs ? (size_t)e.params().max_photon_number : 1),
        num_species(e.params().num_species) {
    const Quadmesh &m = e.mesh();
    E.resize(m, FieldType::E);
    B.resize(m, FieldType::B);
    Ebg.resize(m, FieldType::E);
    Bbg.resize(m, FieldType::B);
    J.resize(m, FieldType::E);
    Rho.resize(num_species);
    for (auto &r : Rho) r.resize(m, FieldType::Scalar, 0b111);
    divE.resize(m, FieldType::Scalar, 0b111);
    divB.resize(m, FieldType::Scalar, 0b000);
    photon_produced.resize(m, FieldType::Scalar, 0b111);
    pair_produced.resize(m, FieldType::Scalar, 0b111);
    bind();
  }

  // sim_data::init_bg_B_field / init_bg_E_field (src/sim_data.h:23-37):
  // the background and the field itself start from f, guards refreshed.
  template <class Func>
  void init_bg_B_field(int component, const Func &f) {
    Bbg.initialize(component, f);
    B.initialize(component, f);
    env.send_array_guard_cells(Bbg.data(component));
    env.send_array_guard_cells(B.data(component));
  }
  template <class Func>
  void init_bg_E_field(int component, const Func &f) {
    Ebg.initialize(component, f);
    E.initialize(component, f);
    env.send_array_guard_cells(Ebg.data(component));
    env.send_array_guard_cells(E.data(component));
  }
  // The device keeps the background fields in Ebg / Bbg, which the kernels
  // read directly; nothing to upload (cuda/sim_data.cu:224-228).
  void init_bg_fields() {}

  // Tells the library that particle slots changed outside its calls (after
  // filling or editing them on the host or with other kernels).
  void particles_modified() {
    ap_check(ap_particles_modified(env.ctx(), particles.number()), "particles_modified");
  }

  // sim_data::fill_multiplicity (cuda/sim_data.cu:268-293): per bulk cell,
  // `multiplicity` e-/e+ pairs at one uniformly random position, at rest,
  // with the given weight, appended after the current number and sorted by
  // cell. The positions come from a seeded host generator (the reference
  // draws them with cuRAND).
  void fill_multiplicity(Scalar weight, int multiplicity, uint64_t seed = 0) {
    const Quadmesh &m = env.mesh();
    std::vector<uint32_t> cells;
    for (int c = 0; c < m.size(); ++c) {
      const int c1 = c % m.dims[0], c2 = (c / m.dims[0]) % m.dims[1];
      const int c3 = c / (m.dims[0] * m.dims[1]);
      const bool bulk = c1 >= m.guard[0] && c1 < m.dims[0] - m.guard[0] && c2 >= m.guard[1] &&
                        c2 < m.dims[1] - m.guard[1] && c3 >= m.guard[2] &&
                        c3 < m.dims[2] - m.guard[2];
      if (bulk) cells.push_back((uint32_t)c);
    }
    const size_t add = cells.size() * 2 * (size_t)multiplicity, n0 = particles.number();
    if (n0 + add > particles.size()) throw ap_error(AP_ERR_CAPACITY, "fill_multiplicity");
    std::vector<float> x1(add), x2(add), x3(add), zero(add, 0.0f), one(add, 1.0f), w(add, weight);
    std::vector<uint32_t> cell(add), flag(add);
    std::vector<uint64_t> id(add, 0);
    std::mt19937_64 gen(seed);
    std::uniform_real_distribution<float> u(0.0f, 1.0f);
    size_t k = 0;
    for (uint32_t c : cells)
      for (int n = 0; n < multiplicity; ++n, k += 2) {
        x1[k] = x1[k + 1] = u(gen);
        x2[k] = x2[k + 1] = u(gen);
        x3[k] = x3[k + 1] = u(gen);
        cell[k] = cell[k + 1] = c;
        flag[k] = 0u << 29;      // electron
        flag[k + 1] = 1u << 29;  // positron
      }
    particle_data &d = particles.data();
    auto up = [&](void *dst, const void *src, size_t b) {
      cuda_check(cudaMemcpy((char *)dst + n0 * b, src, add * b, cudaMemcpyHostToDevice), "fill");
    };
    up(d.x1, x1.data(), 4);
    up(d.x2, x2.data(), 4);
    up(d.x3, x3.data(), 4);
    up(d.p1, zero.data(), 4);
    up(d.p2, zero.data(), 4);
    up(d.p3, zero.data(), 4);
    up(d.E, one.data(), 4);
    up(d.weight, w.data(), 4);
    up(d.cell, cell.data(), 4);
    up(d.id, id.data(), 8);
    up(d.flag, flag.data(), 4);
    particles.set_num(n0 + add);
    particles_modified();
    sort_particles();
  }

  // sim_data::sort_particles (sim_data_impl.hpp:78-89).
  void sort_particles() {
    ap_check(ap_sort_by_cell(env.ctx()), "sort_particles");
    size_t n = 0;
    ap_check(ap_get_number(env.ctx(), &n), "get_number");
    particles.set_num(n);
  }

  sim_environment &env;
  vector_field<Scalar> E, B, Ebg, Bbg, J;
  std::vector<scalar_field<Scalar>> Rho;
  scalar_field<Scalar> divE, divB;
  particles_t particles;
  photons_t photons;  // bound to the library when SimParams::create_pairs is set
  scalar_field<Scalar> photon_produced, pair_produced;
  int num_species;

 private:
  void bind() {
    ap_fields f{};
    for (int i = 0; i < 3; ++i) {
      f.E[i] = E.data(i).view();
      f.B[i] = B.data(i).view();
      f.Ebg[i] = Ebg.data(i).view();
      f.Bbg[i] = Bbg.data(i).view();
      f.J[i] = J.data(i).view();
    }
    for (int s = 0; s < num_species; ++s) f.Rho[s] = Rho[s].data().view();
    f.divE = divE.data().view();
    f.divB = divB.data().view();
    ap_check(ap_bind_fields(env.ctx(), &f), "bind_fields");
    ap_particles p = particles.view();
    ap_check(ap_bind_particles(env.ctx(), &p, particles.number(), particles.size()),
             "bind_particles");
    if (env.params().create_pairs) {
      ap_photons ph = photons.view();
      ap_check(ap_bind_photons(env.ctx(), &ph, photons.number(), photons.size()),
               "bind_photons");
    }
  }
};

}  // namespace Aperture

#endif

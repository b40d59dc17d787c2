/*
 * Oracle pin build, radiation part (TEST INFRASTRUCTURE ONLY): runs the
 * reference's own user radiative functions on the host.
 *
 * Both user-function sets are compiled unmodified from the reference tree:
 * the framework's default src/cuda/radiation/user_radiative_functions.cu
 * (its four functions renamed with dflt_ prefixes by macros, since the
 * pulsar lab's file defines the same names) and the pulsar lab's
 * labs/pulsar/src/cuda/radiation/user_radiative_functions.cu. Both files
 * carry the same include guard, which is cleared between them. CudaRng
 * hands out queued uniforms (shim_rad/cuda/cudarng.h).
 *
 * The drivers restate the passes of radiative_transfer.cu (count, scan,
 * append: emit_photons :196-243, produce_pairs :245-301) with the build's
 * ordering, random draws, ids and capacity rules (oracle/ap_rad.c states
 * them), and call the reference's functions for everything per particle.
 */
#include "ls_host_math.h"
#include "cuda_builtins_host.h"
#include "core/constant_defs.h"
#include "core/typedefs.h"
#include "cuda/constant_mem.h"
#include "cuda/data_ptrs.h"
#include "cuda/cudarng.h"
#include "cuda/grids/grid_log_sph_ptrs.h"
#include "cuda/utils/interpolation.cuh"
#include "utils/util_functions.h"
#include "grids/grid_log_sph.h"
#include "sim_environment.h"

#include <cassert>

ap_ref_dim3 blockIdx, blockDim, threadIdx, gridDim;

/* user_rt_init of the pulsar lab copies its mesh pointers to the device;
 * the pin never calls it. */
#define CudaSafeCall(...) ((void)0)

namespace Aperture {
Quadmesh dev_mesh;
ap_ref_params dev_params;
float dev_charges[8];
float dev_masses[8];
int dev_rank = 0;
unsigned long long dev_ptc_id = 0;
mesh_ptrs_log_sph get_mesh_ptrs(Grid_LogSph &) { return mesh_ptrs_log_sph(); }
Grid &sim_environment::local_grid() {
  static Grid_LogSph g;
  return g;
}
namespace Kernels {
const float *ap_ref_rng_queue = nullptr;
int ap_ref_rng_left = 0;
int ap_ref_rng_underflow = 0;
}  // namespace Kernels
}  // namespace Aperture

#define check_emit_photon dflt_check_emit_photon
#define emit_photon dflt_emit_photon
#define check_produce_pair dflt_check_produce_pair
#define produce_pair dflt_produce_pair
#define user_rt_init dflt_user_rt_init
#include "cuda/radiation/user_radiative_functions.cu"
#undef check_emit_photon
#undef emit_photon
#undef check_produce_pair
#undef produce_pair
#undef user_rt_init
#undef _USER_RADIATIVE_FUNCTIONS_H_
#include "labs/pulsar/src/cuda/radiation/user_radiative_functions.cu"

using namespace Aperture;

extern "C" {

/* Same layouts as or_mesh, or_ptc, or_photons, or_fields and
 * or_rad_params (oracle/ap_oracle.h, oracle/ap_rad.h). */
typedef struct {
  int dims[3]; int guard[3];
  float delta[3]; float inv_delta[3]; float lower[3]; float sizes[3];
  int dimension;
} ref_mesh;
typedef struct {
  float *x1, *x2, *x3, *p1, *p2, *p3, *E, *weight;
  uint32_t *cell; uint64_t *id; uint32_t *flag;
} ref_ptc;
typedef struct {
  float *x1, *x2, *x3, *p1, *p2, *p3, *E, *weight, *path_left;
  uint32_t *cell; uint64_t *id; uint32_t *flag;
} ref_photons;
typedef struct {
  float *E[3], *B[3], *Ebg[3], *Bbg[3], *J[3];
  float *Rho[8];
  float *divE, *divB;
} ref_fields;
typedef struct {
  int model;
  float delta_t, gamma_thr, E_secondary, photon_path, r_cutoff, track_percent;
  float e_curv, l_curv, BQ, omega;
  uint64_t seed;
} ref_rad_params;
typedef struct {
  uint64_t marked, written, dropped;
} ref_rad_counts;

}  // extern "C"

static void set_mesh(const ref_mesh *m) {
  for (int i = 0; i < 3; i++) {
    dev_mesh.dims[i] = m->dims[i];
    dev_mesh.guard[i] = m->guard[i];
    dev_mesh.delta[i] = m->delta[i];
    dev_mesh.inv_delta[i] = m->inv_delta[i];
    dev_mesh.lower[i] = m->lower[i];
    dev_mesh.sizes[i] = m->sizes[i];
    dev_mesh.tileSize[i] = 1;
    dev_mesh.offset[i] = 0;
  }
  dev_mesh.dimension = m->dimension;
}

static void set_params(const ref_rad_params *rp) {
  dev_params.delta_t = rp->delta_t;
  dev_params.gamma_thr = rp->gamma_thr;
  dev_params.E_secondary = rp->E_secondary;
  dev_params.photon_path = rp->photon_path;
  dev_params.r_cutoff = rp->r_cutoff;
  dev_params.track_percent = rp->track_percent;
  dev_params.e_curv = rp->e_curv;
  dev_params.l_curv = rp->l_curv;
  dev_params.BQ = rp->BQ;
  dev_params.omega = rp->omega;
}

static pitchptr<Scalar> pp(float *a, const ref_mesh *m) {
  pitchptr<Scalar> r;
  r.p.ptr = a;
  r.p.pitch = (size_t)m->dims[0] * sizeof(float);
  r.p.xsize = (size_t)m->dims[0];
  r.p.ysize = (size_t)m->dims[1];
  return r;
}

static pitchptr<Scalar> g_rho[8];

static data_ptrs data_of(const ref_fields *f, const ref_mesh *m, const ref_ptc *p,
                         const ref_photons *ph) {
  data_ptrs d;
  d.E1 = pp(f->E[0], m); d.E2 = pp(f->E[1], m); d.E3 = pp(f->E[2], m);
  d.B1 = pp(f->B[0], m); d.B2 = pp(f->B[1], m); d.B3 = pp(f->B[2], m);
  d.Ebg1 = pp(f->Ebg[0], m); d.Ebg2 = pp(f->Ebg[1], m); d.Ebg3 = pp(f->Ebg[2], m);
  d.Bbg1 = pp(f->Bbg[0], m); d.Bbg2 = pp(f->Bbg[1], m); d.Bbg3 = pp(f->Bbg[2], m);
  d.J1 = pp(f->J[0], m); d.J2 = pp(f->J[1], m); d.J3 = pp(f->J[2], m);
  d.divE = pp(f->divE, m); d.divB = pp(f->divB, m);
  for (int s = 0; s < 2; s++) g_rho[s] = pp(f->Rho[s], m);
  d.Rho = g_rho;
  d.particles.x1 = p->x1; d.particles.x2 = p->x2; d.particles.x3 = p->x3;
  d.particles.p1 = p->p1; d.particles.p2 = p->p2; d.particles.p3 = p->p3;
  d.particles.E = p->E; d.particles.weight = p->weight;
  d.particles.cell = p->cell; d.particles.id = p->id; d.particles.flag = p->flag;
  d.photons.x1 = ph->x1; d.photons.x2 = ph->x2; d.photons.x3 = ph->x3;
  d.photons.p1 = ph->p1; d.photons.p2 = ph->p2; d.photons.p3 = ph->p3;
  d.photons.E = ph->E; d.photons.weight = ph->weight; d.photons.path_left = ph->path_left;
  d.photons.cell = ph->cell; d.photons.id = ph->id; d.photons.flag = ph->flag;
  return d;
}

static void queue(const float *u, int n) {
  Kernels::ap_ref_rng_queue = u;
  Kernels::ap_ref_rng_left = n;
}

static const uint32_t kTracked = 1u << 1;  // bit_or(ParticleFlag / PhotonFlag::tracked)

extern "C" {

/* emit_photons: count_photon_produced (:28-64) and produce_photons (:66-97)
 * in slot order; u4 holds the build's four uniforms of every particle slot
 * (the oracle's or_rad_uniforms). Returns 0, or -1 when a user function drew
 * more uniforms than the build gives it. */
int ref_rad_emit_photons(const ref_mesh *m, const ref_rad_params *rp, const ref_ptc *p,
                         size_t ptc_num, const ref_photons *ph, size_t *ph_num, size_t ph_cap,
                         const ref_fields *f, float *photon_produced, const float *u4,
                         uint64_t first_id, ref_rad_counts *out) {
  set_mesh(m);
  set_params(rp);
  Kernels::ap_ref_rng_underflow = 0;
  data_ptrs d = data_of(f, m, p, ph);
  curandState st{0};
  Kernels::CudaRng rng(&st);
  const size_t base = *ph_num;
  size_t rank = 0, written = 0;
  for (uint32_t tid = 0; tid < ptc_num; ++tid) {
    const uint32_t cell = p->cell[tid];
    if (cell == MAX_CELL) continue;
    if (!dev_mesh.is_in_bulk(cell)) continue;
    if (get_ptc_type(p->flag[tid]) == (int)ParticleType::ion) continue;
    const float *u = u4 + 4 * (size_t)tid;
    bool emit;
    if (rp->model == 0) {
      queue(u, 0);
      emit = Kernels::dflt_check_emit_photon(d, tid, rng);
    } else {
      queue(u, 1);
      emit = Kernels::check_emit_photon(d, tid, rng);
    }
    if (!emit) continue;
    if (photon_produced) {
      const int c1 = dev_mesh.get_c1(cell), c2 = dev_mesh.get_c2(cell);
      photon_produced[c1 + (size_t)c2 * m->dims[0]] += p->weight[tid];
    }
    const size_t off = base + rank;
    const uint64_t id = first_id + rank;
    rank++;
    if (off >= ph_cap) continue;
    ph->cell[off] = MAX_CELL;
    if (rp->model == 0) {
      queue(u, 2);
      Kernels::dflt_emit_photon(d, tid, (int)off, rng);
    } else {
      queue(u, 0);
      Kernels::emit_photon(d, tid, (int)off, rng);
    }
    ph->flag[off] = u[2] < dev_params.track_percent ? kTracked : 0u;
    ph->id[off] = id;
    written++;
  }
  const size_t n = base + rank + 1;
  *ph_num = n < ph_cap ? n : ph_cap;
  out->marked = rank;
  out->written = written;
  out->dropped = rank - written;
  return Kernels::ap_ref_rng_underflow ? -1 : 0;
}

/* produce_pairs: count_pairs_produced (:99-138) and produce_pairs
 * (:140-177) in slot order; u4 as above, per photon slot. */
int ref_rad_produce_pairs(const ref_mesh *m, const ref_rad_params *rp, const ref_photons *ph,
                          size_t ph_num, const ref_ptc *p, size_t *ptc_num, size_t ptc_cap,
                          const ref_fields *f, float *pair_produced, const float *u4,
                          uint64_t first_id, ref_rad_counts *out) {
  set_mesh(m);
  set_params(rp);
  Kernels::ap_ref_rng_underflow = 0;
  data_ptrs d = data_of(f, m, p, ph);
  curandState st{0};
  Kernels::CudaRng rng(&st);
  const size_t base = *ptc_num + 20;
  size_t rank = 0, written = 0;
  for (uint32_t tid = 0; tid < ph_num; ++tid) {
    const uint32_t cell = ph->cell[tid];
    if (cell == MAX_CELL || !dev_mesh.is_in_bulk(cell)) continue;
    queue(nullptr, 0);
    const bool pair = rp->model == 0 ? Kernels::dflt_check_produce_pair(d, tid, rng)
                                     : Kernels::check_produce_pair(d, tid, rng);
    if (!pair) continue;
    if (pair_produced) {
      const int c1 = dev_mesh.get_c1(cell), c2 = dev_mesh.get_c2(cell);
      pair_produced[c1 + (size_t)c2 * m->dims[0]] += ph->weight[tid];
    }
    const size_t off = base + 2 * rank;
    const uint64_t id = first_id + 2 * (uint64_t)rank;
    rank++;
    if (off + 1 >= ptc_cap) {
      ph->cell[tid] = MAX_CELL;
      continue;
    }
    const float *u = u4 + 4 * (size_t)tid;
    p->cell[off] = p->cell[off + 1] = MAX_CELL;
    p->flag[off] = p->flag[off + 1] = 0u;
    queue(nullptr, 0);
    if (rp->model == 0)
      Kernels::dflt_produce_pair(d, tid, (uint32_t)off, rng);
    else
      Kernels::produce_pair(d, tid, (uint32_t)off, rng);
    for (int k = 0; k < 2; ++k) {
      if (u[0] < dev_params.track_percent) p->flag[off + k] |= kTracked;
      p->id[off + k] = id + (uint64_t)k;
    }
    written++;
  }
  const size_t n = *ptc_num + 2 * rank + 50;
  *ptc_num = n < ptc_cap ? n : ptc_cap;
  out->marked = rank;
  out->written = written;
  out->dropped = rank - written;
  return Kernels::ap_ref_rng_underflow ? -1 : 0;
}

}  // extern "C"

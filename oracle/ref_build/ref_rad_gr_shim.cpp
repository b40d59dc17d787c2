/*
 * Oracle pin build, 1D GR radiation (TEST INFRASTRUCTURE ONLY): runs the
 * 1D GR lab's own user radiative functions on the host; built a second time
 * with AP_REF_GAP for the 1D gap lab's (labs/1dgap/src/cuda/radiation/
 * user_radiative_functions.cuh, which includes the same headers).
 *
 * labs/1dgr/src/cuda/radiation/user_radiative_functions.cuh is compiled
 * unmodified behind shim_rgr/ (CudaRng with its m_local_state, a no-op
 * inverse_compton for user_rt_init, which the pin never calls) and the
 * 1D GR shims; src/grids/grid_1dgr.cpp is the second translation unit, as
 * in the GR pin. The functions' inverse-Compton lookups are the reference's
 * own device functions (find_n_gamma, binary_search, gen_photon_e,
 * find_ic_rate, find_gg_rate, copied from src/cuda/radiation/rt_ic.cu into
 * oracle/_ref/ic_dev.inc by the Makefile), reading the tables the driver is
 * given (the oracle's, which tests/test_ic_oracle.py pins bit for bit to
 * the reference's own inverse_compton::init) through host stand-ins for
 * their __constant__ symbols; gen_photon_e draws from the same queue of
 * uniforms as CudaRng.
 *
 * The drivers restate the passes of radiative_transfer.cu as the rad pin
 * does (ref_rad_shim.cpp), with the build's draw order: emission test u0,
 * photon energy u1, tracking u2; conversion test u1, tracking u0.
 */
#include "rgr_host_math.h"
#include "cuda_builtins_host.h"
#include "core/constant_defs.h"
#include "core/typedefs.h"
#include "cuda/constant_mem.h"
#include "cuda/data_ptrs.h"
#include "cuda/utils/pitchptr.h"
#include "utils/logger.h"
#include "utils/util_functions.h"

#include <cassert>
#include <map>
#include <string>
#include <vector>

extern "C" {
#include "../ap_ic.h"
}

ap_ref_dim3 blockIdx, blockDim, threadIdx, gridDim;

#define CudaSafeCall(...) ((void)0)

namespace Aperture {
Quadmesh dev_mesh;
ap_ref_params dev_params;
float dev_charges[8];
float dev_masses[8];
int dev_rank = 0;
unsigned long long dev_ptc_id = 0;
unsigned long long dev_ph_id = 0;
/* the tables the shim HDF5 reader of grid_1dgr.cpp serves; unused here */
std::map<std::string, std::vector<float>> ref_gr_tables;
namespace Kernels {
const float *ap_ref_rng_queue = nullptr;
int ap_ref_rng_left = 0;
int ap_ref_rng_underflow = 0;
}  // namespace Kernels
}  // namespace Aperture

#include "cuda/cudarng.h"
#include "grids/grid_1dgr.h"

#include "cuda/radiation/rt_ic_dev.h"

#define MIN_GAMMA 1.01f  /* rt_ic.cu:14-18 */
#define MAX_GAMMA 1.0e15
#define MIN_EP 1.0e-10

namespace Aperture {
namespace Kernels {
/* host stand-ins for rt_ic.cu's __constant__ table symbols */
Scalar dev_ic_dep, dev_ic_dg, dev_ic_dlep;
cudaPitchedPtr dev_ic_dNde, dev_ic_dNde_thomson;
Scalar *dev_ic_rate, *dev_gg_rate, *dev_gammas;
#include "ic_dev.inc"
}  // namespace Kernels
}  // namespace Aperture

#ifdef AP_REF_GAP
#include "labs/1dgap/src/cuda/radiation/user_radiative_functions.cuh"
#else
#include "labs/1dgr/src/cuda/radiation/user_radiative_functions.cuh"
#endif

namespace Aperture {
Grid &sim_environment::local_grid() {
  static Grid_1dGR g;
  return g;
}
}  // namespace Aperture

using namespace Aperture;

extern "C" {

/* Same layouts as or_mesh, or_ptc, or_photons (oracle/ap_oracle.h,
 * oracle/ap_rad.h). */
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
/* The lab's metric arrays in the order of or_rad_gr (oracle/ap_rad.h). */
typedef struct {
  const float *alpha, *D1, *D2, *D3, *B3B1, *gamma_rr, *gamma_ff, *beta_phi, *theta;
  float a, omega;
  const or_ic_tables *ic;
} ref_gr;
typedef struct {
  uint64_t marked, written, dropped;
} ref_rad_counts;

}  // extern "C"

static void set_state(const ref_mesh *m, const ref_gr *g, float delta_t, float track_percent) {
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
  dev_params.delta_t = delta_t;
  dev_params.track_percent = track_percent;
  dev_params.a = g->a;
  dev_params.omega = g->omega;
#ifndef AP_REF_GAP
  Grid_1dGR::mesh_ptrs &mp = Kernels::dev_mesh_ptrs_1dgr;
  mp = Grid_1dGR::mesh_ptrs();
  mp.alpha = g->alpha;
  mp.D1 = g->D1;
  mp.D2 = g->D2;
  mp.D3 = g->D3;
  mp.B3B1 = g->B3B1;
  mp.gamma_rr = g->gamma_rr;
  mp.gamma_ff = g->gamma_ff;
  mp.beta_phi = g->beta_phi;
  mp.theta = g->theta;
#endif
  const or_ic_tables *t = g->ic;
  dev_params.n_gamma = t->n_gamma;
  Kernels::dev_ic_dep = t->dep;
  Kernels::dev_ic_dg = t->dg;
  Kernels::dev_ic_dlep = t->dlep;
  Kernels::dev_ic_rate = t->ic_rate;
  Kernels::dev_gg_rate = t->gg_rate;
  Kernels::dev_gammas = t->gammas;
  /* multi_array<Scalar> rows of n_ep entries (get_cudaPitchedPtr; the
     reference's binary_search takes xsize as the entry count) */
  Kernels::dev_ic_dNde.ptr = t->dNde;
  Kernels::dev_ic_dNde.pitch = (size_t)t->n_ep * sizeof(float);
  Kernels::dev_ic_dNde.xsize = (size_t)t->n_ep;
  Kernels::dev_ic_dNde.ysize = (size_t)t->n_gamma;
  Kernels::dev_ic_dNde_thomson = Kernels::dev_ic_dNde;
  Kernels::dev_ic_dNde_thomson.ptr = t->dNde_thomson;
  Kernels::ap_ref_rng_underflow = 0;
}

static data_ptrs data_of(const ref_ptc *p, const ref_photons *ph) {
  data_ptrs d;
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

static const uint32_t kTracked = 1u << 1;

extern "C" {

/* SimParams::e_min, which the 1D gap lab's emit_photon reads. */
void ref_rgr_set_e_min(float e_min) { dev_params.e_min = e_min; }

/* emit_photons with the lab's check_emit_photon / emit_photon, parents in
 * slot order; u4 holds the build's four uniforms of every particle slot.
 * Returns 0, or -1 when a function drew more uniforms than given. */
int ref_gr_emit_photons(const ref_mesh *m, const ref_gr *g, float delta_t, float track_percent,
                        const ref_ptc *p, size_t ptc_num, const ref_photons *ph, size_t *ph_num,
                        size_t ph_cap, const float *u4, uint64_t first_id, ref_rad_counts *out) {
  set_state(m, g, delta_t, track_percent);
  data_ptrs d = data_of(p, ph);
  curandState st{0};
  Kernels::CudaRng rng(&st);
  const size_t base = *ph_num;
  size_t rank = 0, written = 0;
  for (uint32_t tid = 0; tid < ptc_num; ++tid) {
    const uint32_t cell = p->cell[tid];
    if (cell == MAX_CELL || !dev_mesh.is_in_bulk(cell)) continue;
    if (get_ptc_type(p->flag[tid]) == (int)ParticleType::ion) continue;
    const float *u = u4 + 4 * (size_t)tid;
    queue(u, 1);
    if (!Kernels::check_emit_photon(d, tid, rng)) continue;
    const size_t off = base + rank;
    const uint64_t id = first_id + rank;
    rank++;
    if (off >= ph_cap) continue;
    ph->cell[off] = MAX_CELL;
    queue(u + 1, 2);
    Kernels::emit_photon(d, tid, (int)off, rng);
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

/* produce_pairs with the lab's check_produce_pair / produce_pair, photons
 * in slot order; u4 as above, per photon slot. */
int ref_gr_produce_pairs(const ref_mesh *m, const ref_gr *g, float delta_t,
                         float track_percent, const ref_photons *ph, size_t ph_num,
                         const ref_ptc *p, size_t *ptc_num, size_t ptc_cap, const float *u4,
                         uint64_t first_id, ref_rad_counts *out) {
  set_state(m, g, delta_t, track_percent);
  data_ptrs d = data_of(p, ph);
  curandState st{0};
  Kernels::CudaRng rng(&st);
  const size_t base = *ptc_num + 20;
  size_t rank = 0, written = 0;
  for (uint32_t tid = 0; tid < ph_num; ++tid) {
    const uint32_t cell = ph->cell[tid];
    if (cell == MAX_CELL || !dev_mesh.is_in_bulk(cell)) continue;
    const float *u = u4 + 4 * (size_t)tid;
    queue(u + 1, 1);
    if (!Kernels::check_produce_pair(d, tid, rng)) continue;
    const size_t off = base + 2 * rank;
    const uint64_t id = first_id + 2 * (uint64_t)rank;
    rank++;
    if (off + 1 >= ptc_cap) {
      ph->cell[tid] = MAX_CELL;
      continue;
    }
    p->cell[off] = p->cell[off + 1] = MAX_CELL;
    queue(u, 1);
    Kernels::produce_pair(d, tid, (uint32_t)off, rng);
    for (int k = 0; k < 2; ++k) p->id[off + k] = id + (uint64_t)k;
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

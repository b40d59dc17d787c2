/*
 * Oracle pin build (TEST INFRASTRUCTURE ONLY): the 1D gap lab's kernels run
 * on the host.
 *
 * The Makefile copies update_ptc_1dgap, filter_current1d, beta_phi and
 * update_photon_1dgap from
 * src/cuda/algorithms/ptc_updater_1dgap.cu and update_e_1dgap from
 * field_solver_1dgap.cu into oracle/_ref/ (extract_kernels.py; the rest of
 * that Kernels namespace draws its initial conditions from cuRAND) and
 * includes them unmodified behind the host stand-ins of shim/. Each launch
 * runs as one thread, so the grid-stride loops visit elements in order and
 * atomicAdd is an ordered plain add. The filter reads one element past
 * each end of its arrays; the drivers below give it zero padding there.
 */
#include "cuda_builtins_host.h"
#include "core/constant_defs.h"
#include "core/typedefs.h"
#include "cuda/constant_mem.h"
#include "cuda/data_ptrs.h"
#include "utils/util_functions.h"
#include "cuda/utils/interpolation.cuh"
#include <vector>

ap_ref_dim3 blockIdx, blockDim, threadIdx, gridDim;

namespace Aperture {
Quadmesh dev_mesh;
ap_ref_params dev_params;
float dev_charges[8];
float dev_masses[8];
namespace Kernels {
#include "gap_kernels.inc"
#include "gap_fs_kernels.inc"
}  // namespace Kernels
}  // namespace Aperture

using namespace Aperture;

extern "C" {
/* Same layouts as or_mesh / or_ptc in oracle/ap_oracle.h. */
typedef struct {
  int dims[3]; int guard[3];
  float delta[3]; float inv_delta[3]; float lower[3]; float sizes[3];
  int dimension;
} ref_mesh;
typedef struct {
  float *x1, *x2, *x3, *p1, *p2, *p3, *E, *weight;
  uint32_t *cell; uint64_t *id; uint32_t *flag;
} ref_ptc;
}

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

static pitchptr<Scalar> pp(float *a, const ref_mesh *m) {
  pitchptr<Scalar> r;
  r.p.ptr = a;
  r.p.pitch = (size_t)m->dims[0] * sizeof(float);
  r.p.xsize = (size_t)m->dims[0];
  r.p.ysize = (size_t)m->dims[1];
  return r;
}

static void one_thread() {
  blockIdx = {0, 0, 0};
  threadIdx = {0, 0, 0};
  blockDim = {1, 1, 1};
  gridDim = {1, 1, 1};
}

extern "C" {

void ref_gap_push_deposit(const ref_mesh *m, const ref_ptc *p, size_t num, float dt,
                          float *E3, float *J1, float *const Rho[8], int num_species,
                          const float charges[8], const float masses[8]) {
  set_mesh(m);
  for (int i = 0; i < 8; i++) { dev_charges[i] = charges[i]; dev_masses[i] = masses[i]; }
  data_ptrs d;
  d.E3 = pp(E3, m);
  d.J1 = pp(J1, m);
  pitchptr<Scalar> rho[8];
  for (int s = 0; s < num_species; s++) rho[s] = pp(Rho[s], m);
  d.Rho = rho;
  d.particles.x1 = p->x1; d.particles.x2 = p->x2; d.particles.x3 = p->x3;
  d.particles.p1 = p->p1; d.particles.p2 = p->p2; d.particles.p3 = p->p3;
  d.particles.E = p->E; d.particles.weight = p->weight;
  d.particles.cell = p->cell; d.particles.id = p->id; d.particles.flag = p->flag;
  one_thread();
  Kernels::update_ptc_1dgap(d, num, dt, 0);
}

/* filter_current1d over one row of dims[0] values, zero-padded at both ends. */
void ref_gap_filter(const ref_mesh *m, const float *j, float *tmp, int bnd_lower,
                    int bnd_upper) {
  set_mesh(m);
  const size_t n = (size_t)m->dims[0];
  std::vector<float> a(n + 2, 0.0f), b(n + 2, 0.0f);
  for (size_t i = 0; i < n; i++) a[i + 1] = j[i];
  one_thread();
  Kernels::filter_current1d(pp(a.data() + 1, m), pp(b.data() + 1, m), bnd_lower != 0,
                            bnd_upper != 0);
  for (size_t i = 0; i < n; i++) tmp[i] = b[i + 1];
}

void ref_gap_update_e(const ref_mesh *m, float *E1, float *J1, float j0, float dt) {
  set_mesh(m);
  one_thread();
  Kernels::update_e_1dgap(pp(E1, m), pp(J1, m), j0, dt);
}

}  // extern "C"

extern "C" {

/* Same layout as or_photons (oracle/ap_rad.h). */
typedef struct {
  float *x1, *x2, *x3, *p1, *p2, *p3, *E, *weight, *path_left;
  uint32_t *cell; uint64_t *id; uint32_t *flag;
} ref_photons;

/* update_photon_1dgap (ptc_updater_1dgap.cu:163-192) as one thread. */
void ref_gap_move_photons(const ref_mesh *m, const ref_photons *ph, size_t num, float dt,
                          uint32_t step) {
  set_mesh(m);
  photon_data d;
  d.x1 = ph->x1; d.x2 = ph->x2; d.x3 = ph->x3;
  d.p1 = ph->p1; d.p2 = ph->p2; d.p3 = ph->p3;
  d.E = ph->E; d.weight = ph->weight; d.path_left = ph->path_left;
  d.cell = ph->cell; d.id = ph->id; d.flag = ph->flag;
  one_thread();
  Kernels::update_photon_1dgap(d, num, dt, step);
}

}  // extern "C"

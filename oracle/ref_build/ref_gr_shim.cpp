/*
 * Oracle pin build (TEST INFRASTRUCTURE ONLY): the 1D GR lab's kernels and
 * its coefficient computation run on the host.
 *
 * The Makefile copies update_ptc_1dgr, filter_current1d and
 * update_photon_1dgr from src/cuda/algorithms/ptc_updater_1dgr.cu and update_e_1dgr from
 * field_solver_1dgr.cu into oracle/_ref/ (extract_kernels.py; the rest of
 * that Kernels namespace draws its initial conditions from cuRAND) and
 * includes them unmodified behind the host stand-ins of shim/.
 * src/grids/grid_1dgr.cpp (Grid_1dGR::compute_coef, host code in the
 * reference too) is compiled unmodified as a second translation unit, with
 * shim_gr/ standing in for its Grid base, array<T>, logger and the HDF5
 * reader, which serves the tables the driver registers. Each launch runs
 * as one thread, so the grid-stride loops visit elements in order and
 * atomicAdd is an ordered plain add. The filter reads one element past
 * each end of its arrays; the driver gives it zero padding there.
 */
#include "cuda_builtins_host.h"
#include "core/constant_defs.h"
#include "core/typedefs.h"
#include "cuda/constant_mem.h"
#include "cuda/data_ptrs.h"
#include "utils/util_functions.h"
#include "cuda/utils/interpolation.cuh"
#include "grids/grid_1dgr.h"
#include "utils/hdf_wrapper.h"
#include <cstring>
#include <vector>

ap_ref_dim3 blockIdx, blockDim, threadIdx, gridDim;

namespace Aperture {
Quadmesh dev_mesh;
ap_ref_params dev_params;
float dev_charges[8];
float dev_masses[8];
std::map<std::string, std::vector<float>> ref_gr_tables;
namespace Kernels {
#include "gr_kernels.inc"
#include "gr_fs_kernels.inc"
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

static void set_mesh(Quadmesh &q, const ref_mesh *m) {
  for (int i = 0; i < 3; i++) {
    q.dims[i] = m->dims[i];
    q.guard[i] = m->guard[i];
    q.delta[i] = m->delta[i];
    q.inv_delta[i] = m->inv_delta[i];
    q.lower[i] = m->lower[i];
    q.sizes[i] = m->sizes[i];
    q.tileSize[i] = 1;
    q.offset[i] = 0;
  }
  q.dimension = m->dimension;
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

/* mesh_ptrs order of Grid_1dGR (grid_1dgr.h:16-20) */
static Grid_1dGR::mesh_ptrs mesh_ptrs_of(const float *const co[15]) {
  Grid_1dGR::mesh_ptrs mp;
  mp.D1 = co[0]; mp.D2 = co[1]; mp.D3 = co[2]; mp.alpha = co[3]; mp.theta = co[4];
  mp.K1 = co[5]; mp.K1_j = co[6]; mp.j0 = co[7]; mp.agrr = co[8]; mp.agrf = co[9];
  mp.rho0 = co[10]; mp.gamma_rr = co[11]; mp.gamma_ff = co[12]; mp.beta_phi = co[13];
  mp.B3B1 = co[14];
  return mp;
}

extern "C" {

/* Grid_1dGR::compute_coef from the seven tables (names as in coef.h5). */
void ref_gr_coef(const ref_mesh *m, float a, float omega, float B0, const float *r,
                 const float *B1, const float *B3, const float *jr, const float *rho,
                 const float *th, const float *dpsidth, size_t n, float *const out[15]) {
  const char *names[7] = {"r", "Bu1", "Bu3", "ju1", "rho", "th", "dpsidth"};
  const float *src[7] = {r, B1, B3, jr, rho, th, dpsidth};
  for (int k = 0; k < 7; k++) ref_gr_tables[names[k]] = std::vector<float>(src[k], src[k] + n);
  Grid_1dGR g;
  set_mesh(g.m_mesh, m);
  SimParams p;
  p.omega = omega;
  p.a = a;
  p.B0 = B0;
  g.compute_coef(p);
  array<Scalar> *arr[15] = {&g.m_D1, &g.m_D2, &g.m_D3, &g.m_alpha, &g.m_theta,
                            &g.m_K1, &g.m_K1_j, &g.m_j0, &g.m_agrr, &g.m_agrf,
                            &g.m_rho0, &g.m_gamma_rr, &g.m_gamma_ff, &g.m_beta_phi, &g.m_B3B1};
  for (int k = 0; k < 15; k++)
    std::memcpy(out[k], arr[k]->data(), sizeof(float) * (size_t)m->dims[0]);
}

void ref_gr_push(const ref_mesh *m, const ref_ptc *p, size_t num, float dt, uint32_t step,
                 int data_interval, float a, float omega, float *E3, const float *const co[15],
                 float *J1, float *const Rho[8], int num_species, const float charges[8],
                 const float masses[8]) {
  set_mesh(dev_mesh, m);
  dev_params.a = a;
  dev_params.omega = omega;
  dev_params.data_interval = data_interval;
  for (int i = 0; i < 8; i++) { dev_charges[i] = charges[i]; dev_masses[i] = masses[i]; }
  data_ptrs d;
  d.E3 = pp(E3, m);
  d.J1 = pp(J1, m);
  pitchptr<Scalar> rhos[8];
  for (int s = 0; s < num_species; s++) rhos[s] = pp(Rho[s], m);
  d.Rho = rhos;
  d.particles.x1 = p->x1; d.particles.x2 = p->x2; d.particles.x3 = p->x3;
  d.particles.p1 = p->p1; d.particles.p2 = p->p2; d.particles.p3 = p->p3;
  d.particles.E = p->E; d.particles.weight = p->weight;
  d.particles.cell = p->cell; d.particles.id = p->id; d.particles.flag = p->flag;
  one_thread();
  Kernels::update_ptc_1dgr(d, num, mesh_ptrs_of(co), dt, step);
}

/* filter_current1d over one row of dims[0] values, j and k1 zero-padded at
 * both ends. */
void ref_gr_filter(const ref_mesh *m, const float *j, float *tmp, const float *k1,
                   int bnd_lower, int bnd_upper) {
  set_mesh(dev_mesh, m);
  const size_t n = (size_t)m->dims[0];
  std::vector<float> a(n + 2, 0.0f), b(n + 2, 0.0f), k(n + 2, 0.0f);
  for (size_t i = 0; i < n; i++) {
    a[i + 1] = j[i];
    k[i + 1] = k1[i];
  }
  one_thread();
  Kernels::filter_current1d(pp(a.data() + 1, m), pp(b.data() + 1, m), k.data() + 1,
                            bnd_lower != 0, bnd_upper != 0);
  for (size_t i = 0; i < n; i++) tmp[i] = b[i + 1];
}

void ref_gr_update_e(const ref_mesh *m, float *E1, float *J1, const float *const co[15],
                     float dt) {
  set_mesh(dev_mesh, m);
  one_thread();
  Kernels::update_e_1dgr(pp(E1, m), pp(E1, m), pp(J1, m), mesh_ptrs_of(co), dt);
}

}  // extern "C"

extern "C" {

/* Same layout as or_photons (oracle/ap_rad.h). */
typedef struct {
  float *x1, *x2, *x3, *p1, *p2, *p3, *E, *weight, *path_left;
  uint32_t *cell; uint64_t *id; uint32_t *flag;
} ref_photons;

/* update_photon_1dgr (ptc_updater_1dgr.cu:301-400) as one thread. */
void ref_gr_move_photons(const ref_mesh *m, const ref_photons *ph, size_t num, float dt,
                         uint32_t step, int data_interval, const float *const co[15]) {
  set_mesh(dev_mesh, m);
  dev_params.data_interval = data_interval;
  photon_data d;
  d.x1 = ph->x1; d.x2 = ph->x2; d.x3 = ph->x3;
  d.p1 = ph->p1; d.p2 = ph->p2; d.p3 = ph->p3;
  d.E = ph->E; d.weight = ph->weight; d.path_left = ph->path_left;
  d.cell = ph->cell; d.id = ph->id; d.flag = ph->flag;
  one_thread();
  Kernels::update_photon_1dgr(d, num, mesh_ptrs_of(co), dt, step);
}

}  // extern "C"

/*
 * Oracle pin build (TEST INFRASTRUCTURE ONLY): runs the reference's own
 * kernel bodies on the host.
 *
 * The Makefile extracts the `namespace Kernels { ... }` blocks of
 * src/cuda/algorithms/ptc_updater.cu (lines 19-740) and field_solver.cu
 * (lines 12-328) from the reference tree into oracle/_ref/ at build time and
 * includes them here unmodified, behind host stand-ins for the CUDA
 * built-ins (shim/). A kernel is called once per emulated (block, thread)
 * of the launch shape the reference's host code uses, sequentially, so the
 * grid-stride particle loops visit particles in index order and atomicAdd
 * becomes an ordered plain add. The extern "C" drivers below restate only
 * the launch shapes (ptc_updater.cu:766-793, field_solver.cu:365-503).
 */
#include "cuda_builtins_host.h"
#include "core/constant_defs.h"
#include "core/typedefs.h"
#include "cuda/constant_mem.h"
#include "cuda/data_ptrs.h"
#include "utils/util_functions.h"
#include "cuda/algorithms/ptc_updater_helper.cuh"
#include "cuda/algorithms/vay_push.cuh"

#ifdef AP_REF_MT
#include <omp.h>
#include <stdlib.h>
thread_local ap_ref_dim3 blockIdx, blockDim, threadIdx, gridDim;
#else
ap_ref_dim3 blockIdx, blockDim, threadIdx, gridDim;
#endif

namespace Aperture {
Quadmesh dev_mesh;
ap_ref_params dev_params;
float dev_charges[8];
float dev_masses[8];

#include "ptc_kernels.inc"
#include "fs_kernels.inc"
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

static particle_data to_pd(const ref_ptc *p) {
  particle_data d;
  d.x1 = p->x1; d.x2 = p->x2; d.x3 = p->x3;
  d.p1 = p->p1; d.p2 = p->p2; d.p3 = p->p3;
  d.E = p->E; d.weight = p->weight;
  d.cell = p->cell; d.id = p->id; d.flag = p->flag;
  return d;
}

/* Emulates a launch <<<grid, block>>> of a one-thread-per-cell kernel. */
template <typename F>
static void launch2(unsigned gx, unsigned gy, unsigned bx, unsigned by, F f) {
  gridDim = {gx, gy, 1};
  blockDim = {bx, by, 1};
  for (unsigned y = 0; y < gy; y++)
    for (unsigned x = 0; x < gx; x++)
      for (unsigned ty = 0; ty < by; ty++)
        for (unsigned tx = 0; tx < bx; tx++) {
          blockIdx = {x, y, 0};
          threadIdx = {tx, ty, 0};
          f();
        }
}

extern "C" {

void ref_push(const ref_mesh *m, const ref_ptc *p, size_t num, float dt,
              float *const F[6], const float charges[8],
              const float masses[8]) {
  set_mesh(m);
  for (int i = 0; i < 8; i++) { dev_charges[i] = charges[i]; dev_masses[i] = masses[i]; }
  data_ptrs d;
  d.E1 = pp(F[0], m); d.E2 = pp(F[1], m); d.E3 = pp(F[2], m);
  d.B1 = pp(F[3], m); d.B2 = pp(F[4], m); d.B3 = pp(F[5], m);
  d.particles = to_pd(p);
  one_thread();
  if (dev_mesh.dim() == 1)
    Kernels::ptc_push_cart_1d(d, num, dt);
  else
    Kernels::ptc_push_cart_2d(d, num, dt);
}

void ref_deposit(const ref_mesh *m, const ref_ptc *p, size_t num, float dt,
                 uint32_t step, int data_interval, float *const J[3],
                 float *const Rho[8], int num_species,
                 const float charges[8]) {
  set_mesh(m);
  dev_params.data_interval = data_interval;
  for (int i = 0; i < 8; i++) dev_charges[i] = charges[i];
  data_ptrs d;
  d.J1 = pp(J[0], m); d.J2 = pp(J[1], m); d.J3 = pp(J[2], m);
  pitchptr<Scalar> rho[8];
  for (int s = 0; s < num_species; s++) rho[s] = pp(Rho[s], m);
  d.Rho = rho;
  d.particles = to_pd(p);
  one_thread();
  if (dev_mesh.dim() == 1)
    Kernels::deposit_current_cart_1d(d, num, dt, step);
  else
    Kernels::deposit_current_cart_2d(d, num, dt, step);
}

/* field_solver::update_e_field / update_b_field / compute_divs launch
 * shapes: 1D blocks of 512, 2D blocks of 32 x 16 over the reduced dims. */
void ref_update_e(const ref_mesh *m, float *const E[3], float *const B[3],
                  float *const Bbg[3], float *const J[3], float dt) {
  set_mesh(m);
  auto e1 = pp(E[0], m), e2 = pp(E[1], m), e3 = pp(E[2], m);
  auto b1 = pp(B[0], m), b2 = pp(B[1], m), b3 = pp(B[2], m);
  auto b01 = pp(Bbg[0], m), b02 = pp(Bbg[1], m), b03 = pp(Bbg[2], m);
  auto j1 = pp(J[0], m), j2 = pp(J[1], m), j3 = pp(J[2], m);
  if (dev_mesh.dim() == 1)
    launch2((dev_mesh.reduced_dim(0) + 511) / 512, 1, 512, 1, [&] {
      Kernels::compute_e_update1d(e1, e2, e3, b1, b2, b3, b01, b02, b03, j1, j2, j3, dt);
    });
  else
    launch2((dev_mesh.reduced_dim(0) + 31) / 32, (dev_mesh.reduced_dim(1) + 15) / 16, 32, 16, [&] {
      Kernels::compute_e_update2d(e1, e2, e3, b1, b2, b3, b01, b02, b03, j1, j2, j3, dt);
    });
}

void ref_update_b(const ref_mesh *m, float *const E[3], float *const Ebg[3],
                  float *const B[3], float dt) {
  set_mesh(m);
  auto e1 = pp(E[0], m), e2 = pp(E[1], m), e3 = pp(E[2], m);
  auto e01 = pp(Ebg[0], m), e02 = pp(Ebg[1], m), e03 = pp(Ebg[2], m);
  auto b1 = pp(B[0], m), b2 = pp(B[1], m), b3 = pp(B[2], m);
  if (dev_mesh.dim() == 1)
    launch2((dev_mesh.reduced_dim(0) + 511) / 512, 1, 512, 1, [&] {
      Kernels::compute_b_update1d(e1, e2, e3, e01, e02, e03, b1, b2, b3, dt);
    });
  else
    launch2((dev_mesh.reduced_dim(0) + 31) / 32, (dev_mesh.reduced_dim(1) + 15) / 16, 32, 16, [&] {
      Kernels::compute_b_update2d(e1, e2, e3, e01, e02, e03, b1, b2, b3, dt);
    });
}

void ref_compute_divs(const ref_mesh *m, float *const E[3], float *const B[3],
                      float *const Ebg[3], float *const Bbg[3], float *divE,
                      float *divB) {
  set_mesh(m);
  auto e1 = pp(E[0], m), e2 = pp(E[1], m), e3 = pp(E[2], m);
  auto b1 = pp(B[0], m), b2 = pp(B[1], m), b3 = pp(B[2], m);
  auto e01 = pp(Ebg[0], m), e02 = pp(Ebg[1], m), e03 = pp(Ebg[2], m);
  auto b01 = pp(Bbg[0], m), b02 = pp(Bbg[1], m), b03 = pp(Bbg[2], m);
  auto de = pp(divE, m), db = pp(divB, m);
  if (dev_mesh.dim() == 1)
    launch2((dev_mesh.reduced_dim(0) + 511) / 512, 1, 512, 1, [&] {
      Kernels::compute_divs_1d(e1, e2, e3, b1, b2, b3, e01, e02, e03, b01, b02, b03, de, db);
    });
  else
    launch2((dev_mesh.reduced_dim(0) + 31) / 32, (dev_mesh.reduced_dim(1) + 15) / 16, 32, 16, [&] {
      Kernels::compute_divs_2d(e1, e2, e3, b1, b2, b3, e01, e02, e03, b01, b02, b03, de, db);
    });
}

/* ptc_updater::smooth_current(multi_array&) (ptc_updater.cu:875-912) for
 * one array: filter into tmp, then copy tmp back over the whole array. */
void ref_filter(const ref_mesh *m, float *j, float *tmp, const int bnd[4]) {
  set_mesh(m);
  auto a = pp(j, m), t = pp(tmp, m);
  if (dev_mesh.dim() == 1)
    launch2((dev_mesh.reduced_dim(0) + 511) / 512, 1, 512, 1, [&] {
      Kernels::filter_current_cart_1d(a, t, bnd[0], bnd[1]);
    });
  else
    launch2((dev_mesh.reduced_dim(0) + 31) / 32, (dev_mesh.reduced_dim(1) + 15) / 16, 32, 16, [&] {
      Kernels::filter_current_cart_2d(a, t, bnd[0], bnd[1], bnd[2], bnd[3]);
    });
  size_t n = (size_t)m->dims[0] * m->dims[1] * m->dims[2];
  for (size_t i = 0; i < n; i++) j[i] = tmp[i];
}

#ifdef AP_REF_MT
/* Timing build (libapref_mt.so): the same kernels on all host threads.
 * Each thread runs the push and the deposit as a one-thread launch over a
 * contiguous slice of the particles; the deposit of each thread goes to a
 * private current / charge buffer (the kernels' atomicAdd is a plain add)
 * and the buffers are summed in thread order afterwards. */
static ref_ptc slice(const ref_ptc *p, size_t lo) {
  ref_ptc s = *p;
  s.x1 += lo; s.x2 += lo; s.x3 += lo;
  s.p1 += lo; s.p2 += lo; s.p3 += lo;
  s.E += lo; s.weight += lo; s.cell += lo; s.id += lo; s.flag += lo;
  return s;
}

void ref_push_mt(const ref_mesh *m, const ref_ptc *p, size_t num, float dt,
                 float *const F[6], const float charges[8], const float masses[8],
                 int nthreads) {
  /* the mesh and charges are process globals, set before the threads start */
  set_mesh(m);
  for (int i = 0; i < 8; i++) { dev_charges[i] = charges[i]; dev_masses[i] = masses[i]; }
#pragma omp parallel num_threads(nthreads)
  {
    const int t = omp_get_thread_num(), nt = omp_get_num_threads();
    const size_t lo = num * (size_t)t / nt, hi = num * (size_t)(t + 1) / nt;
    const ref_ptc s = slice(p, lo);
    data_ptrs d;
    d.E1 = pp(F[0], m); d.E2 = pp(F[1], m); d.E3 = pp(F[2], m);
    d.B1 = pp(F[3], m); d.B2 = pp(F[4], m); d.B3 = pp(F[5], m);
    d.particles = to_pd(&s);
    one_thread();
    if (dev_mesh.dim() == 1)
      Kernels::ptc_push_cart_1d(d, hi - lo, dt);
    else
      Kernels::ptc_push_cart_2d(d, hi - lo, dt);
  }
}

void ref_deposit_mt(const ref_mesh *m, const ref_ptc *p, size_t num, float dt,
                    uint32_t step, int data_interval, float *const J[3],
                    float *const Rho[8], int num_species, const float charges[8],
                    int nthreads) {
  set_mesh(m);
  dev_params.data_interval = data_interval;
  for (int i = 0; i < 8; i++) dev_charges[i] = charges[i];
  const size_t ncell = (size_t)m->dims[0] * m->dims[1] * m->dims[2];
  const int ncomp = 3 + num_species;
  float *priv = (float *)calloc((size_t)nthreads * ncomp * ncell, sizeof(float));
  if (!priv) return;
#pragma omp parallel num_threads(nthreads)
  {
    const int t = omp_get_thread_num(), nt = omp_get_num_threads();
    const size_t lo = num * (size_t)t / nt, hi = num * (size_t)(t + 1) / nt;
    const ref_ptc s = slice(p, lo);
    float *base = priv + (size_t)t * ncomp * ncell;
    data_ptrs d;
    d.J1 = pp(base, m); d.J2 = pp(base + ncell, m); d.J3 = pp(base + 2 * ncell, m);
    pitchptr<Scalar> rho[8];
    for (int sp = 0; sp < num_species; sp++) rho[sp] = pp(base + (3 + sp) * ncell, m);
    d.Rho = rho;
    d.particles = to_pd(&s);
    one_thread();
    if (dev_mesh.dim() == 1)
      Kernels::deposit_current_cart_1d(d, hi - lo, dt, step);
    else
      Kernels::deposit_current_cart_2d(d, hi - lo, dt, step);
  }
  for (int t = 0; t < nthreads; t++) {
    const float *base = priv + (size_t)t * ncomp * ncell;
#pragma omp parallel for num_threads(nthreads)
    for (size_t i = 0; i < ncell; i++) {
      for (int c = 0; c < 3; c++) J[c][i] += base[c * ncell + i];
      for (int sp = 0; sp < num_species; sp++) Rho[sp][i] += base[(3 + sp) * ncell + i];
    }
  }
  free(priv);
}
#endif

/* Same layout as or_photons (oracle/ap_rad.h). */
typedef struct {
  float *x1, *x2, *x3, *p1, *p2, *p3, *E, *weight, *path_left;
  uint32_t *cell; uint64_t *id; uint32_t *flag;
} ref_photons;

/* move_photons_cart_1d / _2d<<<256, 512>>> (ptc_updater.cu:627-690,
 * launched at :822-831), one emulated thread. The MPI exchange that follows
 * (send_particles) is not compiled; the caller applies the wrap. */
void ref_move_photons_cart(const ref_mesh *m, const ref_photons *ph, size_t num, float dt) {
  set_mesh(m);
  photon_data d;
  d.x1 = ph->x1; d.x2 = ph->x2; d.x3 = ph->x3;
  d.p1 = ph->p1; d.p2 = ph->p2; d.p3 = ph->p3;
  d.E = ph->E; d.weight = ph->weight; d.path_left = ph->path_left;
  d.cell = ph->cell; d.id = ph->id; d.flag = ph->flag;
  one_thread();
  if (m->dimension == 1)
    Kernels::move_photons_cart_1d(d, num, dt);
  else
    Kernels::move_photons_cart_2d(d, num, dt);
}

}  // extern "C"

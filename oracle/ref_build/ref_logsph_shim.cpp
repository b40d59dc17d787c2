/*
 * Oracle pin build, log-spherical part (TEST INFRASTRUCTURE ONLY): runs the
 * reference's own log-spherical code on the host.
 *
 * The Makefile extracts the `namespace Kernels { ... }` blocks of
 * src/cuda/algorithms/ptc_updater_logsph.cu (lines 20-668) and
 * field_solver_logsph.cu (lines 14-347) into oracle/_ref/ at build time and
 * includes them here unmodified, after the reference's
 * user_push_2d_logsph.cuh, behind host stand-ins for the CUDA built-ins
 * (shim/, shim_ls/). src/grids/grid_log_sph.cpp (Grid_LogSph::compute_coef,
 * host code in the reference too) is compiled unmodified as a second
 * translation unit. Each kernel runs once per emulated (block, thread) of
 * the launch shape the reference's host code uses, sequentially, so
 * grid-stride loops visit elements in index order and atomicAdd is an
 * ordered plain add. The extern "C" drivers restate only the launch shapes
 * (ptc_updater_logsph.cu:681-836, field_solver_logsph.cu:354-428).
 */
#include "ls_host_math.h"
#include "cuda_builtins_host.h"
#include "core/constant_defs.h"
#include "core/typedefs.h"
#include "cuda/constant_mem.h"
#include "cuda/data_ptrs.h"
#include "cuda/grids/grid_log_sph_ptrs.h"
#include "utils/util_functions.h"
#include "cuda/algorithms/ptc_updater_helper.cuh"
#include "cuda/algorithms/user_push_2d_logsph.cuh"
#include "grids/grid_log_sph.h"

ap_ref_dim3 blockIdx, blockDim, threadIdx, gridDim;

namespace Aperture {
Quadmesh dev_mesh;
ap_ref_params dev_params;
float dev_charges[8];
float dev_masses[8];
int dev_rank = 0;
unsigned long long dev_ptc_id = 0;

#include "ptc_logsph_kernels.inc"
#include "fs_logsph_kernels.inc"
}  // namespace Aperture

using namespace Aperture;

extern "C" {

/* Same layouts as or_mesh / or_ptc (oracle/ap_oracle.h) and or_ls_params
 * (oracle/ap_logsph.h). */
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
  float compactness, omega, gravity, rad_cooling_coef, B0, damping_coef;
  int rad_cooling_on, damping_length;
} ref_ls_params;

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

static void set_params(const ref_ls_params *lp, int data_interval, int num_species) {
  dev_params.data_interval = data_interval;
  dev_params.num_species = num_species;
  dev_params.compactness = lp->compactness;
  dev_params.omega = lp->omega;
  dev_params.gravity = lp->gravity;
  dev_params.rad_cooling_coef = lp->rad_cooling_coef;
  dev_params.B0 = lp->B0;
  dev_params.damping_coef = lp->damping_coef;
  dev_params.rad_cooling_on = lp->rad_cooling_on != 0;
  dev_params.damping_length = lp->damping_length;
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

static particle_data to_pd(const ref_ptc *p) {
  particle_data d;
  d.x1 = p->x1; d.x2 = p->x2; d.x3 = p->x3;
  d.p1 = p->p1; d.p2 = p->p2; d.p3 = p->p3;
  d.E = p->E; d.weight = p->weight;
  d.cell = p->cell; d.id = p->id; d.flag = p->flag;
  return d;
}

static mesh_ptrs_log_sph mesh_ptrs_of(float *const c[13], const ref_mesh *m) {
  mesh_ptrs_log_sph r;
  r.l1_e = pp(c[0], m); r.l2_e = pp(c[1], m); r.l3_e = pp(c[2], m);
  r.l1_b = pp(c[3], m); r.l2_b = pp(c[4], m); r.l3_b = pp(c[5], m);
  r.A1_e = pp(c[6], m); r.A2_e = pp(c[7], m); r.A3_e = pp(c[8], m);
  r.A1_b = pp(c[9], m); r.A2_b = pp(c[10], m); r.A3_b = pp(c[11], m);
  r.dV = pp(c[12], m);
  return r;
}

/* data_ptrs over field arrays in the order E[3], B[3], Ebg[3], Bbg[3], J[3],
 * Rho[8], divE, divB (or_fields). */
struct ref_fields {
  float *E[3], *B[3], *Ebg[3], *Bbg[3], *J[3];
  float *Rho[8];
  float *divE, *divB;
};

static pitchptr<Scalar> g_rho[8];

static data_ptrs data_of(const ref_fields *f, const ref_mesh *m, int num_species) {
  data_ptrs d;
  d.E1 = pp(f->E[0], m); d.E2 = pp(f->E[1], m); d.E3 = pp(f->E[2], m);
  d.B1 = pp(f->B[0], m); d.B2 = pp(f->B[1], m); d.B3 = pp(f->B[2], m);
  d.Ebg1 = pp(f->Ebg[0], m); d.Ebg2 = pp(f->Ebg[1], m); d.Ebg3 = pp(f->Ebg[2], m);
  d.Bbg1 = pp(f->Bbg[0], m); d.Bbg2 = pp(f->Bbg[1], m); d.Bbg3 = pp(f->Bbg[2], m);
  d.J1 = pp(f->J[0], m); d.J2 = pp(f->J[1], m); d.J3 = pp(f->J[2], m);
  d.divE = pp(f->divE, m); d.divB = pp(f->divB, m);
  for (int s = 0; s < num_species; s++) g_rho[s] = pp(f->Rho[s], m);
  d.Rho = g_rho;
  return d;
}

extern "C" {

/* Grid_LogSph::compute_coef (grid_log_sph.cpp:11-126), unmodified. */
void ref_ls_coef(const ref_mesh *m, float *const out[13]) {
  Grid_LogSph g;
  for (int i = 0; i < 3; i++) {
    g.m_mesh.dims[i] = m->dims[i];
    g.m_mesh.guard[i] = m->guard[i];
    g.m_mesh.delta[i] = m->delta[i];
    g.m_mesh.inv_delta[i] = m->inv_delta[i];
    g.m_mesh.lower[i] = m->lower[i];
    g.m_mesh.sizes[i] = m->sizes[i];
    g.m_mesh.tileSize[i] = 1;
    g.m_mesh.offset[i] = 0;
  }
  g.m_mesh.dimension = m->dimension;
  SimParams params;
  g.compute_coef(params);
  const multi_array<Scalar> *arr[13] = {&g.m_l1_e, &g.m_l2_e, &g.m_l3_e, &g.m_l1_b, &g.m_l2_b,
                                        &g.m_l3_b, &g.m_A1_e, &g.m_A2_e, &g.m_A3_e, &g.m_A1_b,
                                        &g.m_A2_b, &g.m_A3_b, &g.m_dV};
  size_t n = (size_t)m->dims[0] * m->dims[1];
  for (int k = 0; k < 13; k++)
    for (size_t o = 0; o < n; o++) out[k][o] = arr[k]->m_v[o];
}

/* vay_push_logsph_2d<<<512, 256>>> (ptc_updater_logsph.cu:701-703), one
 * emulated thread. */
void ref_ls_push(const ref_mesh *m, const ref_ls_params *lp, const ref_ptc *p, size_t num,
                 float dt, float *const F[6], const float charges[8], const float masses[8]) {
  set_mesh(m);
  set_params(lp, 1, 3);
  for (int i = 0; i < 8; i++) { dev_charges[i] = charges[i]; dev_masses[i] = masses[i]; }
  data_ptrs d;
  d.E1 = pp(F[0], m); d.E2 = pp(F[1], m); d.E3 = pp(F[2], m);
  d.B1 = pp(F[3], m); d.B2 = pp(F[4], m); d.B3 = pp(F[5], m);
  d.particles = to_pd(p);
  curandState st{12345};
  one_thread();
  Kernels::vay_push_logsph_2d(d, num, dt, &st);
}

/* measure_surface_density<<<256, 512>>> (ptc_updater_logsph.cu:441-490,
 * launched at :856-858), one emulated thread; se / sp hold
 * dims1 - 2 guard1 floats. */
void ref_ls_surface_density(const ref_mesh *m, const ref_ptc *p, size_t num, float *se,
                            float *sp) {
  set_mesh(m);
  one_thread();
  Kernels::measure_surface_density(to_pd(p), num, se, sp);
}

/* deposit_and_move_2d_log_sph<1> (ptc_updater_logsph.cu:715-718). */
void ref_ls_deposit(const ref_mesh *m, const ref_ls_params *lp, const ref_ptc *p, size_t num,
                    float dt, uint32_t step, int data_interval, float *const J[3],
                    float *const Rho[8], int num_species, float *const coef[13],
                    const float charges[8]) {
  set_mesh(m);
  set_params(lp, data_interval, num_species);
  for (int i = 0; i < 8; i++) dev_charges[i] = charges[i];
  data_ptrs d;
  d.J1 = pp(J[0], m); d.J2 = pp(J[1], m); d.J3 = pp(J[2], m);
  for (int s = 0; s < num_species; s++) g_rho[s] = pp(Rho[s], m);
  d.Rho = g_rho;
  d.particles = to_pd(p);
  one_thread();
  Kernels::deposit_and_move_2d_log_sph<1>(d, num, mesh_ptrs_of(coef, m), dt, step, true, true);
}

/* process_j, axis_rho_lower / upper, ptc_outflow. */
void ref_ls_process_j(const ref_mesh *m, float *const J[3], float *const Rho[8], int num_species,
                      float *const coef[13], float dt) {
  set_mesh(m);
  dev_params.num_species = num_species;
  data_ptrs d;
  d.J1 = pp(J[0], m); d.J2 = pp(J[1], m); d.J3 = pp(J[2], m);
  for (int s = 0; s < num_species; s++) g_rho[s] = pp(Rho[s], m);
  d.Rho = g_rho;
  one_thread();
  Kernels::process_j(d, mesh_ptrs_of(coef, m), dt);
}

void ref_ls_axis_rho(const ref_mesh *m, float *J3, float *const coef[13]) {
  set_mesh(m);
  data_ptrs d;
  d.J3 = pp(J3, m);
  one_thread();
  Kernels::axis_rho_lower(d, mesh_ptrs_of(coef, m));
  Kernels::axis_rho_upper(d, mesh_ptrs_of(coef, m));
}

void ref_ls_ptc_outflow(const ref_mesh *m, const ref_ls_params *lp, const ref_ptc *p, size_t num) {
  set_mesh(m);
  set_params(lp, 1, 3);
  one_thread();
  Kernels::ptc_outflow(to_pd(p), num);
}

/* filter_current_logsph over (reduced / 32, reduced / 16) blocks of
 * 32 x 16, all four boundaries; writes tmp only. */
void ref_ls_filter(const ref_mesh *m, float *j, float *tmp, float *A) {
  set_mesh(m);
  auto a = pp(j, m), t = pp(tmp, m), w = pp(A, m);
  launch2(dev_mesh.reduced_dim(0) / 32, dev_mesh.reduced_dim(1) / 16, 32, 16,
          [&] { Kernels::filter_current_logsph(a, t, w, true, true, true, true); });
}

/* field_solver_logsph::update_fields: compute_b, compute_e, compute_divs
 * over (reduced / 32, reduced / 16) blocks of 32 x 16. */
void ref_ls_update_fields(const ref_mesh *m, const ref_ls_params *lp, const ref_fields *f,
                          float *const coef[13], float dt) {
  set_mesh(m);
  set_params(lp, 1, 3);
  data_ptrs d = data_of(f, m, 0);
  mesh_ptrs_log_sph mp = mesh_ptrs_of(coef, m);
  unsigned gx = dev_mesh.reduced_dim(0) / 32, gy = dev_mesh.reduced_dim(1) / 16;
  launch2(gx, gy, 32, 16, [&] { Kernels::compute_b_update_logsph(d, mp, dt); });
  launch2(gx, gy, 32, 16, [&] { Kernels::compute_e_update_logsph(d, mp, dt); });
  launch2(gx, gy, 32, 16, [&] { Kernels::compute_divs_logsph(d, mp); });
}

/* field_solver_logsph::apply_boundary(data, omega, time), one rank: all
 * four boundaries, each kernel with one emulated thread. */
void ref_ls_field_boundary(const ref_mesh *m, const ref_ls_params *lp, const ref_fields *f,
                           float omega) {
  set_mesh(m);
  set_params(lp, 1, 3);
  data_ptrs d = data_of(f, m, 0);
  one_thread();
  Kernels::stellar_boundary(d, omega);
  Kernels::outflow_boundary_sph(d);
  Kernels::axis_boundary_lower(d);
  Kernels::axis_boundary_upper(d);
}

/* Same layout as or_photons (oracle/ap_rad.h). */
typedef struct {
  float *x1, *x2, *x3, *p1, *p2, *p3, *E, *weight, *path_left;
  uint32_t *cell; uint64_t *id; uint32_t *flag;
} ref_photons;

/* move_photons<<<256, 512>>> (ptc_updater_logsph.cu:58-131, launched at
 * :797-800), one emulated thread. send_particles and clear_guard_cells
 * that follow are not compiled; the caller removes what left the bulk. */
void ref_ls_move_photons(const ref_mesh *m, float r_cutoff, const ref_photons *ph, size_t num,
                         float dt) {
  set_mesh(m);
  dev_params.r_cutoff = r_cutoff;
  photon_data d;
  d.x1 = ph->x1; d.x2 = ph->x2; d.x3 = ph->x3;
  d.p1 = ph->p1; d.p2 = ph->p2; d.p3 = ph->p3;
  d.E = ph->E; d.weight = ph->weight; d.path_left = ph->path_left;
  d.cell = ph->cell; d.id = ph->id; d.flag = ph->flag;
  one_thread();
  Kernels::move_photons(d, num, dt, true, true);
}

}  // extern "C"

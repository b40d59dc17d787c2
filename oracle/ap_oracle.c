/*
 * CPU oracle for the Aperture3 particle update (TEST INFRASTRUCTURE ONLY).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
 * it, as the checker. See ap_oracle.h for conventions.
 *
 * Every function cites the reference file:line it restates. Build with
 * -ffp-contract=off (oracle/Makefile) so no multiply-add is fused.
 */
#include "ap_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ParticleFlag bits (src/core/enum_types.h:76-87) and the species field in
 * the top 3 bits of the flag (src/utils/util_functions.h:29-33, 66-69). */
#define FLAG_IGNORE_CURRENT (1u << 3)
#define FLAG_IGNORE_EM (1u << 4)
static inline int ptc_type(uint32_t flag) { return (int)(flag >> 29); }

/* spline_t<1>, cloud-in-cell (src/cuda/utils/interpolation.cuh:28-37). */
static inline float cic(float dx) {
  float a = fabsf(dx);
  float w = 1.0f - a;
  return w > 0.0f ? w : 0.0f;
}

/* interp_cell (interpolation.cuh:79-87): distance from the particle at
 * c + rel to the node of cell t, which sits at t + 0.5 (stagger 0) or
 * t + 1 (stagger 1). */
static inline float interp_cell(float rel, int c, int t, int stagger) {
  float x = ((float)t + (stagger == 0 ? 0.5f : 1.0f)) - (rel + (float)c);
  return cic(x);
}

/* Quadmesh helpers (quadmesh.h:200-251). */
static inline uint32_t get_c1(const or_mesh *m, uint32_t c) {
  return c % (uint32_t)m->dims[0];
}
static inline uint32_t get_c2(const or_mesh *m, uint32_t c) {
  return (c / (uint32_t)m->dims[0]) % (uint32_t)m->dims[1];
}
static inline uint32_t get_c3(const or_mesh *m, uint32_t c) {
  return c / ((uint32_t)m->dims[0] * (uint32_t)m->dims[1]);
}
static inline int in_bulk3(const or_mesh *m, int c1, int c2, int c3) {
  return (c1 >= m->guard[0] && c1 < m->dims[0] - m->guard[0]) &&
         (c2 >= m->guard[1] && c2 < m->dims[1] - m->guard[1]) &&
         (c3 >= m->guard[2] && c3 < m->dims[2] - m->guard[2]);
}
static inline int in_bulk(const or_mesh *m, uint32_t c) {
  return in_bulk3(m, (int)get_c1(m, c), (int)get_c2(m, c), (int)get_c3(m, c));
}

/* vay_push (src/cuda/algorithms/vay_push.cuh:8-30); E and B are already
 * multiplied by q dt / (2 m). */
static inline void vay_push(float *p1, float *p2, float *p3, float *gamma,
                            float E1, float E2, float E3, float B1, float B2,
                            float B3) {
  float g = *gamma;
  float up1 = *p1 + 2.0f * E1 + (*p2 * B3 - *p3 * B2) / g;
  float up2 = *p2 + 2.0f * E2 + (*p3 * B1 - *p1 * B3) / g;
  float up3 = *p3 + 2.0f * E3 + (*p1 * B2 - *p2 * B1) / g;
  float tt = B1 * B1 + B2 * B2 + B3 * B3;
  float ut = up1 * B1 + up2 * B2 + up3 * B3;
  float sigma = 1.0f + up1 * up1 + up2 * up2 + up3 * up3 - tt;
  float inv_gamma2 =
      2.0f / (sigma + sqrtf(sigma * sigma + 4.0f * (tt + ut * ut)));
  float s = 1.0f / (1.0f + inv_gamma2 * tt);
  g = 1.0f / sqrtf(inv_gamma2);
  *p1 = (up1 + B1 * ut * inv_gamma2 + (up2 * B3 - up3 * B2) / g) * s;
  *p2 = (up2 + B2 * ut * inv_gamma2 + (up3 * B1 - up1 * B3) / g) * s;
  *p3 = (up3 + B3 * ut * inv_gamma2 + (up1 * B2 - up2 * B1) / g) * s;
  *gamma = g;
}

/* Interpolator1D / Interpolator2D with spline_t<1> (interpolation.cuh:
 * 146-209): 3 points per dim from c - 1, accumulated in loop order. */
static inline float interp1d(const float *f, float x1, int c1, int st0) {
  float r = 0.0f;
  for (int i = 0; i <= 2; i++) {
    int ii = i + c1 - 1;
    r += f[ii] * interp_cell(x1, c1, ii, st0);
  }
  return r;
}
static inline float interp2d(const float *f, int pitch, float x1, float x2,
                             int c1, int c2, int st0, int st1) {
  float r = 0.0f;
  for (int j = 0; j <= 2; j++) {
    int jj = j + c2 - 1;
    for (int i = 0; i <= 2; i++) {
      int ii = i + c1 - 1;
      r += f[ii + (size_t)jj * pitch] * interp_cell(x1, c1, ii, st0) *
           interp_cell(x2, c2, jj, st1);
    }
  }
  return r;
}

/* Staggers of E1..B3 used by the pusher (ptc_updater.cu:55-60):
 * E1 0b110, E2 0b101, E3 0b011, B1 0b001, B2 0b010, B3 0b100. */
static const int kStag[6] = {6, 5, 3, 1, 2, 4};

static int push_one_nan(const or_ptc *p, size_t idx) {
  float a = p->p1[idx], b = p->p2[idx], c = p->p3[idx];
  return (a != a || b != b || c != c);
}

/* ptc_push_cart_1d, ptc_updater.cu:21-76. */
uint64_t or_push_cart_1d(const or_mesh *m, or_ptc *p, size_t num, float dt,
                         float *const F[6], const float charges[8],
                         const float masses[8]) {
  uint64_t nan_count = 0;
#pragma omp parallel for reduction(+ : nan_count) schedule(static)
  for (size_t idx = 0; idx < num; idx++) {
    uint32_t c = p->cell[idx];
    if (c == OR_MAX_CELL) continue;
    if (!in_bulk(m, c)) {
      p->cell[idx] = OR_MAX_CELL;
      continue;
    }
    uint32_t flag = p->flag[idx];
    int sp = ptc_type(flag);
    float x1 = p->x1[idx];
    float p1 = p->p1[idx], p2 = p->p2[idx], p3 = p->p3[idx];
    float q_over_m = dt * 0.5f * charges[sp] / masses[sp];
    if (push_one_nan(p, idx)) {
      /* The reference prints and traps; the oracle counts and skips. */
      nan_count++;
      continue;
    }
    float gamma = sqrtf(1.0f + p1 * p1 + p2 * p2 + p3 * p3);
    if (!(flag & FLAG_IGNORE_EM)) {
      int c1 = (int)c;
      float fe[6];
      for (int k = 0; k < 6; k++)
        fe[k] = interp1d(F[k], x1, c1, kStag[k] & 1) * q_over_m;
      vay_push(&p1, &p2, &p3, &gamma, fe[0], fe[1], fe[2], fe[3], fe[4],
               fe[5]);
      p->p1[idx] = p1;
      p->p2[idx] = p2;
      p->p3[idx] = p3;
      p->E[idx] = gamma;
    }
  }
  return nan_count;
}

/* ptc_push_cart_2d, ptc_updater.cu:78-141. */
uint64_t or_push_cart_2d(const or_mesh *m, or_ptc *p, size_t num, float dt,
                         float *const F[6], const float charges[8],
                         const float masses[8]) {
  uint64_t nan_count = 0;
  const int pitch = m->dims[0];
#pragma omp parallel for reduction(+ : nan_count) schedule(static)
  for (size_t idx = 0; idx < num; idx++) {
    uint32_t c = p->cell[idx];
    if (c == OR_MAX_CELL) continue;
    if (!in_bulk(m, c)) {
      p->cell[idx] = OR_MAX_CELL;
      continue;
    }
    int c1 = (int)get_c1(m, c);
    int c2 = (int)get_c2(m, c);
    uint32_t flag = p->flag[idx];
    int sp = ptc_type(flag);
    float x1 = p->x1[idx], x2 = p->x2[idx];
    float p1 = p->p1[idx], p2 = p->p2[idx], p3 = p->p3[idx];
    float q_over_m = dt * 0.5f * charges[sp] / masses[sp];
    if (push_one_nan(p, idx)) {
      nan_count++;
      continue;
    }
    float gamma = sqrtf(1.0f + p1 * p1 + p2 * p2 + p3 * p3);
    if (!(flag & FLAG_IGNORE_EM)) {
      float fe[6];
      for (int k = 0; k < 6; k++)
        fe[k] = interp2d(F[k], pitch, x1, x2, c1, c2, kStag[k] & 1,
                         (kStag[k] >> 1) & 1) *
                q_over_m;
      vay_push(&p1, &p2, &p3, &gamma, fe[0], fe[1], fe[2], fe[3], fe[4],
               fe[5]);
      p->p1[idx] = p1;
      p->p2[idx] = p2;
      p->p3[idx] = p3;
      p->E[idx] = gamma;
    }
  }
  return nan_count;
}

/* movement2d / center2d (src/cuda/algorithms/ptc_updater_helper.cuh:26-41),
 * as called from deposit_current_cart_2d. */
static inline float movement2d(float sx0, float sx1, float sy0, float sy1) {
  return (sy1 - sy0) * 0.5f * (sx0 + sx1);
}
static inline float center2d(float sx0, float sx1, float sy0, float sy1) {
  return (2.0f * sx1 * sy1 + sx0 * sy1 + sx1 * sy0 + 2.0f * sx0 * sy0) *
         0.1666667f;
}

/* The deposit is written once as a macro over the accumulator type T so
 * the FP32 and FP64-accumulation variants share every FP32 expression. */

/* deposit_current_cart_1d, ptc_updater.cu:220-293. */
#define DEFINE_DEPOSIT_1D(NAME, T)                                            \
  uint64_t NAME(const or_mesh *m, or_ptc *p, size_t num, float dt,            \
                uint32_t step, int data_interval, T *const J[3],              \
                T *const Rho[8], const float charges[8]) {                    \
    uint64_t far = 0;                                                         \
    int do_rho = ((step + 1) % (uint32_t)data_interval) == 0;                 \
    for (size_t idx = 0; idx < num; idx++) {                                  \
      uint32_t c = p->cell[idx];                                              \
      if (c == OR_MAX_CELL) continue;                                         \
      float v1 = p->p1[idx], v2 = p->p2[idx], v3 = p->p3[idx];                \
      float gamma = p->E[idx];                                                \
      uint32_t flag = p->flag[idx];                                           \
      int sp = ptc_type(flag);                                                \
      float w = p->weight[idx];                                               \
      float old_x1 = p->x1[idx], old_x2 = p->x2[idx], old_x3 = p->x3[idx];    \
      float y = old_x2, z = old_x3;                                           \
      v1 = v1 / gamma;                                                        \
      v2 = v2 / gamma;                                                        \
      v3 = v3 / gamma;                                                        \
      float new_x1 = old_x1 + (v1 * dt) / m->delta[0];                        \
      int dc1 = (int)floorf(new_x1);                                          \
      if (dc1 > 1 || dc1 < -1) far++;                                         \
      new_x1 -= (float)dc1;                                                   \
      p->cell[idx] = c + (uint32_t)dc1;                                       \
      p->x1[idx] = new_x1;                                                    \
      p->x2[idx] = y + v2 * dt;                                               \
      p->x3[idx] = z + v3 * dt;                                               \
      if (flag & FLAG_IGNORE_CURRENT) continue;                               \
      float weight = charges[sp] * w;                                         \
      int i_0 = (dc1 == -1 ? -2 : -1);                                        \
      int i_1 = (dc1 == 1 ? 1 : 0);                                           \
      float djx = 0.0f;                                                       \
      for (int i = i_0; i <= i_1; i++) {                                      \
        float sx0 = cic(-old_x1 + i + 1);                                     \
        float sx1 = cic(-new_x1 + (i + 1 - dc1));                             \
        long off = (long)i + (long)c;                                         \
        djx += sx1 - sx0;                                                     \
        J[0][off + 1] += -weight * djx;                                       \
        float val1 = 0.5f * (sx0 + sx1);                                      \
        J[1][off] += weight * v2 * val1;                                      \
        J[2][off] += weight * v3 * val1;                                      \
        if (do_rho) Rho[sp][off] += weight * sx1;                             \
      }                                                                       \
    }                                                                         \
    return far;                                                               \
  }

/* deposit_current_cart_2d, ptc_updater.cu:295-386. */
#define DEFINE_DEPOSIT_2D(NAME, T)                                            \
  uint64_t NAME(const or_mesh *m, or_ptc *p, size_t num, float dt,            \
                uint32_t step, int data_interval, T *const J[3],              \
                T *const Rho[8], const float charges[8]) {                    \
    uint64_t far = 0;                                                         \
    const long pitch = m->dims[0];                                            \
    int do_rho = ((step + 1) % (uint32_t)data_interval) == 0;                 \
    for (size_t idx = 0; idx < num; idx++) {                                  \
      uint32_t c = p->cell[idx];                                              \
      if (c == OR_MAX_CELL) continue;                                         \
      int c1 = (int)get_c1(m, c);                                             \
      int c2 = (int)get_c2(m, c);                                             \
      float v1 = p->p1[idx], v2 = p->p2[idx], v3 = p->p3[idx];                \
      float gamma = p->E[idx];                                                \
      uint32_t flag = p->flag[idx];                                           \
      int sp = ptc_type(flag);                                                \
      float w = p->weight[idx];                                               \
      float old_x1 = p->x1[idx], old_x2 = p->x2[idx], old_x3 = p->x3[idx];    \
      v1 = v1 / gamma;                                                        \
      v2 = v2 / gamma;                                                        \
      v3 = v3 / gamma;                                                        \
      float new_x1 = old_x1 + (v1 * dt) * m->inv_delta[0];                    \
      float new_x2 = old_x2 + (v2 * dt) * m->inv_delta[1];                    \
      int dc1 = (int)floorf(new_x1);                                          \
      int dc2 = (int)floorf(new_x2);                                          \
      if (dc1 > 1 || dc1 < -1 || dc2 > 1 || dc2 < -1) far++;                  \
      new_x1 -= (float)dc1;                                                   \
      new_x2 -= (float)dc2;                                                   \
      p->cell[idx] = (uint32_t)((c1 + dc1) + (c2 + dc2) * m->dims[0]);        \
      p->x1[idx] = new_x1;                                                    \
      p->x2[idx] = new_x2;                                                    \
      p->x3[idx] = old_x3 + v3 * dt;                                          \
      if (flag & FLAG_IGNORE_CURRENT) continue;                               \
      float weight = -charges[sp] * w;                                        \
      int j_0 = (dc2 == -1 ? -2 : -1);                                        \
      int j_1 = (dc2 == 1 ? 1 : 0);                                           \
      int i_0 = (dc1 == -1 ? -2 : -1);                                        \
      int i_1 = (dc1 == 1 ? 1 : 0);                                           \
      float djy[3] = {0.0f, 0.0f, 0.0f};                                      \
      for (int j = j_0; j <= j_1; j++) {                                      \
        float sy0 = cic(-old_x2 + j + 1);                                     \
        float sy1 = cic(-new_x2 + (j + 1 - dc2));                             \
        long j_off = (long)(j + c2) * pitch;                                  \
        float djx = 0.0f;                                                     \
        for (int i = i_0; i <= i_1; i++) {                                    \
          float sx0 = cic(-old_x1 + i + 1);                                   \
          float sx1 = cic(-new_x1 + (i + 1 - dc1));                           \
          long off = j_off + (i + c1);                                        \
          djx += movement2d(sy0, sy1, sx0, sx1);                              \
          J[0][off + 1] += weight * djx;                                      \
          djy[i - i_0] += movement2d(sx0, sx1, sy0, sy1);                     \
          J[1][off + pitch] += weight * djy[i - i_0];                         \
          float val2 = center2d(sx0, sx1, sy0, sy1);                          \
          J[2][off] += -weight * v3 * val2;                                   \
          if (do_rho) {                                                       \
            float s1 = sx1 * sy1;                                             \
            Rho[sp][off] += -weight * s1;                                     \
          }                                                                   \
        }                                                                     \
      }                                                                       \
    }                                                                         \
    return far;                                                               \
  }

DEFINE_DEPOSIT_1D(or_deposit_cart_1d, float)
DEFINE_DEPOSIT_1D(or_deposit_cart_1d_f64, double)
DEFINE_DEPOSIT_2D(or_deposit_cart_2d, float)
DEFINE_DEPOSIT_2D(or_deposit_cart_2d_f64, double)

/* ------------------------------------------------------------------ */
/* Guard cells on one rank (cuda/sim_environment.cpp:9-127). A strip of */
/* `guard` layers along `dim`, full extent in the other dims, is copied */
/* (or added) from src_lo to dst_lo.                                     */

#define DEFINE_STRIP(NAME, T, OP)                                             \
  static void NAME(const or_mesh *m, T *a, int dim, int src_lo, int dst_lo) { \
    int n0 = m->dims[0], n1 = m->dims[1], n2 = m->dims[2];                    \
    int g = m->guard[dim];                                                    \
    int ext[3] = {n0, n1, n2};                                                \
    ext[dim] = g;                                                             \
    for (int k = 0; k < ext[2]; k++)                                          \
      for (int j = 0; j < ext[1]; j++)                                        \
        for (int i = 0; i < ext[0]; i++) {                                    \
          int s[3] = {i, j, k}, d[3] = {i, j, k};                             \
          s[dim] += src_lo;                                                   \
          d[dim] += dst_lo;                                                   \
          size_t si = (size_t)s[0] + (size_t)n0 * (s[1] + (size_t)n1 * s[2]); \
          size_t di = (size_t)d[0] + (size_t)n0 * (d[1] + (size_t)n1 * d[2]); \
          OP;                                                                 \
        }                                                                     \
  }

DEFINE_STRIP(strip_copy, float, a[di] = a[si])
DEFINE_STRIP(strip_add, float, a[di] += a[si])
DEFINE_STRIP(strip_add_f64, double, a[di] += a[si])

static int mesh_dim(const or_mesh *m) {
  if (m->dims[1] <= 1 && m->dims[2] <= 1) return 1;
  if (m->dims[2] <= 1) return 2;
  return 3;
}

/* send_array_guard_cells_single_dir for dir -1 then +1, dims in order
 * (sim_environment_impl.hpp:286-294, cuda/sim_environment.cpp:9-69).
 * On one periodic rank both neighbours are the rank itself, so the
 * "received" strip is the rank's own sent strip. The send buffer is a
 * snapshot taken before the receive, which matters only for tiny grids. */
void or_send_guard_cells(const or_mesh *m, float *a, const int periodic[3]) {
  int nd = mesh_dim(m);
  for (int dim = 0; dim < nd; dim++) {
    if (!periodic[dim]) continue;
    int g = m->guard[dim], n = m->dims[dim];
    /* dir -1: interior [g, 2g) -> upper guard [n - g, n) */
    strip_copy(m, a, dim, g, n - g);
    /* dir +1: interior [n - 2g, n - g) -> lower guard [0, g) */
    strip_copy(m, a, dim, n - 2 * g, 0);
  }
}

/* send_add_array_guard_cells_single_dir (cuda/sim_environment.cpp:71-127):
 * lower guard [0, g) adds into [n - 2g, n - g), then upper guard
 * [n - g, n) adds into [g, 2g). Guard values are left as they are. */
void or_send_add_guard_cells(const or_mesh *m, float *a,
                             const int periodic[3]) {
  int nd = mesh_dim(m);
  for (int dim = 0; dim < nd; dim++) {
    if (!periodic[dim]) continue;
    int g = m->guard[dim], n = m->dims[dim];
    strip_add(m, a, dim, 0, n - 2 * g);
    strip_add(m, a, dim, n - g, g);
  }
}

void or_send_add_guard_cells_f64(const or_mesh *m, double *a,
                                 const int periodic[3]) {
  int nd = mesh_dim(m);
  for (int dim = 0; dim < nd; dim++) {
    if (!periodic[dim]) continue;
    int g = m->guard[dim], n = m->dims[dim];
    strip_add_f64(m, a, dim, 0, n - 2 * g);
    strip_add_f64(m, a, dim, n - g, g);
  }
}

/* find_zone (quadmesh.h:264-273) and the cell shift of
 * copy_component_to_buffer (kernels.cu:134-142). Returns 1 when the
 * particle is kept (every dim it left is periodic). */
static int wrap_one(const or_mesh *m, uint32_t cell, const int periodic[3],
                    uint32_t *new_cell, int *zone_out) {
  int c[3] = {(int)get_c1(m, cell), (int)get_c2(m, cell),
              (int)get_c3(m, cell)};
  int z[3];
  for (int d = 0; d < 3; d++)
    z[d] = (c[d] >= m->guard[d]) + (c[d] >= (m->dims[d] - m->guard[d]));
  int zone = z[0] + 3 * z[1] + 9 * z[2];
  *zone_out = zone;
  if (zone == 13) {
    *new_cell = cell;
    return 1;
  }
  int nd = mesh_dim(m);
  int dz = (nd > 2 ? z[2] - 1 : 0);
  int dy = (nd > 1 ? z[1] - 1 : 0);
  int dx = z[0] - 1;
  int red0 = m->dims[0] - 2 * m->guard[0];
  int red1 = m->dims[1] - 2 * m->guard[1];
  int red2 = m->dims[2] - 2 * m->guard[2];
  int dcell = -dz * red2 * m->dims[0] * m->dims[1] - dy * red1 * m->dims[0] -
              dx * red0;
  *new_cell = cell + (uint32_t)dcell;
  int keep = 1;
  if (dx != 0 && !periodic[0]) keep = 0;
  if (dy != 0 && !periodic[1]) keep = 0;
  if (dz != 0 && !periodic[2]) keep = 0;
  return keep;
}

uint64_t or_wrap_particles(const or_mesh *m, or_ptc *p, size_t num,
                           const int periodic[3]) {
  uint64_t lost = 0;
  for (size_t n = 0; n < num; n++) {
    uint32_t c = p->cell[n];
    if (c == OR_MAX_CELL) continue;
    uint32_t nc;
    int zone;
    int keep = wrap_one(m, c, periodic, &nc, &zone);
    if (zone == 13) continue;
    if (keep) {
      p->cell[n] = nc;
    } else {
      p->cell[n] = OR_MAX_CELL;
      lost++;
    }
  }
  return lost;
}

static void copy_ptc(or_ptc *p, size_t dst, size_t src) {
  p->x1[dst] = p->x1[src];
  p->x2[dst] = p->x2[src];
  p->x3[dst] = p->x3[src];
  p->p1[dst] = p->p1[src];
  p->p2[dst] = p->p2[src];
  p->p3[dst] = p->p3[src];
  p->E[dst] = p->E[src];
  p->weight[dst] = p->weight[src];
  p->cell[dst] = p->cell[src];
  p->id[dst] = p->id[src];
  p->flag[dst] = p->flag[src];
}

/* send_particles on one rank: wrapped particles are appended after the
 * current number in ascending zone order, and keep their relative order
 * within a zone (the reference's atomic slot order within a zone is not
 * defined; only the set of appended records is). */
size_t or_send_particles(const or_mesh *m, or_ptc *p, size_t num, size_t cap,
                         const int periodic[3]) {
  size_t out = num;
  for (int zone_pass = 0; zone_pass < 27; zone_pass++) {
    if (zone_pass == 13) continue;
    for (size_t n = 0; n < num; n++) {
      uint32_t c = p->cell[n];
      if (c == OR_MAX_CELL) continue;
      uint32_t nc;
      int zone;
      int keep = wrap_one(m, c, periodic, &nc, &zone);
      if (zone != zone_pass) continue;
      if (keep && out < cap) {
        copy_ptc(p, out, n);
        p->cell[out] = nc;
        out++;
      }
      p->cell[n] = OR_MAX_CELL;
    }
  }
  return out;
}

/* ------------------------------------------------------------------ */
/* Yee FDTD, field_solver.cu. Loops run over the bulk cells only.        */

#define AT(a, i, j) ((a)[(size_t)(i) + (size_t)(j) * (size_t)pitch])

/* compute_e_update1d, field_solver.cu:14-43. */
void or_update_e_1d(const or_mesh *m, or_fields *f, float dt) {
  const int pitch = m->dims[0];
  float *e1 = f->E[0], *e2 = f->E[1], *e3 = f->E[2];
  const float *b2 = f->B[1], *b3 = f->B[2];
  const float *b02 = f->Bbg[1], *b03 = f->Bbg[2];
  const float *j1 = f->J[0], *j2 = f->J[1], *j3 = f->J[2];
  (void)pitch;
  for (int n1 = m->guard[0]; n1 < m->dims[0] - m->guard[0]; n1++) {
    e1[n1] -= dt * j1[n1];
    e2[n1] += dt * ((b3[n1] - b3[n1 + 1] - b03[n1] + b03[n1 + 1]) *
                        m->inv_delta[0] -
                    j2[n1]);
    e3[n1] += dt * ((b2[n1 + 1] - b2[n1] - b02[n1 + 1] + b02[n1]) *
                        m->inv_delta[0] -
                    j3[n1]);
  }
}

/* compute_b_update1d, field_solver.cu:133-158. */
void or_update_b_1d(const or_mesh *m, or_fields *f, float dt) {
  const float *e2 = f->E[1], *e3 = f->E[2];
  const float *e02 = f->Ebg[1], *e03 = f->Ebg[2];
  float *b2 = f->B[1], *b3 = f->B[2];
  for (int n1 = m->guard[0]; n1 < m->dims[0] - m->guard[0]; n1++) {
    b2[n1] -= dt * (e3[n1 - 1] - e3[n1] - e03[n1 - 1] + e03[n1]) *
              m->inv_delta[0];
    b3[n1] -= dt * (e2[n1] - e2[n1 - 1] - e02[n1] + e02[n1 - 1]) *
              m->inv_delta[0];
  }
}

/* compute_divs_1d, field_solver.cu:237-259. */
void or_compute_divs_1d(const or_mesh *m, or_fields *f) {
  const float *e1 = f->E[0], *e01 = f->Ebg[0];
  const float *b1 = f->B[0], *b01 = f->Bbg[0];
  for (int n1 = m->guard[0]; n1 < m->dims[0] - m->guard[0]; n1++) {
    f->divE[n1] =
        (e1[n1 + 1] - e01[n1 + 1] - e1[n1] + e01[n1]) * m->inv_delta[0];
    f->divB[n1] =
        (b1[n1] - b01[n1] - b1[n1 - 1] + b01[n1 - 1]) * m->inv_delta[0];
  }
}

/* compute_e_update2d, field_solver.cu:45-84. */
void or_update_e_2d(const or_mesh *m, or_fields *f, float dt) {
  const int pitch = m->dims[0];
  float *e1 = f->E[0], *e2 = f->E[1], *e3 = f->E[2];
  const float *b1 = f->B[0], *b2 = f->B[1], *b3 = f->B[2];
  const float *b01 = f->Bbg[0], *b02 = f->Bbg[1], *b03 = f->Bbg[2];
  const float *j1 = f->J[0], *j2 = f->J[1], *j3 = f->J[2];
  const float id0 = m->inv_delta[0], id1 = m->inv_delta[1];
#pragma omp parallel for schedule(static)
  for (int n2 = m->guard[1]; n2 < m->dims[1] - m->guard[1]; n2++)
    for (int n1 = m->guard[0]; n1 < m->dims[0] - m->guard[0]; n1++) {
      AT(e1, n1, n2) +=
          dt * ((AT(b3, n1, n2 + 1) - AT(b3, n1, n2) - AT(b03, n1, n2 + 1) +
                 AT(b03, n1, n2)) *
                    id1 -
                AT(j1, n1, n2));
      AT(e2, n1, n2) +=
          dt * ((AT(b3, n1, n2) - AT(b3, n1 + 1, n2) - AT(b03, n1, n2) +
                 AT(b03, n1 + 1, n2)) *
                    id0 -
                AT(j2, n1, n2));
      AT(e3, n1, n2) +=
          dt * ((AT(b2, n1 + 1, n2) - AT(b2, n1, n2) - AT(b02, n1 + 1, n2) +
                 AT(b02, n1, n2)) *
                    id0 +
                (AT(b1, n1, n2) - AT(b1, n1, n2 + 1) - AT(b01, n1, n2) +
                 AT(b01, n1, n2 + 1)) *
                    id1 -
                AT(j3, n1, n2));
    }
}

/* compute_b_update2d, field_solver.cu:160-193. */
void or_update_b_2d(const or_mesh *m, or_fields *f, float dt) {
  const int pitch = m->dims[0];
  const float *e1 = f->E[0], *e2 = f->E[1], *e3 = f->E[2];
  const float *e01 = f->Ebg[0], *e02 = f->Ebg[1], *e03 = f->Ebg[2];
  float *b1 = f->B[0], *b2 = f->B[1], *b3 = f->B[2];
  const float id0 = m->inv_delta[0], id1 = m->inv_delta[1];
#pragma omp parallel for schedule(static)
  for (int n2 = m->guard[1]; n2 < m->dims[1] - m->guard[1]; n2++)
    for (int n1 = m->guard[0]; n1 < m->dims[0] - m->guard[0]; n1++) {
      AT(b1, n1, n2) -= dt *
                        (AT(e3, n1, n2) - AT(e3, n1, n2 - 1) -
                         AT(e03, n1, n2) + AT(e03, n1, n2 - 1)) *
                        id1;
      AT(b2, n1, n2) -= dt *
                        (AT(e3, n1 - 1, n2) - AT(e3, n1, n2) -
                         AT(e03, n1 - 1, n2) + AT(e03, n1, n2)) *
                        id0;
      AT(b3, n1, n2) -=
          dt * ((AT(e2, n1, n2) - AT(e2, n1 - 1, n2) - AT(e02, n1, n2) +
                 AT(e02, n1 - 1, n2)) *
                    id0 +
                (AT(e1, n1, n2 - 1) - AT(e1, n1, n2) - AT(e01, n1, n2 - 1) +
                 AT(e01, n1, n2)) *
                    id1);
    }
}

/* compute_divs_2d, field_solver.cu:261-288. */
void or_compute_divs_2d(const or_mesh *m, or_fields *f) {
  const int pitch = m->dims[0];
  const float *e1 = f->E[0], *e2 = f->E[1];
  const float *e01 = f->Ebg[0], *e02 = f->Ebg[1];
  const float *b1 = f->B[0], *b2 = f->B[1];
  const float *b01 = f->Bbg[0], *b02 = f->Bbg[1];
  const float id0 = m->inv_delta[0], id1 = m->inv_delta[1];
#pragma omp parallel for schedule(static)
  for (int n2 = m->guard[1]; n2 < m->dims[1] - m->guard[1]; n2++)
    for (int n1 = m->guard[0]; n1 < m->dims[0] - m->guard[0]; n1++) {
      AT(f->divE, n1, n2) =
          (AT(e1, n1 + 1, n2) - AT(e01, n1 + 1, n2) - AT(e1, n1, n2) +
           AT(e01, n1, n2)) *
              id0 +
          (AT(e2, n1, n2 + 1) - AT(e02, n1, n2 + 1) - AT(e2, n1, n2) +
           AT(e02, n1, n2)) *
              id1;
      AT(f->divB, n1, n2) =
          (AT(b1, n1, n2) - AT(b01, n1, n2) - AT(b1, n1 - 1, n2) +
           AT(b01, n1 - 1, n2)) *
              id0 +
          (AT(b2, n1, n2) - AT(b02, n1, n2) - AT(b2, n1, n2 - 1) +
           AT(b02, n1, n2 - 1)) *
              id1;
    }
}

static void send_guard3(const or_mesh *m, float *const a[3],
                        const int periodic[3]) {
  for (int c = 0; c < 3; c++) or_send_guard_cells(m, a[c], periodic);
}

/* field_solver::update_fields, field_solver.cu:334-358. The host passes a
 * double dt; each kernel receives it converted to float. */
void or_update_fields(const or_mesh *m, or_fields *f, double dt, uint32_t step,
                      const int periodic[3]) {
  int nd = mesh_dim(m);
  if (step == 0) {
    float half = (float)(0.5 * dt);
    if (nd == 1)
      or_update_e_1d(m, f, half);
    else
      or_update_e_2d(m, f, half);
    send_guard3(m, f->E, periodic);
  }
  float dtf = (float)dt;
  if (nd == 1)
    or_update_b_1d(m, f, dtf);
  else
    or_update_b_2d(m, f, dtf);
  send_guard3(m, f->B, periodic);
  if (nd == 1)
    or_update_e_1d(m, f, dtf);
  else
    or_update_e_2d(m, f, dtf);
  send_guard3(m, f->E, periodic);
  if (nd == 1)
    or_compute_divs_1d(m, f);
  else
    or_compute_divs_2d(m, f);
}

/* filter_current_cart_1d, ptc_updater.cu:501-522. */
void or_filter_1d(const or_mesh *m, float *j, float *tmp, const int bnd[4]) {
  int g = m->guard[0], n = m->dims[0];
  for (int n1 = g; n1 < n - g; n1++) {
    int dp = (bnd[1] && n1 == n - g - 1) ? 0 : 1;
    int dm = (bnd[0] && n1 == g) ? 0 : 1;
    float t = 0.5f * j[n1];
    t += 0.25f * j[n1 + dp];
    t += 0.25f * j[n1 - dm];
    tmp[n1] = t;
  }
  for (int n1 = g; n1 < n - g; n1++) j[n1] = tmp[n1];
}

/* filter_current_cart_2d, ptc_updater.cu:524-560. */
void or_filter_2d(const or_mesh *m, float *j, float *tmp, const int bnd[4]) {
  const int pitch = m->dims[0];
  int g0 = m->guard[0], g1 = m->guard[1];
  int n0 = m->dims[0], n1d = m->dims[1];
  for (int b = g1; b < n1d - g1; b++)
    for (int a = g0; a < n0 - g0; a++) {
      int xp = (bnd[1] && a == n0 - g0 - 1) ? 0 : 1;
      int xm = (bnd[0] && a == g0) ? 0 : 1;
      int yp = (bnd[3] && b == n1d - g1 - 1) ? 0 : 1;
      int ym = (bnd[2] && b == g1) ? 0 : 1;
      float t = 0.25f * AT(j, a, b);
      t += 0.125f * AT(j, a + xp, b);
      t += 0.125f * AT(j, a - xm, b);
      t += 0.125f * AT(j, a, b + yp);
      t += 0.125f * AT(j, a, b - ym);
      t += 0.0625f * AT(j, a + xp, b + yp);
      t += 0.0625f * AT(j, a - xm, b + yp);
      t += 0.0625f * AT(j, a + xp, b - ym);
      t += 0.0625f * AT(j, a - xm, b - ym);
      AT(tmp, a, b) = t;
    }
  for (int b = g1; b < n1d - g1; b++)
    for (int a = g0; a < n0 - g0; a++) AT(j, a, b) = AT(tmp, a, b);
}

/* ------------------------------------------------------------------ */
/* ptc_updater::update_particles (ptc_updater.cu:748-841).              */

static void zero_field(const or_mesh *m, float *a) {
  memset(a, 0, sizeof(float) * (size_t)m->dims[0] * m->dims[1] * m->dims[2]);
}

uint64_t or_update_particles(const or_mesh *m, or_ptc *p, size_t num,
                             or_fields *f, double dt, uint32_t step,
                             int data_interval, int num_species,
                             int current_smoothing, const float charges[8],
                             const float masses[8], const int periodic[3],
                             int nthreads) {
  int nd = mesh_dim(m);
  size_t ncell = (size_t)m->dims[0] * m->dims[1] * m->dims[2];
  for (int c = 0; c < 3; c++) zero_field(m, f->J[c]);
  for (int s = 0; s < num_species; s++) zero_field(m, f->Rho[s]);
  float dtf = (float)dt;
  float *F[6] = {f->E[0], f->E[1], f->E[2], f->B[0], f->B[1], f->B[2]};
  uint64_t nan_count = 0, far = 0;
  if (num == 0) goto wrap;
#ifdef _OPENMP
  if (nthreads < 1) nthreads = 1;
  omp_set_num_threads(nthreads);
#else
  nthreads = 1;
#endif
  nan_count = (nd == 1) ? or_push_cart_1d(m, p, num, dtf, F, charges, masses)
                        : or_push_cart_2d(m, p, num, dtf, F, charges, masses);
  if (nthreads == 1) {
    far = (nd == 1) ? or_deposit_cart_1d(m, p, num, dtf, step, data_interval,
                                         f->J, f->Rho, charges)
                    : or_deposit_cart_2d(m, p, num, dtf, step, data_interval,
                                         f->J, f->Rho, charges);
  } else {
    /* Private current / charge buffers per thread, reduced in thread
     * order after a static split of the particle range. */
    int ncomp = 3 + num_species;
    float *priv = (float *)calloc((size_t)nthreads * ncomp * ncell,
                                  sizeof(float));
#pragma omp parallel num_threads(nthreads) reduction(+ : far)
    {
#ifdef _OPENMP
      int t = omp_get_thread_num();
      int nt = omp_get_num_threads();
#else
      int t = 0, nt = 1;
#endif
      size_t lo = num * (size_t)t / nt, hi = num * (size_t)(t + 1) / nt;
      float *base = priv + (size_t)t * ncomp * ncell;
      float *Jt[3] = {base, base + ncell, base + 2 * ncell};
      float *Rt[8] = {0};
      for (int s = 0; s < num_species; s++) Rt[s] = base + (3 + s) * ncell;
      or_ptc sub = *p;
      sub.x1 += lo; sub.x2 += lo; sub.x3 += lo;
      sub.p1 += lo; sub.p2 += lo; sub.p3 += lo;
      sub.E += lo; sub.weight += lo; sub.cell += lo; sub.id += lo;
      sub.flag += lo;
      far += (nd == 1) ? or_deposit_cart_1d(m, &sub, hi - lo, dtf, step,
                                            data_interval, Jt, Rt, charges)
                       : or_deposit_cart_2d(m, &sub, hi - lo, dtf, step,
                                            data_interval, Jt, Rt, charges);
    }
    for (int t = 0; t < nthreads; t++) {
      float *base = priv + (size_t)t * ncomp * ncell;
      for (int c = 0; c < 3; c++)
        for (size_t i = 0; i < ncell; i++) f->J[c][i] += base[c * ncell + i];
      for (int s = 0; s < num_species; s++)
        for (size_t i = 0; i < ncell; i++)
          f->Rho[s][i] += base[(3 + s) * ncell + i];
    }
    free(priv);
  }
  for (int c = 0; c < 3; c++) or_send_add_guard_cells(m, f->J[c], periodic);
  if ((step + 1) % (uint32_t)data_interval == 0)
    for (int s = 0; s < num_species; s++)
      or_send_add_guard_cells(m, f->Rho[s], periodic);
  if (current_smoothing > 0) {
    float *tmp = (float *)calloc(ncell, sizeof(float));
    int bnd[4] = {!periodic[0], !periodic[0], !periodic[1], !periodic[1]};
    for (int it = 0; it < current_smoothing; it++) {
      for (int c = 0; c < 3; c++) {
        if (nd == 1)
          or_filter_1d(m, f->J[c], tmp, bnd);
        else
          or_filter_2d(m, f->J[c], tmp, bnd);
      }
      send_guard3(m, f->J, periodic);
      if ((step + 1) % (uint32_t)data_interval == 0)
        for (int s = 0; s < num_species; s++) {
          if (nd == 1)
            or_filter_1d(m, f->Rho[s], tmp, bnd);
          else
            or_filter_2d(m, f->Rho[s], tmp, bnd);
          or_send_guard_cells(m, f->Rho[s], periodic);
        }
    }
    free(tmp);
  }
wrap:;
  uint64_t lost = or_wrap_particles(m, p, num, periodic);
  (void)far;
  uint64_t hi = nan_count > 0xFFFFFFFFu ? 0xFFFFFFFFu : nan_count;
  uint64_t lo = lost > 0xFFFFFFFFu ? 0xFFFFFFFFu : lost;
  return (hi << 32) | lo;
}

/* ------------------------------------------------------------------ */
/* Sorting.                                                             */

/* Stable counting sort, the two passes of particle_base_impl.hpp:266-295
 * (count into partition[key + 1], prefix sum, then rank = running count). */
void or_stable_counting_sort(const uint32_t *keys, size_t n, uint32_t nkeys,
                             uint32_t *perm) {
  uint64_t *part = (uint64_t *)calloc((size_t)nkeys + 1, sizeof(uint64_t));
  for (size_t i = 0; i < n; i++) part[keys[i] + 1]++;
  for (uint32_t k = 1; k <= nkeys; k++) part[k] += part[k - 1];
  for (size_t i = 0; i < n; i++) perm[part[keys[i]]++] = (uint32_t)i;
  free(part);
}

size_t or_sort_by_cell(const or_mesh *m, or_ptc *p, size_t num) {
  uint32_t ncells =
      (uint32_t)((size_t)m->dims[0] * m->dims[1] * m->dims[2]);
  uint32_t *keys = (uint32_t *)malloc(sizeof(uint32_t) * (num ? num : 1));
  uint32_t *perm = (uint32_t *)malloc(sizeof(uint32_t) * (num ? num : 1));
  size_t live = 0;
  for (size_t i = 0; i < num; i++) {
    keys[i] = (p->cell[i] == OR_MAX_CELL) ? ncells : p->cell[i];
    live += (p->cell[i] != OR_MAX_CELL);
  }
  or_stable_counting_sort(keys, num, ncells + 1, perm);
  /* Gather through a copy (the reference permutes cycles in place with the
   * same result). */
#define GATHER(FIELD, T)                                                  \
  {                                                                       \
    T *tmp = (T *)malloc(sizeof(T) * (num ? num : 1));                    \
    for (size_t r = 0; r < num; r++) tmp[r] = p->FIELD[perm[r]];          \
    memcpy(p->FIELD, tmp, sizeof(T) * num);                               \
    free(tmp);                                                            \
  }
  GATHER(x1, float) GATHER(x2, float) GATHER(x3, float)
  GATHER(p1, float) GATHER(p2, float) GATHER(p3, float)
  GATHER(E, float) GATHER(weight, float) GATHER(cell, uint32_t)
  GATHER(id, uint64_t) GATHER(flag, uint32_t)
#undef GATHER
  free(keys);
  free(perm);
  return live;
}

uint32_t or_tile_key(const or_mesh *m, const int tile[2], uint32_t cell) {
  int r0 = m->dims[0] - 2 * m->guard[0];
  int r1 = m->dims[1] - 2 * m->guard[1];
  uint32_t nt0 = (uint32_t)((r0 + tile[0] - 1) / tile[0]);
  uint32_t nt1 = (uint32_t)((r1 + tile[1] - 1) / tile[1]);
  if (mesh_dim(m) == 1) nt1 = 1;
  uint32_t nt = nt0 * nt1;
  if (cell == OR_MAX_CELL || !in_bulk(m, cell)) return nt;
  int c1 = (int)get_c1(m, cell) - m->guard[0];
  int c2 = (int)get_c2(m, cell) - m->guard[1];
  uint32_t t0 = (uint32_t)(c1 / tile[0]);
  uint32_t t1 = (mesh_dim(m) == 1) ? 0 : (uint32_t)(c2 / tile[1]);
  return t0 + nt0 * t1;
}

size_t or_tile_order(const or_mesh *m, const int tile[2], const uint32_t *cell,
                     const uint32_t *order_in, size_t n, uint32_t *order_out,
                     uint32_t *tile_start) {
  uint32_t nt = or_tile_key(m, tile, OR_MAX_CELL);
  uint32_t *keys = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
  uint32_t *perm = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
  for (size_t r = 0; r < n; r++) keys[r] = or_tile_key(m, tile, cell[order_in[r]]);
  or_stable_counting_sort(keys, n, nt + 1, perm);
  size_t live = 0;
  for (uint32_t t = 0; t <= nt; t++) tile_start[t] = 0;
  for (size_t r = 0; r < n; r++)
    if (keys[r] < nt) {
      live++;
      tile_start[keys[r] + 1]++;
    }
  for (uint32_t t = 1; t <= nt; t++) tile_start[t] += tile_start[t - 1];
  for (size_t r = 0; r < live; r++) order_out[r] = order_in[perm[r]];
  free(keys);
  free(perm);
  return live;
}

/* ------------------------------------------------------------------ */
/* Philox4x32-10 and pair injection (see ap_oracle.h).                 */

static inline uint32_t or_mulhi(uint32_t a, uint32_t b) {
  return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
}

void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int round = 0; round < 10; round++) {
    uint32_t hi0 = or_mulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    uint32_t hi1 = or_mulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

size_t or_inject_pairs(or_ptc *p, size_t num, size_t cap, float dt, uint32_t step,
                       float gamma_thr, float free_path, float pair_energy,
                       uint64_t seed, uint64_t first_id, uint64_t *emitted,
                       uint64_t *dropped) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  const size_t room = cap > num ? (cap - num) / 2 : 0;
  float q = sqrtf(0.25f * pair_energy * pair_energy - 1.0f);
  if (q != q) q = 0.0f;
  size_t k = 0, want = 0;
  for (size_t idx = 0; idx < num; idx++) {
    if (p->cell[idx] == OR_MAX_CELL) continue;
    float gamma = p->E[idx];
    if (!(gamma > gamma_thr)) continue;
    float p1 = p->p1[idx], p2 = p->p2[idx], p3 = p->p3[idx];
    float pm = sqrtf(p1 * p1 + p2 * p2 + p3 * p3);
    float ds = (pm / gamma) * dt;
    double prob = 1.0 - exp(-(double)ds / (double)free_path);
    uint64_t id = p->id[idx];
    const uint32_t ctr[4] = {step, (uint32_t)id, (uint32_t)(id >> 32), 0u};
    uint32_t out[4];
    or_philox4x32_10(ctr, key, out);
    double u = ((double)(out[0] >> 8) + 0.5) * (1.0 / 16777216.0);
    if (!(u < prob)) continue;
    want++;
    if (k >= room) continue;
    float gn = gamma - pair_energy;
    float scale = sqrtf(gn * gn - 1.0f) / pm;
    p->p1[idx] = p1 * scale;
    p->p2[idx] = p2 * scale;
    p->p3[idx] = p3 * scale;
    p->E[idx] = gn;
    float pp = p1 > 0.0f ? q : (p1 < 0.0f ? -q : 0.0f);
    float ep = sqrtf(1.0f + pp * pp);
    for (int m = 0; m < 2; m++) {
      size_t d = num + 2 * k + (size_t)m;
      p->x1[d] = p->x1[idx];
      p->x2[d] = p->x2[idx];
      p->x3[d] = p->x3[idx];
      p->p1[d] = pp;
      p->p2[d] = 0.0f;
      p->p3[d] = 0.0f;
      p->E[d] = ep;
      p->weight[d] = p->weight[idx];
      p->cell[d] = p->cell[idx];
      p->flag[d] = (1u << 7) | ((uint32_t)m << 29);
      p->id[d] = first_id + 2 * (uint64_t)k + (uint64_t)m;
    }
    k++;
  }
  if (emitted) *emitted = k;
  if (dropped) *dropped = want - k;
  return num + 2 * k;
}

/* ------------------------------------------------------------------------
 * 1D gap lab (ptc_updater_1dgap.cu, field_solver_1dgap.cu). */

/* Quadmesh::pos(i, n, pos_in_cell) (quadmesh.h:144-150) in dimension 0. */
static inline float gap_pos(const or_mesh *m, int n, float x) {
  return m->lower[0] + m->delta[0] * ((float)(n - m->guard[0]) + x);
}

/* update_ptc_1dgap (ptc_updater_1dgap.cu:75-161); J1 / Rho adds through
 * the two accumulator types of the f32 and f64 entry points. */
#define GAP_BODY(ACC_T)                                                          \
  uint64_t far = 0;                                                              \
  const int g = m->guard[0], n0 = m->dims[0];                                    \
  for (size_t idx = 0; idx < num; idx++) {                                       \
    uint32_t c = p->cell[idx];                                                   \
    if (c == OR_MAX_CELL) continue;                                                 \
    if ((int)c < g || (int)c >= n0 - g) { /* is_in_bulk */                       \
      p->cell[idx] = OR_MAX_CELL;                                                   \
      continue;                                                                  \
    }                                                                            \
    float p1 = p->p1[idx];                                                       \
    const float x1 = p->x1[idx];                                                 \
    float gamma = p->E[idx];                                                     \
    const uint32_t flag = p->flag[idx];                                          \
    const int sp = ptc_type(flag);                                               \
    float beta = gap_pos(m, (int)c, x1); /* beta_phi(x) = x */                   \
    const float Dr = (x1 < 0.5f ? E3[c] * (0.5f + x1) + E3[c - 1] * (0.5f - x1)  \
                                : E3[c] * (1.5f - x1) + E3[c + 1] * (x1 - 0.5f)); \
    const float E_term = Dr * charges[sp] / masses[sp] * dt;                     \
    p1 += E_term;                                                                \
    const double sgn = beta < 0.0 ? -1.0 : 1.0;                                  \
    const double f = ((double)gamma - sgn * (double)p1) /                        \
                     (1.0 + (double)(beta * beta));                              \
    p1 = (float)((double)p1 + (double)(beta / gamma) * f * f * (double)dt);      \
    p->p1[idx] = p1;                                                             \
    gamma = sqrtf(1.0f + p1 * p1 + beta * beta);                                 \
    float vr = (float)((sgn * (double)p1 / (double)gamma + (double)(beta * beta)) / \
                       (1.0 + (double)(beta * beta)));                           \
    if (beta < 0.0f) vr *= -1.0f;                                                \
    float new_x1 = x1 + vr * dt * m->inv_delta[0];                               \
    const int dc1 = (int)floorf(new_x1);                                         \
    if (dc1 > 1 || dc1 < -1) far++;                                              \
    new_x1 -= (float)dc1;                                                        \
    p->cell[idx] = (uint32_t)((int)c + dc1);                                     \
    p->x1[idx] = new_x1;                                                         \
    beta = gap_pos(m, (int)c + dc1, new_x1);                                     \
    gamma = sqrtf(1.0f + p1 * p1 + beta * beta);                                 \
    p->E[idx] = gamma;                                                           \
    if (!(flag & FLAG_IGNORE_CURRENT)) {                                         \
      const float weight = -charges[sp] * p->weight[idx];                        \
      const int i0 = (dc1 == -1 ? -2 : -1), i1 = (dc1 == 1 ? 1 : 0);             \
      float djx = 0.0f;                                                          \
      for (int i = i0; i <= i1; i++) {                                           \
        const float sx0 = cic(-x1 + i + 1);                                      \
        const float sx1 = cic(-new_x1 + (i + 1 - dc1));                          \
        djx += sx1 - sx0;                                                        \
        J1[i + (int)c + 1] += (ACC_T)(weight * djx * m->delta[0] / dt);          \
        Rho[sp][i + (int)c] += (ACC_T)(-weight * sx1);                           \
      }                                                                          \
    }                                                                            \
  }                                                                              \
  return far;

uint64_t or_update_ptc_1dgap(const or_mesh *m, or_ptc *p, size_t num, float dt,
                             const float *E3, float *J1, float *const Rho[8],
                             const float charges[8], const float masses[8]) {
  GAP_BODY(float)
}

uint64_t or_update_ptc_1dgap_f64(const or_mesh *m, or_ptc *p, size_t num, float dt,
                                 const float *E3, double *J1, double *const Rho[8],
                                 const float charges[8], const float masses[8]) {
  GAP_BODY(double)
}
#undef GAP_BODY

/* filter_current1d (ptc_updater_1dgap.cu:196-213). */
void or_filter_gap(const or_mesh *m, const float *j, float *tmp, const int bnd[2]) {
  const int g = m->guard[0], n = m->dims[0];
  for (int i = 0; i < n; i++) {
    const int dp = (bnd[1] && i == n - g - 1) ? 0 : 1;
    const int dm = (bnd[0] && i == g) ? 0 : 1;
    const float jp = (i + dp < n) ? j[i + dp] : 0.0f;
    const float jm = (i - dm >= 0) ? j[i - dm] : 0.0f;
    float t = 0.5f * j[i];
    t += 0.25f * jp;
    t += 0.25f * jm;
    tmp[i] = t;
  }
}

uint64_t or_update_particles_1dgap(const or_mesh *m, or_ptc *p, size_t num, or_fields *f,
                                   float dt, int smoothing, int num_species,
                                   const float charges[8], const float masses[8],
                                   const int bnd[2]) {
  const size_t n = (size_t)m->dims[0];
  if (num == 0) return 0;
  for (int c = 0; c < 3; c++) zero_field(m, f->J[c]);
  for (int s = 0; s < num_species; s++) zero_field(m, f->Rho[s]);
  /* E3 = E1, smoothed through E2 (ptc_updater_1dgap.cu:232-240) */
  memcpy(f->E[2], f->E[0], n * sizeof(float));
  for (int it = 0; it < smoothing; it++) {
    or_filter_gap(m, f->E[2], f->E[1], bnd);
    memcpy(f->E[2], f->E[1], n * sizeof(float));
  }
  const uint64_t far = or_update_ptc_1dgap(m, p, num, dt, f->E[2], f->J[0], f->Rho, charges,
                                           masses);
  float *tmp = (float *)calloc(n, sizeof(float));
  for (int it = 0; it < smoothing; it++) {
    or_filter_gap(m, f->J[0], tmp, bnd);
    memcpy(f->J[0], tmp, n * sizeof(float));
    for (int s = 0; s < num_species; s++) {
      or_filter_gap(m, f->Rho[s], tmp, bnd);
      memcpy(f->Rho[s], tmp, n * sizeof(float));
    }
  }
  free(tmp);
  return far;
}

/* update_e_1dgap (field_solver_1dgap.cu:14-24) with j0 = B0 * 1.6
 * (field_solver_1dgap.cu:33). */
void or_update_fields_1dgap(const or_mesh *m, float *E1, const float *J1, float B0, float dt) {
  const float j0 = (float)(B0 * 1.6);
  for (int i = m->guard[0] + 1; i < m->dims[0] - m->guard[0] - 1; i++)
    E1[i] += (j0 - J1[i]) * dt;
}

/* ------------------------------------------------------------------------
 * Log-spherical surface injection (ptc_updater_logsph.cu:301-393, 441-490,
 * 849-870), build semantics as documented in ap_oracle.h. */

static inline float ls_pos(const or_mesh *m, int dim, int n, float x) {
  return m->lower[dim] + m->delta[dim] * ((float)(n - m->guard[dim]) + x);
}

void or_ls_surface_density(const or_mesh *m, const or_ptc *p, size_t num, double *se,
                           double *sp_) {
  const int d0 = m->dims[0], d1 = m->dims[1], g0 = m->guard[0], g1 = m->guard[1];
  const int red = d1 - 2 * g1;
  const int ic = g0 + 2;
  for (int r = 0; r < red; r++) se[r] = sp_[r] = 0.0;
  for (size_t idx = 0; idx < num; idx++) {
    const uint32_t c = p->cell[idx];
    if (c == OR_MAX_CELL) continue;
    const int c1 = (int)(c % (uint32_t)d0), c2 = (int)(c / (uint32_t)d0);
    if (!(c1 >= ic - 1 && c1 <= ic - 1 + 3)) continue;
    const int s = ptc_type(p->flag[idx]);
    double *a = s == 0 ? se : (s == 2 ? sp_ : NULL);
    if (!a) continue;
    const float wt = p->weight[idx];
    const int r = c2 - g1;
    const int at[5] = {r - 2 > 0 ? r - 2 : 0, r - 1 > 0 ? r - 1 : 0, r,
                       r + 1 < red - 1 ? r + 1 : red - 1, r + 2 < red - 1 ? r + 2 : red - 1};
    const float k[5] = {1.0f, 4.0f, 6.0f, 4.0f, 1.0f};
    for (int q = 0; q < 5; q++) a[at[q]] += (double)(k[q] * wt / 3.0f / 16.0f);
  }
}

size_t or_ls_inject(const or_mesh *m, or_ptc *p, size_t num, size_t cap, int inj, float p1,
                    float w, float q_e, uint64_t seed, uint32_t call, uint64_t first_id) {
  const int d0 = m->dims[0], d1 = m->dims[1], g0 = m->guard[0], g1 = m->guard[1];
  const int red = d1 - 2 * g1;
  const size_t add = (size_t)2 * inj * red;
  if (num + add > cap) return num;
  const int ic = g0 + 2;
  double *se = (double *)calloc((size_t)red, sizeof(double));
  double *sp_ = (double *)calloc((size_t)red, sizeof(double));
  or_ls_surface_density(m, p, num, se, sp_);
  const float inv_d = 1.0f / m->delta[1];
  const float gamma = (float)sqrt(1.0 + (double)(p1 * p1) + (double)(0.0f * 0.0f));
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int r = 0; r < red; r++) {
    const int i = r + g1;
    const float dens = (float)(se[r] > sp_[r] ? se[r] : sp_[r]);
    const float sin_c = sinf(ls_pos(m, 1, i, 0.5f));
    const int on = i >= g1 + 1 && i < d1 - g1 - 1 && !(q_e * dens > 1.5f * (inv_d * inv_d) * sin_c);
    for (int n = 0; n < inj; n++) {
      const size_t s0 = num + 2 * ((size_t)r * inj + n);
      for (int h = 0; h < 2; h++) {
        const size_t s = s0 + h;
        p->id[s] = first_id + (s - num);
        if (!on) {
          p->cell[s] = OR_MAX_CELL;
          continue;
        }
        const uint32_t ctr[4] = {call, (uint32_t)i, (uint32_t)n, 0u};
        uint32_t out[4];
        or_philox4x32_10(ctr, key, out);
        const float x2 = (float)(((double)(out[0] >> 8) + 0.5) * (1.0 / 16777216.0));
        const float th = ls_pos(m, 1, i, x2);
        const float st = sinf(th), ct = cosf(th);
        const float sg = (float)((0.0f < ct) - (ct < 0.0f));
        p->x1[s] = 0.5f;
        p->x2[s] = x2;
        p->x3[s] = 0.0f;
        p->p1[s] = p1 * 2.0f * fabsf(ct);
        p->p2[s] = p1 * st * sg;
        p->p3[s] = 0.0f;
        p->E[s] = gamma;
        p->cell[s] = (uint32_t)(ic + i * d0);
        p->weight[s] = w * st;
        p->flag[s] = (1u << 6) | ((uint32_t)h << 29); /* primary; e- then e+ */
      }
    }
  }
  free(se);
  free(sp_);
  return num + add;
}

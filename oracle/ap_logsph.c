/*
 * CPU oracle for the log-spherical particle update and field solver (TEST
 * INFRASTRUCTURE ONLY). Compiled twice: without LS_DOUBLE as the *_f32
 * FP32-literal restatement, with LS_DOUBLE as the *_f64 full-FP64 truth.
 * See ap_logsph.h for the list of reference sources restated here.
 *
 * In the FP32 build every expression keeps the reference's operation order
 * and its mixed types: float literals stay float, the reference's double
 * literals (1.0e-5, CONST_PI, 2.0, -1.0, ...) promote the expression to
 * double exactly where the reference's does, and the unqualified float
 * transcendentals the device code calls (expf, sinf, cosf, acosf, logf,
 * atan2f) are the C library's float functions. Grid_LogSph::compute_coef is
 * host code in the reference and is restated with its double
 * intermediates and float storage. The file is compiled with
 * -ffp-contract=off.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "ap_logsph.h"

#define LS_MAX_CELL 0xFFFFFFFFu
#define LS_FLAG_IGNORE_CURRENT (1u << 3)
#define LS_FLAG_IGNORE_EM (1u << 4)
#define LS_CONST_PI 3.14159265358979323846
#define LS_ION 2

#ifdef LS_DOUBLE
typedef double real;
typedef double pos_t;
typedef or_ptc_d PTC;
typedef or_fields_d FLD;
#define SUF(n) n##_f64
#define EXPR exp
#define SINR sin
#define COSR cos
#define ACOSR acos
#define LOGR log
#define ATAN2R atan2
#define SQRTR sqrt
#define FLOORR floor
#define FABSR fabs
#else
typedef float real;
typedef float pos_t;
typedef or_ptc PTC;
typedef or_fields FLD;
#define SUF(n) n##_f32
#define EXPR expf
#define SINR sinf
#define COSR cosf
#define ACOSR acosf
#define LOGR logf
#define ATAN2R atan2f
#define SQRTR sqrtf
#define FLOORR floorf
#define FABSR fabsf
#endif

static inline int ls_type(uint32_t flag) { return (int)(flag >> 29); }

/* Quadmesh::delta / lower (quadmesh.h). The FP64 build derives delta from
 * the box size in double, as a USE_DOUBLE Quadmesh would hold it. */
static inline real ls_delta(const or_mesh *m, int i) {
#ifdef LS_DOUBLE
  return (double)m->sizes[i] / (double)(m->dims[i] - 2 * m->guard[i]);
#else
  return m->delta[i];
#endif
}

/* Quadmesh::pos(i, n, pos_in_cell), quadmesh.h:144-150. The integer
 * stagger overload (quadmesh.h:132-134) passes 0.5 (stagger 0) or 1.0. */
static inline real ls_pos(const or_mesh *m, int i, int n, real x) {
  return (real)m->lower[i] + ls_delta(m, i) * ((real)(n - m->guard[i]) + x);
}

#define AT2(a, i, j) ((a)[(size_t)(i) + (size_t)(j) * (size_t)m->dims[0]])

/* spline_t<1> (interpolation.cuh:28-37). */
static inline real ls_cic(real dx) {
  real a = FABSR(dx);
  real w = (real)1.0f - a;
  return w > (real)0.0f ? w : (real)0.0f;
}

/* Interpolator2D with spline_t<1> (interpolation.cuh:146-171). */
static inline real ls_interp2d(const or_mesh *m, const real *f, pos_t x1,
                               pos_t x2, int c1, int c2, int st0, int st1) {
  real r = 0.0f;
  for (int j = 0; j <= 2; j++) {
    int jj = j + c2 - 1;
    real wy = ls_cic(((real)jj + (st1 == 0 ? (real)0.5f : (real)1.0f)) -
                     ((real)x2 + (real)c2));
    for (int i = 0; i <= 2; i++) {
      int ii = i + c1 - 1;
      real wx = ls_cic(((real)ii + (st0 == 0 ? (real)0.5f : (real)1.0f)) -
                       ((real)x1 + (real)c1));
      r += AT2(f, ii, jj) * wx * wy;
    }
  }
  return r;
}

static const int kLsStag[6] = {6, 5, 3, 1, 2, 4};

/* vay_push.cuh:8-30. */
static inline void ls_vay(real *p1, real *p2, real *p3, real *gamma, real E1,
                          real E2, real E3, real B1, real B2, real B3) {
  real g = *gamma;
  real up1 = *p1 + 2.0f * E1 + (*p2 * B3 - *p3 * B2) / g;
  real up2 = *p2 + 2.0f * E2 + (*p3 * B1 - *p1 * B3) / g;
  real up3 = *p3 + 2.0f * E3 + (*p1 * B2 - *p2 * B1) / g;
  real tt = B1 * B1 + B2 * B2 + B3 * B3;
  real ut = up1 * B1 + up2 * B2 + up3 * B3;
  real sigma = 1.0f + up1 * up1 + up2 * up2 + up3 * up3 - tt;
  real inv_gamma2 =
      2.0f / (sigma + SQRTR(sigma * sigma + 4.0f * (tt + ut * ut)));
  real s = 1.0f / (1.0f + inv_gamma2 * tt);
  g = 1.0f / SQRTR(inv_gamma2);
  *p1 = (up1 + B1 * ut * inv_gamma2 + (up2 * B3 - up3 * B2) / g) * s;
  *p2 = (up2 + B2 * ut * inv_gamma2 + (up3 * B1 - up1 * B3) / g) * s;
  *p3 = (up3 + B3 * ut * inv_gamma2 + (up1 * B2 - up2 * B1) / g) * s;
  *gamma = g;
}

/* alpha_gr and beta_phi (field_solver_logsph.cu:16-26). */
static inline real ls_alpha(real r) {
  (void)r;
  return 1.0f;
}
static inline real ls_beta_phi(const or_ls_params *lp, real r, real theta) {
  return -0.4f * (real)lp->compactness * (real)lp->omega * SINR(theta) /
         (r * r);
}

/* cart2logsph / logsph2cart (ptc_updater_logsph.cu:26-44). */
static inline void ls_cart2logsph(real *v1, real *v2, real *v3, real x1,
                                  real x2, real x3) {
  (void)x1;
  real v1n = *v1, v2n = *v2, v3n = *v3;
  real c2 = COSR(x2), s2 = SINR(x2), c3 = COSR(x3), s3 = SINR(x3);
  *v1 = v1n * s2 * c3 + v2n * s2 * s3 + v3n * c2;
  *v2 = v1n * c2 * c3 + v2n * c2 * s3 - v3n * s2;
  *v3 = -v1n * s3 + v2n * c3;
}
static inline void ls_logsph2cart(real *v1, real *v2, real *v3, real x1,
                                  real x2, real x3) {
  (void)x1;
  real v1n = *v1, v2n = *v2, v3n = *v3;
  real c2 = COSR(x2), s2 = SINR(x2), c3 = COSR(x3), s3 = SINR(x3);
  *v1 = v1n * s2 * c3 + v2n * c2 * c3 - v3n * s3;
  *v2 = v1n * s2 * s3 + v2n * c2 * s3 + v3n * c3;
  *v3 = v1n * c2 - v2n * s2;
}

/* ------------------------------------------------------------------ */
/* Grid_LogSph::compute_coef (grid_log_sph.cpp:11-126) with r_g = 0.     */

#ifdef LS_DOUBLE
static double ls_l1(double r, double rs) {
  double a = sqrt(1.0 - rs / r);
  return r * a + 0.5 * rs * log(2.0 * r * (1.0 + a) - rs);
}
static double ls_A2(double r, double rs) {
  double a = sqrt(1.0 - rs / r);
  return 0.25 * r * a * (2.0 * r + 3.0 * rs) +
         0.375 * rs * rs * log(2.0 * r * (1.0 + a) - rs);
}
static double ls_V3(double r, double rs) {
  double a = sqrt(1.0 - rs / r);
  return r * a * (8.0 * r * r + 10.0 * r * rs + 15.0 * rs * rs) / 24.0 +
         0.3125 * rs * rs * rs * log(2.0 * r * (1.0 + a) - rs);
}
#else
/* grid_log_sph.h:23-38: Scalar (float) arguments and results, double
 * intermediates where the literals make them double. */
static float ls_alpha_h(float r, float rs) { return (float)sqrt(1.0 - (double)(rs / r)); }
static float ls_l1(float r, float rs) {
  float a = ls_alpha_h(r, rs);
  return (float)((double)(r * a) +
                 0.5 * (double)rs * log(2.0 * (double)r * (1.0 + (double)a) - (double)rs));
}
static float ls_A2(float r, float rs) {
  float a = ls_alpha_h(r, rs);
  return (float)(0.25 * (double)r * (double)a * (2.0 * (double)r + 3.0 * (double)rs) +
                 0.375 * (double)rs * (double)rs *
                     log(2.0 * (double)r * (1.0 + (double)a) - (double)rs));
}
static float ls_V3(float r, float rs) {
  float a = ls_alpha_h(r, rs);
  return (float)((double)(r * a) *
                     (8.0 * (double)r * (double)r + 10.0 * (double)r * (double)rs +
                      15.0 * (double)rs * (double)rs) /
                     24.0 +
                 0.3125 * (double)rs * (double)rs * (double)rs *
                     log(2.0 * (double)r * (1.0 + (double)a) - (double)rs));
}
#endif

void SUF(or_ls_coef)(const or_mesh *m, real *const c[OR_NCOEF]) {
  const real r_g = 0.0f;
  const double d0 = (double)ls_delta(m, 0), d1 = (double)ls_delta(m, 1);
  const double d01 = (double)(ls_delta(m, 0) * ls_delta(m, 1));
  for (int j = 0; j < m->dims[1]; j++) {
    double x2 = (double)ls_pos(m, 1, j, 0.5f);
    double x2s = (double)ls_pos(m, 1, j, 1.0f);
    for (int i = 0; i < m->dims[0]; i++) {
      double x1 = (double)ls_pos(m, 0, i, 0.5f);
      double x1s = (double)ls_pos(m, 0, i, 1.0f);
      double r_plus = exp(x1 + d0);
      double r = exp(x1);
      double rs = exp(x1s);
      double rs_minus = exp(x1s - d0);
      size_t o = (size_t)i + (size_t)j * (size_t)m->dims[0];
      c[OR_L1E][o] = ls_l1((real)rs, r_g) - ls_l1((real)rs_minus, r_g);
      c[OR_L2E][o] = (real)(rs * d1);
      c[OR_L3E][o] = (real)(rs * sin(x2s));
      c[OR_L1B][o] = ls_l1((real)r_plus, r_g) - ls_l1((real)r, r_g);
      c[OR_L2B][o] = (real)(r * d1);
      c[OR_L3B][o] = (real)(r * sin(x2));
      c[OR_A1E][o] = (real)(r * r * (cos(x2) - cos(x2 + d1)));
      if (fabs(x2s) < 1.0e-5)
        c[OR_A1E][o] = (real)(r * r * 2.0 * (1.0 - cos(0.5 * d1)));
      else if (fabs(x2s - LS_CONST_PI) < 1.0e-5)
        c[OR_A1E][o] = (real)(r * r * 2.0 * (1.0 - cos(0.5 * d1)));
      real a2e = ls_A2((real)r_plus, r_g) - ls_A2((real)r, r_g);
      c[OR_A2E][o] = (real)((double)a2e * sin(x2));
      c[OR_A3E][o] = (real)((double)a2e * d1);
      c[OR_A1B][o] = (real)(rs * rs * (cos(x2s - d1) - cos(x2s)));
      real a2b = ls_A2((real)rs, r_g) - ls_A2((real)rs_minus, r_g);
      c[OR_A2B][o] = (real)((double)a2b * sin(x2s));
      c[OR_A3B][o] = (real)((double)a2b * d1);
      real v3 = ls_V3((real)r_plus, r_g) - ls_V3((real)r, r_g);
      c[OR_DV][o] = (real)((double)v3 * (cos(x2) - cos(x2 + d1)) / d01);
      if (fabs(x2s) < 1.0e-5 || fabs(x2s - LS_CONST_PI) < 1.0e-5)
        c[OR_DV][o] = (real)((double)v3 * 2.0 * (1.0 - cos(0.5 * d1)) / d01);
    }
  }
}

/* ------------------------------------------------------------------ */
/* user_push_2d_logsph<1> (user_push_2d_logsph.cuh:14-114) with gravity  */
/* (gravity.cuh:12-26) and sync_kill_perp (sync_cooling.cuh:59-86).      */

static inline void ls_sync_kill_perp(const or_ls_params *lp, real *p1,
                                     real *p2, real *p3, real *gamma, real B1,
                                     real B2, real B3, real q_over_m) {
  B1 /= q_over_m;
  B2 /= q_over_m;
  B3 /= q_over_m;
  real p = SQRTR(*p1 * *p1 + *p2 * *p2 + *p3 * *p3);
  real B_sqr = B1 * B1 + B2 * B2 + B3 * B3;
  real pdotB = (*p1 * B1 + *p2 * B2 + *p3 * B3);
  real coef = (real)lp->rad_cooling_coef;
  real delta_p1 = -coef * (*p1 - B1 * pdotB / B_sqr);
  real delta_p2 = -coef * (*p2 - B2 * pdotB / B_sqr);
  real delta_p3 = -coef * (*p3 - B3 * pdotB / B_sqr);
  real f = SQRTR(B_sqr) / (real)lp->B0;
  *p1 += delta_p1 * f;
  *p2 += delta_p2 * f;
  *p3 += delta_p3 * f;
  p = SQRTR(*p1 * *p1 + *p2 * *p2 + *p3 * *p3);
  *gamma = SQRTR(1.0f + p * p);
}

static uint64_t ls_push(const or_mesh *m, const or_ls_params *lp, PTC *p,
                        size_t num, real dt, real *const F[6],
                        const float charges[8], const float masses[8]) {
  uint64_t nan_count = 0;
  for (size_t idx = 0; idx < num; idx++) {
    uint32_t c = p->cell[idx];
    if (c == LS_MAX_CELL) continue;
    int c1 = (int)(c % (uint32_t)m->dims[0]);
    int c2 = (int)((c / (uint32_t)m->dims[0]) % (uint32_t)m->dims[1]);
    if (!(c1 >= m->guard[0] && c1 < m->dims[0] - m->guard[0] &&
          c2 >= m->guard[1] && c2 < m->dims[1] - m->guard[1])) {
      p->cell[idx] = LS_MAX_CELL;
      continue;
    }
    uint32_t flag = p->flag[idx];
    int sp = ls_type(flag);
    pos_t old_x1 = p->x1[idx], old_x2 = p->x2[idx];
    real p1 = p->p1[idx], p2 = p->p2[idx], p3 = p->p3[idx];
    real gamma;
    real r = EXPR(ls_pos(m, 0, c1, old_x1));
    real alpha = ls_alpha(r);
    real q_over_m = dt * 0.5f * (real)charges[sp] / (real)masses[sp];
    if (p1 != p1 || p2 != p2 || p3 != p3) {  /* the reference traps */
      nan_count++;
      continue;
    }
    gamma = SQRTR(1.0f + p1 * p1 + p2 * p2 + p3 * p3);
    if (!(flag & LS_FLAG_IGNORE_EM)) {
      real fe[6];
      for (int k = 0; k < 6; k++)
        fe[k] = alpha *
                ls_interp2d(m, F[k], old_x1, old_x2, c1, c2, kLsStag[k] & 1,
                            (kLsStag[k] >> 1) & 1) *
                q_over_m;
      ls_vay(&p1, &p2, &p3, &gamma, fe[0], fe[1], fe[2], fe[3], fe[4], fe[5]);
      /* gravity(), applied unconditionally with strength dev_params.gravity */
      p1 -= dt * (real)lp->gravity * (real)masses[sp] /
            (r * r * FABSR((real)charges[sp]));
      gamma = SQRTR(1.0f + p1 * p1 + p2 * p2 + p3 * p3);
      if (lp->rad_cooling_on && sp != LS_ION)
        ls_sync_kill_perp(lp, &p1, &p2, &p3, &gamma, fe[3], fe[4], fe[5],
                          q_over_m);
      p->p1[idx] = p1;
      p->p2[idx] = p2;
      p->p3[idx] = p3;
      p->E[idx] = gamma;
    }
  }
  return nan_count;
}

/* movement2d / center2d (ptc_updater_helper.cuh:26-41). */
static inline real ls_movement2d(real sx0, real sx1, real sy0, real sy1) {
  return (sy1 - sy0) * 0.5f * (sx0 + sx1);
}
static inline real ls_center2d(real sx0, real sx1, real sy0, real sy1) {
  return (2.0f * sx1 * sy1 + sx0 * sy1 + sx1 * sy0 + 2.0f * sx0 * sy0) *
         0.1666667f;
}

static inline void ls_acc(void *a, int acc64, size_t o, real v) {
  if (acc64)
    ((double *)a)[o] += (double)v;
  else
    ((real *)a)[o] += v;
}

/* deposit_and_move_2d_log_sph<1> (ptc_updater_logsph.cu:134-282). */
static uint64_t ls_deposit(const or_mesh *m, const or_ls_params *lp, PTC *p,
                           size_t num, real dt, uint32_t step,
                           int data_interval, void *const J[3],
                           void *const Rho[8], int acc64, const real *dV,
                           const float charges[8]) {
  uint64_t far = 0;
  const size_t pitch = (size_t)m->dims[0];
  const real d0 = ls_delta(m, 0), d1 = ls_delta(m, 1);
  const int do_rho = ((step + 1) % (uint32_t)data_interval) == 0;
  for (size_t idx = 0; idx < num; idx++) {
    uint32_t c = p->cell[idx];
    if (c == LS_MAX_CELL) continue;
    int c1 = (int)(c % (uint32_t)m->dims[0]);
    int c2 = (int)((c / (uint32_t)m->dims[0]) % (uint32_t)m->dims[1]);
    real v1 = p->p1[idx], v2 = p->p2[idx], v3 = p->p3[idx];
    real gamma = p->E[idx];
    uint32_t flag = p->flag[idx];
    int sp = ls_type(flag);
    real w = p->weight[idx];
    pos_t old_x1 = p->x1[idx], old_x2 = p->x2[idx], old_x3 = p->x3[idx];

    real r1 = ls_pos(m, 0, c1, old_x1);
    real exp_r1 = EXPR(r1);
    real r2 = ls_pos(m, 1, c2, old_x2);
    v1 = v1 / gamma;
    v2 = v2 / gamma;
    v3 = v3 / gamma;
    real v3_gr = v3 - ls_beta_phi(lp, exp_r1, r2);

    real x = exp_r1 * SINR(r2) * COSR((real)old_x3);
    real y = exp_r1 * SINR(r2) * SINR((real)old_x3);
    real z = exp_r1 * COSR(r2);
    ls_logsph2cart(&v1, &v2, &v3_gr, r1, r2, (real)old_x3);
    x += ls_alpha(exp_r1) * v1 * dt;
    y += ls_alpha(exp_r1) * v2 * dt;
    z += ls_alpha(exp_r1) * v3_gr * dt;
    real r1p = SQRTR(x * x + y * y + z * z);
    real r2p = ACOSR(z / r1p);
    real exp_r1p = r1p;
    r1p = LOGR(r1p);
    real r3p = ATAN2R(y, x);

    ls_cart2logsph(&v1, &v2, &v3_gr, r1p, r2p, r3p);
    real np1 = v1 * gamma;
    real np2 = v2 * gamma;
    real np3 = (v3_gr + ls_beta_phi(lp, exp_r1p, r2p)) * gamma;

    pos_t new_x1 = (pos_t)(old_x1 + (r1p - r1) / d0);
    pos_t new_x2 = (pos_t)(old_x2 + (r2p - r2) / d1);
    int dc1 = (int)FLOORR(new_x1);
    int dc2 = (int)FLOORR(new_x2);
    if (dc1 > 1 || dc1 < -1 || dc2 > 1 || dc2 < -1) far++;
    new_x1 -= (pos_t)dc1;
    new_x2 -= (pos_t)dc2;
    /* reflect around the axis; p *= -1.0 is an exact negation */
    if (ls_pos(m, 1, c2 + dc2, new_x2) < 0.0f) {
      dc2 += 1;
      new_x2 = 1.0f - new_x2;
      np2 = -np2;
      np3 = -np3;
    }
    if ((double)ls_pos(m, 1, c2 + dc2, new_x2) >= LS_CONST_PI) {
      dc2 -= 1;
      new_x2 = 1.0f - new_x2;
      np2 = -np2;
      np3 = -np3;
    }
    p->p1[idx] = np1;
    p->p2[idx] = np2;
    p->p3[idx] = np3;
    p->cell[idx] = (uint32_t)((c1 + dc1) + (c2 + dc2) * m->dims[0]);
    p->x1[idx] = new_x1;
    p->x2[idx] = new_x2;
    p->x3[idx] = (pos_t)r3p;

    if (flag & LS_FLAG_IGNORE_CURRENT) continue;
    real weight = -(real)charges[sp] * w;
    int j_0 = (dc2 == -1 ? -2 : -1);
    int j_1 = (dc2 == 1 ? 1 : 0);
    int i_0 = (dc1 == -1 ? -2 : -1);
    int i_1 = (dc1 == 1 ? 1 : 0);
    real djy[3] = {0.0f, 0.0f, 0.0f};
    for (int j = j_0; j <= j_1; j++) {
      real sy0 = ls_cic(-old_x2 + j + 1);
      real sy1 = ls_cic(-new_x2 + (j + 1 - dc2));
      size_t j_off = (size_t)(j + c2) * pitch;
      real djx = 0.0f;
      for (int i = i_0; i <= i_1; i++) {
        real sx0 = ls_cic(-old_x1 + i + 1);
        real sx1 = ls_cic(-new_x1 + (i + 1 - dc1));
        size_t off = j_off + (size_t)(i + c1);
        real val0 = ls_movement2d(sy0, sy1, sx0, sx1);
        djx += val0;
        ls_acc(J[0], acc64, off + 1, weight * djx);
        real val1 = ls_movement2d(sx0, sx1, sy0, sy1);
        djy[i - i_0] += val1;
        ls_acc(J[1], acc64, off + pitch, weight * djy[i - i_0]);
        real val2 = ls_center2d(sx0, sx1, sy0, sy1);
        ls_acc(J[2], acc64, off, -weight * v3_gr * val2 / dV[off]);
        if (do_rho) {
          real s1 = sx1 * sy1;
          ls_acc(Rho[sp], acc64, off, -weight * s1);
        }
      }
    }
  }
  return far;
}

/* process_j (ptc_updater_logsph.cu:284-299), every cell incl. guards. */
static void ls_process_j(const or_mesh *m, real *const J[3], real *const Rho[8],
                         int num_species, const real *A1e, const real *A2e,
                         const real *dV, real dt) {
  size_t n = (size_t)m->dims[0] * (size_t)m->dims[1];
  real w = ls_delta(m, 0) * ls_delta(m, 1) / dt;
  for (size_t o = 0; o < n; o++) {
    J[0][o] *= w / A1e[o];
    J[1][o] *= w / A2e[o];
    for (int s = 0; s < num_species; s++) Rho[s][o] /= dV[o];
  }
}

/* axis_rho_lower / axis_rho_upper (ptc_updater_logsph.cu:414-438). */
static void ls_axis_rho(const or_mesh *m, real *J3) {
  int j_0 = m->guard[1];
  int j_last = m->dims[1] - m->guard[1];
  for (int i = 0; i < m->dims[0]; i++) {
    AT2(J3, i, j_0 - 1) = 0.0f;
    AT2(J3, i, j_0) = 0.0f;
  }
  for (int i = 0; i < m->dims[0]; i++) {
    AT2(J3, i, j_last) = 0.0f;
    AT2(J3, i, j_last - 1) = 0.0f;
  }
}

/* ptc_outflow (ptc_updater_logsph.cu:440-455). */
static void ls_ptc_outflow(const or_mesh *m, const or_ls_params *lp, PTC *p,
                           size_t num) {
  for (size_t idx = 0; idx < num; idx++) {
    uint32_t c = p->cell[idx];
    if (c == LS_MAX_CELL) continue;
    int c1 = (int)(c % (uint32_t)m->dims[0]);
    uint32_t flag = p->flag[idx];
    if (flag & LS_FLAG_IGNORE_EM) continue;
    if (c1 > m->dims[0] - lp->damping_length + 2) p->flag[idx] = flag | LS_FLAG_IGNORE_EM;
  }
}

/* filter_current_logsph (ptc_updater_logsph.cu:616-666), bulk cells,
 * then the bulk of tmp is copied back into j. */
static void ls_filter(const or_mesh *m, real *j, real *tmp, const real *A,
                      const int bnd[4]) {
  int g0 = m->guard[0], g1 = m->guard[1];
  int n0 = m->dims[0], n1d = m->dims[1];
  for (int b = g1; b < n1d - g1; b++)
    for (int a = g0; a < n0 - g0; a++) {
      int xp = (bnd[1] && a == n0 - g0 - 1) ? 0 : 1;
      int xm = (bnd[0] && a == g0) ? 0 : 1;
      int yp = (bnd[3] && b == n1d - g1 - 1) ? 0 : 1;
      int ym = (bnd[2] && b == g1) ? 0 : 1;
      real t = 0.25f * AT2(j, a, b) * AT2(A, a, b);
      t += 0.125f * AT2(j, a + xp, b) * AT2(A, a + xp, b);
      t += 0.125f * AT2(j, a - xm, b) * AT2(A, a - xm, b);
      t += 0.125f * AT2(j, a, b + yp) * AT2(A, a, b + yp);
      t += 0.125f * AT2(j, a, b - ym) * AT2(A, a, b - ym);
      t += 0.0625f * AT2(j, a + xp, b + yp) * AT2(A, a + xp, b + yp);
      t += 0.0625f * AT2(j, a - xm, b + yp) * AT2(A, a - xm, b + yp);
      t += 0.0625f * AT2(j, a + xp, b - ym) * AT2(A, a + xp, b - ym);
      t += 0.0625f * AT2(j, a - xm, b - ym) * AT2(A, a - xm, b - ym);
      t /= AT2(A, a, b);
      AT2(tmp, a, b) = t;
    }
  for (int b = g1; b < n1d - g1; b++)
    for (int a = g0; a < n0 - g0; a++) AT2(j, a, b) = AT2(tmp, a, b);
}

/* ------------------------------------------------------------------ */
/* field_solver_logsph kernels (field_solver_logsph.cu:29-345).          */

/* compute_b_update_logsph, :117-185. */
static void ls_update_b(const or_mesh *m, const or_ls_params *lp, FLD *f,
                        real *const c[OR_NCOEF], real dt) {
  real *E1 = f->E[0], *E2 = f->E[1], *E3 = f->E[2];
  real *Eb1 = f->Ebg[0], *Eb2 = f->Ebg[1], *Eb3 = f->Ebg[2];
  real *B1 = f->B[0], *B2 = f->B[1], *B3 = f->B[2];
  real *Bb1 = f->Bbg[0], *Bb2 = f->Bbg[1];
  const real d1 = ls_delta(m, 1);
  for (int n2 = m->guard[1]; n2 < m->dims[1] - m->guard[1]; n2++)
    for (int n1 = m->guard[0]; n1 < m->dims[0] - m->guard[0]; n1++) {
      real r1 = EXPR(ls_pos(m, 0, n1, 1.0f));
      real r0 = EXPR(ls_pos(m, 0, n1 - 1, 1.0f));
      real r = EXPR(ls_pos(m, 0, n1, 0.5f));
      AT2(B1, n1, n2) +=
          -dt *
          ((AT2(E3, n1, n2) - AT2(Eb3, n1, n2)) * ls_alpha(r1) * AT2(c[OR_L3E], n1, n2) -
           (AT2(E3, n1, n2 - 1) - AT2(Eb3, n1, n2 - 1)) * ls_alpha(r1) *
               AT2(c[OR_L3E], n1, n2 - 1)) /
          AT2(c[OR_A1B], n1, n2);
      AT2(B2, n1, n2) +=
          -dt *
          ((AT2(E3, n1 - 1, n2) - AT2(Eb3, n1 - 1, n2)) * ls_alpha(r0) *
               AT2(c[OR_L3E], n1 - 1, n2) -
           (AT2(E3, n1, n2) - AT2(Eb3, n1, n2)) * ls_alpha(r1) * AT2(c[OR_L3E], n1, n2)) /
          AT2(c[OR_A2B], n1, n2);
      AT2(B3, n1, n2) +=
          -dt *
          ((((AT2(E2, n1, n2) - AT2(Eb2, n1, n2)) * ls_alpha(r1) +
             AT2(Bb1, n1, n2) * ls_beta_phi(lp, r1, ls_pos(m, 1, n2, 0.5f))) *
                AT2(c[OR_L2E], n1, n2) -
            ((AT2(E2, n1 - 1, n2) - AT2(Eb2, n1 - 1, n2)) * ls_alpha(r0) +
             AT2(Bb1, n1 - 1, n2) * ls_beta_phi(lp, r0, ls_pos(m, 1, n2, 0.5f))) *
                AT2(c[OR_L2E], n1 - 1, n2) +
            ((AT2(E1, n1, n2 - 1) - AT2(Eb1, n1, n2 - 1)) * ls_alpha(r) -
             AT2(Bb2, n1, n2 - 1) * ls_beta_phi(lp, r, ls_pos(m, 1, n2 - 1, 1.0f))) *
                AT2(c[OR_L1E], n1, n2 - 1) -
            ((AT2(E1, n1, n2) - AT2(Eb1, n1, n2)) * ls_alpha(r) -
             AT2(Bb2, n1, n2) * ls_beta_phi(lp, r, ls_pos(m, 1, n2, 1.0f))) *
                AT2(c[OR_L1E], n1, n2)) /
           AT2(c[OR_A3B], n1, n2));
    }
  /* axis at theta = 0 (the thread of the first bulk row) */
  for (int n2 = m->guard[1]; n2 < m->dims[1] - m->guard[1]; n2++) {
    if (!(FABSR(ls_pos(m, 1, n2, 1.0f) - d1) < 1.0e-5)) continue;
    for (int n1 = m->guard[0]; n1 < m->dims[0] - m->guard[0]; n1++)
      AT2(B2, n1, m->guard[1] - 1) = AT2(f->Bbg[1], n1, m->guard[1] - 1);
  }
}

/* compute_e_update_logsph, :29-114. */
static void ls_update_e(const or_mesh *m, const or_ls_params *lp, FLD *f,
                        real *const c[OR_NCOEF], real dt) {
  (void)lp;
  real *E1 = f->E[0], *E2 = f->E[1], *E3 = f->E[2];
  real *B1 = f->B[0], *B2 = f->B[1], *B3 = f->B[2];
  real *Bb1 = f->Bbg[0], *Bb2 = f->Bbg[1], *Bb3 = f->Bbg[2];
  real *J1 = f->J[0], *J2 = f->J[1], *J3 = f->J[2];
  const real d1 = ls_delta(m, 1);
  for (int n2 = m->guard[1]; n2 < m->dims[1] - m->guard[1]; n2++)
    for (int n1 = m->guard[0]; n1 < m->dims[0] - m->guard[0]; n1++) {
      real r = EXPR(ls_pos(m, 0, n1, 1.0f));
      real r1 = EXPR(ls_pos(m, 0, n1 + 1, 0.5f));
      real r0 = EXPR(ls_pos(m, 0, n1, 0.5f));
      if (fabs((double)ls_pos(m, 1, n2, 1.0f) - LS_CONST_PI) < 1.0e-5) {
        AT2(E1, n1, n2) +=
            dt * (-4.0f * (AT2(B3, n1, n2) - AT2(Bb3, n1, n2)) * ls_alpha(r0) / (d1 * r0) -
                  AT2(J1, n1, n2));
      } else {
        AT2(E1, n1, n2) +=
            dt * (((AT2(B3, n1, n2 + 1) - AT2(Bb3, n1, n2 + 1)) * ls_alpha(r0) *
                       AT2(c[OR_L3B], n1, n2 + 1) -
                   (AT2(B3, n1, n2) - AT2(Bb3, n1, n2)) * ls_alpha(r0) * AT2(c[OR_L3B], n1, n2)) /
                      AT2(c[OR_A1E], n1, n2) -
                  AT2(J1, n1, n2));
      }
      AT2(E2, n1, n2) +=
          dt * (((AT2(B3, n1, n2) - AT2(Bb3, n1, n2)) * ls_alpha(r0) * AT2(c[OR_L3B], n1, n2) -
                 (AT2(B3, n1 + 1, n2) - AT2(Bb3, n1 + 1, n2)) * ls_alpha(r1) *
                     AT2(c[OR_L3B], n1 + 1, n2)) /
                    AT2(c[OR_A2E], n1, n2) -
                AT2(J2, n1, n2));
      AT2(E3, n1, n2) +=
          dt * (((AT2(B2, n1 + 1, n2) - AT2(Bb2, n1 + 1, n2)) * ls_alpha(r1) *
                     AT2(c[OR_L2B], n1 + 1, n2) -
                 (AT2(B2, n1, n2) - AT2(Bb2, n1, n2)) * ls_alpha(r0) * AT2(c[OR_L2B], n1, n2) +
                 (AT2(B1, n1, n2) - AT2(Bb1, n1, n2)) * ls_alpha(r) * AT2(c[OR_L1B], n1, n2) -
                 (AT2(B1, n1, n2 + 1) - AT2(Bb1, n1, n2 + 1)) * ls_alpha(r) *
                     AT2(c[OR_L1B], n1, n2 + 1)) /
                    AT2(c[OR_A3E], n1, n2) -
                AT2(J3, n1, n2));
    }
  /* axis at theta = 0 (after the __syncthreads of the reference kernel;
   * these cells are not read by the main update) */
  for (int n2 = m->guard[1]; n2 < m->dims[1] - m->guard[1]; n2++) {
    if (!(FABSR(ls_pos(m, 1, n2, 1.0f) - d1) < 1.0e-5)) continue;
    const int a = m->guard[1] - 1;
    for (int n1 = m->guard[0]; n1 < m->dims[0] - m->guard[0]; n1++) {
      real r0 = EXPR(ls_pos(m, 0, n1, 0.5f));
      AT2(E3, n1, a) = AT2(f->Ebg[2], n1, a);
      AT2(E1, n1, a) +=
          dt * (4.0f * (AT2(B3, n1, a + 1) - AT2(Bb3, n1, a + 1)) * ls_alpha(r0) / (d1 * r0) -
                AT2(J1, n1, a));
    }
  }
}

/* compute_divs_logsph, :188-250. */
static void ls_divs(const or_mesh *m, FLD *f, real *const c[OR_NCOEF]) {
  real *E1 = f->E[0], *E2 = f->E[1];
  real *Eb1 = f->Ebg[0], *Eb2 = f->Ebg[1];
  real *B1 = f->B[0], *B2 = f->B[1];
  real *Bb1 = f->Bbg[0], *Bb2 = f->Bbg[1];
  const real d0 = ls_delta(m, 0), d1 = ls_delta(m, 1);
  for (int n2 = m->guard[1]; n2 < m->dims[1] - m->guard[1]; n2++)
    for (int n1 = m->guard[0]; n1 < m->dims[0] - m->guard[0]; n1++) {
      if (ls_pos(m, 0, n1, 1.0f) > d0) {
        AT2(f->divE, n1, n2) =
            ((AT2(E1, n1 + 1, n2) - AT2(Eb1, n1 + 1, n2)) * AT2(c[OR_A1E], n1 + 1, n2) -
             (AT2(E1, n1, n2) - AT2(Eb1, n1, n2)) * AT2(c[OR_A1E], n1, n2) +
             (AT2(E2, n1, n2 + 1) - AT2(Eb2, n1, n2 + 1)) * AT2(c[OR_A2E], n1, n2 + 1) -
             (AT2(E2, n1, n2) - AT2(Eb2, n1, n2)) * AT2(c[OR_A2E], n1, n2)) /
            (AT2(c[OR_DV], n1, n2) * d0 * d1);
        if (FABSR(ls_pos(m, 1, n2, 1.0f) - (real)m->sizes[1] + (real)m->lower[1]) < 1.0e-5) {
          AT2(f->divE, n1, n2) =
              (real)(((double)((AT2(E1, n1 + 1, n2) - AT2(Eb1, n1 + 1, n2)) *
                                   AT2(c[OR_A1E], n1 + 1, n2) -
                               (AT2(E1, n1, n2) - AT2(Eb1, n1, n2)) * AT2(c[OR_A1E], n1, n2)) -
                      2.0 * (double)(AT2(E2, n1, n2) - AT2(Eb2, n1, n2)) *
                          (double)AT2(c[OR_A2E], n1, n2)) /
                     (double)(AT2(c[OR_DV], n1, n2) * d0 * d1));
        }
      }
      AT2(f->divB, n1, n2) =
          ((AT2(B1, n1, n2) - AT2(Bb1, n1, n2)) * AT2(c[OR_A1B], n1, n2) -
           (AT2(B1, n1 - 1, n2) - AT2(Bb1, n1 - 1, n2)) * AT2(c[OR_A1B], n1 - 1, n2) +
           (AT2(B2, n1, n2) - AT2(Bb2, n1, n2)) * AT2(c[OR_A2B], n1, n2) -
           (AT2(B2, n1, n2 - 1) - AT2(Bb2, n1, n2 - 1)) * AT2(c[OR_A2B], n1, n2 - 1)) /
          (AT2(c[OR_DV], n1, n2) * d0 * d1);
    }
  for (int n2 = m->guard[1]; n2 < m->dims[1] - m->guard[1]; n2++) {
    /* the reference tests abs(pos) - delta here, not abs(pos - delta) */
    if (!(FABSR(ls_pos(m, 1, n2, 1.0f)) - d1 < 1.0e-5)) continue;
    const int a = m->guard[1] - 1;
    for (int n1 = m->guard[0]; n1 < m->dims[0] - m->guard[0]; n1++)
      AT2(f->divE, n1, a) =
          ((AT2(E1, n1 + 1, a) - AT2(Eb1, n1 + 1, a)) * AT2(c[OR_A1E], n1 + 1, a) -
           (AT2(E1, n1, a) - AT2(Eb1, n1, a)) * AT2(c[OR_A1E], n1, a) +
           2.0f * (AT2(E2, n1, a + 1) - AT2(Eb2, n1, a + 1)) * AT2(c[OR_A2E], n1, a + 1)) /
          (AT2(c[OR_DV], n1, a) * d0 * d1);
  }
}

/* stellar_boundary, outflow_boundary_sph, axis_boundary_lower/upper
 * (:252-345) in the order field_solver_logsph::apply_boundary runs them. */
static void ls_field_boundary(const or_mesh *m, const or_ls_params *lp,
                              FLD *f, real omega) {
  real *E1 = f->E[0], *E2 = f->E[1], *E3 = f->E[2];
  real *Eb1 = f->Ebg[0], *Eb2 = f->Ebg[1], *Eb3 = f->Ebg[2];
  real *B1 = f->B[0], *B2 = f->B[1], *B3 = f->B[2];
  real *Bb1 = f->Bbg[0], *Bb2 = f->Bbg[1], *Bb3 = f->Bbg[2];
  for (int j = 0; j < m->dims[1]; j++) {
    real theta_s = ls_pos(m, 1, j, 1.0f);
    real theta = ls_pos(m, 1, j, 0.5f);
    for (int i = 0; i < m->guard[0]; i++) {
      real r_s = EXPR(ls_pos(m, 0, i, 1.0f));
      real r = EXPR(ls_pos(m, 0, i, 0.5f));
      real omega_LT = 0.4f * omega * (real)lp->compactness;
      AT2(B1, i, j) = AT2(Bb1, i, j);
      AT2(B3, i, j) = AT2(Bb3, i, j);
      AT2(E2, i, j) = -(omega - omega_LT) * SINR(theta) * AT2(Bb1, i, j) / ls_alpha(r_s) /
                          r_s / r_s +
                      AT2(Eb2, i, j);
      AT2(E1, i, j) = (omega - omega_LT) * SINR(theta_s) * AT2(Bb2, i, j) / ls_alpha(r_s) /
                          r / r +
                      AT2(Eb1, i, j);
      AT2(B2, i, j) = AT2(Bb2, i, j);
      AT2(B3, i, j) = AT2(Bb3, i, j);
    }
  }
  for (int j = 0; j < m->dims[1]; j++)
    for (int i = 0; i < lp->damping_length; i++) {
      int n1 = m->dims[0] - lp->damping_length + i;
      real q = (real)i / (real)lp->damping_length;
      real lambda = 1.0f - (real)lp->damping_coef * (q * q);
      AT2(E1, n1, j) = lambda * (AT2(E1, n1, j) - AT2(Eb1, n1, j)) + AT2(Eb1, n1, j);
      AT2(E2, n1, j) = lambda * (AT2(E2, n1, j) - AT2(Eb2, n1, j)) + AT2(Eb2, n1, j);
      AT2(E3, n1, j) = lambda * (AT2(E3, n1, j) - AT2(Eb3, n1, j)) + AT2(Eb3, n1, j);
      AT2(B3, n1, j) = lambda * (AT2(B3, n1, j) - AT2(Bb3, n1, j)) + AT2(Bb3, n1, j);
    }
  const int g = m->guard[1];
  for (int i = 0; i < m->dims[0]; i++) {
    AT2(E3, i, g - 1) = AT2(Eb3, i, g - 1);
    AT2(E2, i, g - 1) = -(AT2(E2, i, g) - AT2(Eb2, i, g)) + AT2(Eb2, i, g - 1);
    AT2(B3, i, g - 1) = AT2(Bb3, i, g - 1);
    AT2(B3, i, g) = AT2(Bb3, i, g);
    AT2(B2, i, g - 1) = AT2(Bb2, i, g - 1);
    AT2(B1, i, g - 1) = (AT2(B1, i, g) - AT2(Bb1, i, g)) + AT2(Bb1, i, g - 1);
  }
  const int jl = m->dims[1] - g;
  for (int i = 0; i < m->dims[0]; i++) {
    AT2(E3, i, jl - 1) = AT2(Eb3, i, jl - 1);
    AT2(E2, i, jl) = -(AT2(E2, i, jl - 1) - AT2(Eb2, i, jl - 1)) + AT2(Eb2, i, jl);
    AT2(B3, i, jl) = AT2(Bb3, i, jl);
    AT2(B3, i, jl - 1) = AT2(Bb3, i, jl - 1);
    AT2(B2, i, jl - 1) = AT2(Bb2, i, jl - 1);
    AT2(B1, i, jl) = (AT2(B1, i, jl - 1) - AT2(Bb1, i, jl - 1)) + AT2(Bb1, i, jl);
  }
}

/* ------------------------------------------------------------------ */
/* Exported entry points.                                              */

#ifndef LS_DOUBLE
uint64_t or_ls_push_f32(const or_mesh *m, const or_ls_params *lp, or_ptc *p,
                        size_t num, float dt, float *const F[6],
                        const float charges[8], const float masses[8]) {
  return ls_push(m, lp, p, num, dt, F, charges, masses);
}
uint64_t or_ls_deposit_f32(const or_mesh *m, const or_ls_params *lp,
                           or_ptc *p, size_t num, float dt, uint32_t step,
                           int data_interval, void *const J[3],
                           void *const Rho[8], int acc64, const float *dV,
                           const float charges[8]) {
  return ls_deposit(m, lp, p, num, dt, step, data_interval, J, Rho, acc64, dV,
                    charges);
}
void or_ls_process_j_f32(const or_mesh *m, float *const J[3],
                         float *const Rho[8], int num_species,
                         const float *A1e, const float *A2e, const float *dV,
                         float dt) {
  ls_process_j(m, J, Rho, num_species, A1e, A2e, dV, dt);
}
void or_ls_axis_rho_f32(const or_mesh *m, float *J3) { ls_axis_rho(m, J3); }
void or_ls_ptc_outflow_f32(const or_mesh *m, const or_ls_params *lp,
                           or_ptc *p, size_t num) {
  ls_ptc_outflow(m, lp, p, num);
}
void or_ls_filter_f32(const or_mesh *m, float *j, float *tmp, const float *A,
                      const int bnd[4]) {
  ls_filter(m, j, tmp, A, bnd);
}
void or_ls_update_b_f32(const or_mesh *m, const or_ls_params *lp,
                        or_fields *f, float *const c[OR_NCOEF], float dt) {
  ls_update_b(m, lp, f, c, dt);
}
void or_ls_update_e_f32(const or_mesh *m, const or_ls_params *lp,
                        or_fields *f, float *const c[OR_NCOEF], float dt) {
  ls_update_e(m, lp, f, c, dt);
}
void or_ls_divs_f32(const or_mesh *m, or_fields *f, float *const c[OR_NCOEF]) {
  ls_divs(m, f, c);
}
#endif

void SUF(or_ls_field_boundary)(const or_mesh *m, const or_ls_params *lp,
                               FLD *f, float omega) {
  ls_field_boundary(m, lp, f, (real)omega);
}

void SUF(or_ls_update_fields)(const or_mesh *m, const or_ls_params *lp,
                              FLD *f, real *const c[OR_NCOEF], double dt) {
  const real dtr = (real)dt;
  ls_update_b(m, lp, f, c, dtr);
  ls_update_e(m, lp, f, c, dtr);
  ls_divs(m, f, c);
}

/* Particles out of the bulk after the move: send_particles on one rank
 * with no periodic dim drops them (sim_environment_impl.hpp:319-412). */
static uint64_t ls_drop_outside(const or_mesh *m, PTC *p, size_t num) {
  uint64_t lost = 0;
  for (size_t idx = 0; idx < num; idx++) {
    uint32_t c = p->cell[idx];
    if (c == LS_MAX_CELL) continue;
    int c1 = (int)(c % (uint32_t)m->dims[0]);
    int c2 = (int)((c / (uint32_t)m->dims[0]) % (uint32_t)m->dims[1]);
    if (!(c1 >= m->guard[0] && c1 < m->dims[0] - m->guard[0] &&
          c2 >= m->guard[1] && c2 < m->dims[1] - m->guard[1])) {
      p->cell[idx] = LS_MAX_CELL;
      lost++;
    }
  }
  return lost;
}

/* ptc_updater_logsph::update_particles + apply_boundary
 * (ptc_updater_logsph.cu:681-836). */
uint64_t SUF(or_ls_update_particles)(const or_mesh *m, const or_ls_params *lp,
                                     PTC *p, size_t num, FLD *f,
                                     real *const c[OR_NCOEF], double dt,
                                     uint32_t step, int data_interval,
                                     int num_species, int current_smoothing,
                                     const float charges[8],
                                     const float masses[8], int acc64) {
  const size_t n = (size_t)m->dims[0] * (size_t)m->dims[1];
  const real dtr = (real)dt;
  for (int k = 0; k < 3; k++) memset(f->J[k], 0, sizeof(real) * n);
  for (int s = 0; s < num_species; s++) memset(f->Rho[s], 0, sizeof(real) * n);
  real *const F[6] = {f->E[0], f->E[1], f->E[2], f->B[0], f->B[1], f->B[2]};
  uint64_t nan = ls_push(m, lp, p, num, dtr, F, charges, masses);
  if (acc64) {
    double *acc = (double *)calloc(n * (size_t)(3 + num_species), sizeof(double));
    void *J[3], *R[8] = {0};
    for (int k = 0; k < 3; k++) J[k] = acc + (size_t)k * n;
    for (int s = 0; s < num_species; s++) R[s] = acc + (size_t)(3 + s) * n;
    ls_deposit(m, lp, p, num, dtr, step, data_interval, J, R, 1, c[OR_DV], charges);
    /* one rounding of each exact-ish FP64 sum to the working type */
    for (int k = 0; k < 3; k++)
      for (size_t o = 0; o < n; o++) f->J[k][o] = (real)((double *)J[k])[o];
    for (int s = 0; s < num_species; s++)
      for (size_t o = 0; o < n; o++) f->Rho[s][o] = (real)((double *)R[s])[o];
    free(acc);
  } else {
    void *J[3] = {f->J[0], f->J[1], f->J[2]}, *R[8] = {0};
    for (int s = 0; s < num_species; s++) R[s] = f->Rho[s];
    ls_deposit(m, lp, p, num, dtr, step, data_interval, J, R, 0, c[OR_DV], charges);
  }
  ls_process_j(m, f->J, f->Rho, num_species, c[OR_A1E], c[OR_A2E], c[OR_DV], dtr);
  if (current_smoothing > 0) {
    real *tmp = (real *)calloc(n, sizeof(real));
    const int bnd[4] = {1, 1, 1, 1};
    const int do_rho = ((step + 1) % (uint32_t)data_interval) == 0;
    for (int it = 0; it < current_smoothing; it++) {
      ls_filter(m, f->J[0], tmp, c[OR_A1E], bnd);
      ls_filter(m, f->J[1], tmp, c[OR_A2E], bnd);
      ls_filter(m, f->J[2], tmp, c[OR_A3E], bnd);
      if (do_rho)
        for (int s = 0; s < num_species; s++) ls_filter(m, f->Rho[s], tmp, c[OR_DV], bnd);
    }
    free(tmp);
  }
  uint64_t lost = ls_drop_outside(m, p, num);
  ls_axis_rho(m, f->J[2]);
  ls_ptc_outflow(m, lp, p, num);
  if (nan > 0xFFFFFFFFull) nan = 0xFFFFFFFFull;
  if (lost > 0xFFFFFFFFull) lost = 0xFFFFFFFFull;
  return (nan << 32) | lost;
}

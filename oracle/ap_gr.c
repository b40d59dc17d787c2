/*
 * CPU oracle, 1D GR lab (TEST INFRASTRUCTURE ONLY): restatement of
 *   Grid_1dGR::compute_coef           src/grids/grid_1dgr.cpp:21-187
 *   update_ptc_1dgr                   src/cuda/algorithms/ptc_updater_1dgr.cu:137-300
 *   filter_current1d (K1-weighted)    ptc_updater_1dgr.cu:388-404
 *   ptc_updater_1dgr::update_particles ptc_updater_1dgr.cu:418-473
 *   update_e_1dgr                     src/cuda/algorithms/field_solver_1dgr.cu:14-24
 * The reference mixes float and double (double literals such as 1.0 and
 * 2.0 promote an expression); every expression below keeps the types and
 * the operation order of the cited line. The reference reads its tabulated
 * input (r, Bu1, Bu3, ju1, rho, th, dpsidth) from labs/1dgr/coef.h5; here
 * the caller passes the same seven arrays.
 */
#include "ap_gr.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define FLAG_IGNORE_CURRENT (1u << 3)
#define FLAG_TRACKED (1u << 1) /* ParticleFlag::tracked (enum_types.h:76-87) */

static inline float sqf(float x) { return x * x; }
static inline double sqd(double x) { return x * x; }

/* spline_t<1> (src/cuda/utils/interpolation.cuh:28-37). */
static inline float cic(float dx) {
  float w = 1.0f - fabsf(dx);
  return w > 0.0f ? w : 0.0f;
}

void or_gr_coef(const or_mesh *m, float a, float omega, float B0, const float *v_r,
                const float *v_B1, const float *v_B3, const float *v_jr, const float *v_rho,
                const float *v_theta, const float *v_dpsidth, size_t ntab, float *const co[OR_GR_NCOEF]) {
  const int n_size = m->dims[0];
  for (int k = 0; k < OR_GR_NCOEF; k++) memset(co[k], 0, sizeof(float) * (size_t)n_size);
  size_t n_data = 0, n_mid = 0;
  for (int n = 0; n < n_size; n++) {
    /* grid_1dgr.cpp:89-99 */
    double xi = m->lower[0] + (float)(n - m->guard[0] + 1) * m->delta[0];
    double rp = 1.0 + sqrt(1.0 - a * a);
    double rm = 1.0 - sqrt(1.0 - a * a);
    double exp_xi = exp(xi * (rp - rm));
    double r = (rp - rm * exp_xi) / (1.0 - exp_xi);
    while (n_data + 2 < ntab && v_r[n_data + 1] < r) n_data += 1;
    double x = (r - v_r[n_data]) / (float)(v_r[n_data + 1] - v_r[n_data]);
    float B1 = v_B1[n_data] * (1.0 - x) + v_B1[n_data + 1] * x;
    float B3 = v_B3[n_data] * (1.0 - x) + v_B3[n_data + 1] * x;
    float theta = v_theta[n_data] * (1.0 - x) + v_theta[n_data + 1] * x;
    float b31 = B3 / B1;
    co[OR_GR_B3B1][n] = b31;
    co[OR_GR_RHO0][n] = B0 * (v_rho[n_data] * (1.0 - x) + v_rho[n_data + 1] * x);
    /* :110-139 */
    float Sigma = r * r + (float)(a * a * sqf(cosf(theta)));
    float Delta = r * r - 2.0 * r + a * a;
    float A = sqd(r * r + a * a) - (float)(Delta * a * a * sqf(sinf(theta)));
    float w = 2.0 * a * r / A;
    float g11 = Sigma / Delta;
    float g22 = Sigma;
    float g33 = A * sqf(sinf(theta)) / Sigma;
    float sqrt_gamma = sqrtf(g11 * g22 * g33);
    co[OR_GR_K1][n] =
        (Delta * sqrt_gamma) / (v_dpsidth[n_data] * (1.0 - x) + v_dpsidth[n_data + 1] * x);
    co[OR_GR_D1][n] = (b31 * g33 * (omega - w)) * Delta;
    co[OR_GR_D2][n] = (g11 + b31 * b31 * g33) * Delta * Delta;
    co[OR_GR_D3][n] = g33 * sqf(omega - w);
    co[OR_GR_ALPHA][n] = sqrtf(Delta * Sigma / A);
    co[OR_GR_GAMMA_RR][n] = 1.0 / g11;
    co[OR_GR_GAMMA_FF][n] = 1.0 / g33;
    co[OR_GR_BETA_PHI][n] = -2.0 * a * r / A;
    /* :151-182 (the interpolation weight y uses r, as the reference does) */
    double xi_mid = m->lower[0] + ((n - m->guard[0]) + 0.5) * m->delta[0];
    double exp_xi_mid = exp(xi_mid * (rp - rm));
    double r_mid = (rp - rm * exp_xi_mid) / (1.0 - exp_xi_mid);
    while (n_mid + 2 < ntab && v_r[n_mid + 1] < r_mid) n_mid += 1;
    double y = (r - v_r[n_mid]) / (float)(v_r[n_mid + 1] - v_r[n_mid]);
    co[OR_GR_J0][n] = B0 * (v_jr[n_mid] * (1.0 - y) + v_jr[n_mid + 1] * y) / Delta;
    float theta_mid = v_theta[n_mid] * (1.0 - y) + v_theta[n_mid + 1] * y;
    Sigma = r_mid * r_mid + (float)(a * a * sqf(cosf(theta_mid)));
    Delta = r_mid * r_mid - 2.0 * r_mid + a * a;
    A = sqd(r_mid * r_mid + a * a) - (float)(Delta * a * a * sqf(sinf(theta_mid)));
    g11 = Sigma / Delta;
    g22 = Sigma;
    g33 = A * sqf(sinf(theta_mid)) / Sigma;
    sqrt_gamma = sqrtf(g11 * g22 * g33);
    co[OR_GR_K1_J][n] =
        (Delta * sqrt_gamma) / (v_dpsidth[n_mid] * (1.0 - y) + v_dpsidth[n_mid + 1] * y);
    co[OR_GR_AGRR][n] = Delta * Delta * sqrtf(Delta * Sigma / A) * g11;
  }
}

/* Quadmesh::pos(0, n, x) (quadmesh.h:144-150). */
static inline float mesh_pos0(const or_mesh *m, int n, float x) {
  return m->lower[0] + m->delta[0] * ((float)(n - m->guard[0]) + x);
}

#define DEFINE_GR_PUSH(NAME, ACC)                                                           \
  uint64_t NAME(const or_mesh *m, or_ptc *p, size_t num, float dt, uint32_t step,           \
                int data_interval, float a, float omega, const float *E3,                   \
                const float *const co[OR_GR_NCOEF], ACC *J1, ACC *const Rho[8],             \
                const float charges[8], const float masses[8]) {                            \
    const float *D1c = co[OR_GR_D1], *D2c = co[OR_GR_D2], *D3c = co[OR_GR_D3];              \
    const float *alc = co[OR_GR_ALPHA], *agc = co[OR_GR_AGRR], *thc = co[OR_GR_THETA];      \
    const float *K1 = co[OR_GR_K1], *K1j = co[OR_GR_K1_J], *b31c = co[OR_GR_B3B1];          \
    const int g = m->guard[0], n0 = m->dims[0];                                             \
    const float inv_delta = m->inv_delta[0], delta = m->delta[0];                           \
    uint64_t far = 0;                                                                       \
    for (size_t idx = 0; idx < num; idx++) {                                                \
      uint32_t c = p->cell[idx];                                                            \
      if (c == OR_MAX_CELL) continue;                                                       \
      if ((int)c < g || (int)c >= n0 - g) {                                                 \
        p->cell[idx] = OR_MAX_CELL;                                                         \
        continue;                                                                           \
      }                                                                                     \
      float p1 = p->p1[idx], x1 = p->x1[idx], u0 = p->E[idx];                               \
      float nx1 = 1.0f - x1;                                                                \
      uint32_t flag = p->flag[idx];                                                         \
      int sp = (int)(flag >> 29);                                                           \
      float xi = mesh_pos0(m, (int)c, x1);                                                  \
      const float rp = 1.0f + sqrtf(1.0f - a * a);                                          \
      const float rm = 1.0f - sqrtf(1.0f - a * a);                                          \
      float exp_xi = expf(xi * (rp - rm));                                                  \
      float r = (rp - rm * exp_xi) / (1.0 - exp_xi);                                        \
      float alpha = alc[c] * x1 + alc[c - 1] * nx1;                                         \
      float D1 = D1c[c] * x1 + D1c[c - 1] * nx1;                                            \
      float D2 = D2c[c] * x1 + D2c[c - 1] * nx1;                                            \
      float D3 = D3c[c] * x1 + D3c[c - 1] * nx1;                                            \
      float Dxi = (x1 < 0.5f ? E3[c] * (0.5f + x1) + E3[c - 1] * (0.5f - x1)                \
                             : E3[c] * (1.5f - x1) + E3[c + 1] * (x1 - 0.5f));              \
      float agrr = agc[c] * x1 + agc[c - 1] * nx1;                                          \
      float Er = agrr * Dxi;                                                                \
      float vr = (p1 / u0 - D1) / D2;                                                       \
      float da2dr = (sqf(alc[c]) - sqf(alc[c - 1])) * inv_delta;                            \
      float dD1dr = (D1c[c] - D1c[c - 1]) * inv_delta;                                      \
      float dD2dr = (D2c[c] - D2c[c - 1]) * inv_delta;                                      \
      float dD3dr = (D3c[c] - D3c[c - 1]) * inv_delta;                                      \
      float dDelta_dr = 2.0f * r - 2.0;                                                     \
      float gr_term = -0.5f * u0 *                                                          \
                          (da2dr - (dD3dr + 2.0f * (dD1dr - D1 * dDelta_dr) * vr +           \
                                    (dD2dr - 2.0f * D2 * dDelta_dr) * vr * vr)) *           \
                          dt +                                                              \
                      dDelta_dr * p1 * vr * dt;                                             \
      p1 += gr_term;                                                                        \
      float E_term = Er * charges[sp] / masses[sp] * dt;                                    \
      p1 += E_term;                                                                         \
      u0 = sqrtf((D2 + p1 * p1) / (D2 * (alpha * alpha - D3) + D1 * D1));                   \
      p->p1[idx] = p1;                                                                      \
      vr = (p1 / u0 - D1) / D2;                                                             \
      if (step % (uint32_t)data_interval == 0 && (flag & FLAG_TRACKED)) {                   \
        float theta = thc[c] * x1 + thc[c - 1] * nx1;                                       \
        float Sigma = (r * r + a * a * sqf(cosf(theta)));                                   \
        float Delta = (r * r - 2.0f * r + a * a);                                           \
        float g_00 = -(1.0f - 2.0f * r / Sigma);                                            \
        float g_03 = -4.0 * r * a * sqf(sinf(theta)) / Sigma;                               \
        float B31 = b31c[c] * x1 + b31c[c - 1] * nx1;                                       \
        float u0inf = (g_00 + g_03 * omega) * u0 + g_03 * B31 * Delta * u0 * vr;            \
        p->p2[idx] = u0inf;                                                                 \
      }                                                                                     \
      float new_x1 = x1 + vr * dt * inv_delta;                                              \
      int dc1 = (int)floorf(new_x1);                                                        \
      if (dc1 > 1 || dc1 < -1) {                                                            \
        /* the reference prints and reads past the coefficients; emptied */               \
        far++;                                                                              \
        p->cell[idx] = OR_MAX_CELL;                                                         \
        continue;                                                                           \
      }                                                                                     \
      new_x1 -= (float)dc1;                                                                 \
      p->cell[idx] = c + dc1;                                                               \
      p->x1[idx] = new_x1;                                                                  \
      nx1 = 1.0f - new_x1;                                                                  \
      uint32_t cn = c + dc1;                                                                \
      alpha = alc[cn] * new_x1 + alc[cn - 1] * nx1;                                         \
      D1 = D1c[cn] * new_x1 + D1c[cn - 1] * nx1;                                            \
      D2 = D2c[cn] * new_x1 + D2c[cn - 1] * nx1;                                            \
      D3 = D3c[cn] * new_x1 + D3c[cn - 1] * nx1;                                            \
      u0 = sqrtf((D2 + p1 * p1) / (D2 * (alpha * alpha - D3) + D1 * D1));                   \
      p->E[idx] = u0;                                                                       \
      if (!(flag & FLAG_IGNORE_CURRENT)) {                                                  \
        float weight = -charges[sp] * p->weight[idx];                                       \
        int i_0 = (dc1 == -1 ? -2 : -1);                                                    \
        int i_1 = (dc1 == 1 ? 1 : 0);                                                       \
        float djx = 0.0f;                                                                   \
        for (int i = i_0; i <= i_1; i++) {                                                  \
          float sx0 = cic(-x1 + i + 1);                                                     \
          float sx1 = cic(-new_x1 + (i + 1 - dc1));                                         \
          djx += sx1 - sx0;                                                                 \
          J1[i + (int)c + 1] += weight * djx / K1j[i + (int)c + 1] * delta / dt;            \
          Rho[sp][i + (int)c] += -weight * sx1 / K1[i + (int)c];                            \
        }                                                                                   \
      }                                                                                     \
    }                                                                                       \
    return far;                                                                             \
  }

DEFINE_GR_PUSH(or_update_ptc_1dgr, float)
DEFINE_GR_PUSH(or_update_ptc_1dgr_f64, double)

/* filter_current1d of the GR lab (ptc_updater_1dgr.cu:388-404): every cell
 * [0, dims0) of j weighted by k1, from j into tmp. The reference reads one
 * element past each end of the arrays at i = 0 and i = dims0 - 1; that
 * element counts as 0 here. */
void or_filter_gr(const or_mesh *m, const float *j, float *tmp, const float *k1,
                  const int bnd[2]) {
  const int n0 = m->dims[0], g = m->guard[0];
  for (int i = 0; i < n0; i++) {
    int dxp = (bnd[1] && i == n0 - g - 1) ? 0 : 1;
    int dxm = (bnd[0] && i == g) ? 0 : 1;
    const int ip = i + dxp, im = i - dxm;
    const float jp = ip < n0 ? j[ip] : 0.0f, kp = ip < n0 ? k1[ip] : 0.0f;
    const float jm = im >= 0 ? j[im] : 0.0f, km = im >= 0 ? k1[im] : 0.0f;
    float t = 0.5f * j[i] * k1[i];
    t += 0.25f * jp * kp;
    t += 0.25f * jm * km;
    t /= k1[i];
    tmp[i] = t;
  }
}

uint64_t or_update_particles_1dgr(const or_mesh *m, or_ptc *p, size_t num, or_fields *f,
                                  float dt, uint32_t step, int data_interval, int smoothing,
                                  int num_species, float a, float omega,
                                  const float *const co[OR_GR_NCOEF], const float charges[8],
                                  const float masses[8], const int bnd[2]) {
  const size_t n0 = (size_t)m->dims[0];
  uint64_t far = 0;
  if (num == 0) return 0;
  for (int c = 0; c < 3; c++) memset(f->J[c], 0, sizeof(float) * n0);
  for (int s = 0; s < num_species; s++) memset(f->Rho[s], 0, sizeof(float) * n0);
  memcpy(f->E[2], f->E[0], sizeof(float) * n0);
  for (int it = 0; it < smoothing; it++) {
    or_filter_gr(m, f->E[2], f->E[1], co[OR_GR_K1_J], bnd);
    memcpy(f->E[2], f->E[1], sizeof(float) * n0);
  }
  far = or_update_ptc_1dgr(m, p, num, dt, step, data_interval, a, omega, f->E[2], co, f->J[0],
                           f->Rho, charges, masses);
  float *tmp = (float *)calloc(n0, sizeof(float));
  for (int it = 0; it < smoothing; it++) {
    or_filter_gr(m, f->J[0], tmp, co[OR_GR_K1_J], bnd);
    memcpy(f->J[0], tmp, sizeof(float) * n0);
    for (int s = 0; s < num_species; s++) {
      or_filter_gr(m, f->Rho[s], tmp, co[OR_GR_K1], bnd);
      memcpy(f->Rho[s], tmp, sizeof(float) * n0);
    }
  }
  free(tmp);
  return far;
}

void or_update_e_1dgr(const or_mesh *m, float *E1, const float *J1, const float *j0, float dt) {
  for (int i = m->guard[0] + 1; i < m->dims[0] - m->guard[0] - 5; i++)
    E1[i] += (j0[i] - J1[i]) * dt;
}

/*
 * CPU oracle, photons and pair production (TEST INFRASTRUCTURE ONLY).
 *
 * Restates, in FP32 with the reference's operation order (compiled with
 * -ffp-contract=off), the photon movers of the particle updaters and the
 * radiative_transfer module with its three user-function sets:
 *   - the framework's default: src/cuda/radiation/user_radiative_functions.cu
 *   - the pulsar lab's:        labs/pulsar/src/cuda/radiation/
 *                              user_radiative_functions.cu
 *   - the 1D GR lab's:         labs/1dgr/src/cuda/radiation/
 *                              user_radiative_functions.cuh (with the
 *                              inverse-Compton tables of ap_ic.c), and the
 *                              1D GR photon mover
 *   - the 1D gap lab's:        labs/1dgap/src/cuda/radiation/
 *                              user_radiative_functions.cuh (the same
 *                              tables), and the 1D gap photon mover
 * The float transcendentals are the C library's expf, sinf, cosf, acosf,
 * logf, atan2f (the reference's device code calls the float overloads);
 * rho_c's pow and chi's square root take double arguments there and here.
 *
 * Build semantics that replace the reference's (the same in the library):
 *   - random numbers: the reference draws from per-thread cuRAND XORWOW
 *     states in thread order; here each particle (photon) draws four
 *     uniforms in (0, 1] from Philox4x32-10 keyed on the run's seed with
 *     counter (pass, id, tag), so the result does not depend on scheduling.
 *     The draws are used as: default model u0 = photon energy, u1 = free
 *     path, u2 = tracking; pulsar model u0 = emission test, u2 = tracking;
 *     1D GR and gap models u0 = emission test, u1 = photon energy,
 *     u2 = tracking; pair production u0 = tracking (1D GR and gap: u1 =
 *     conversion test);
 *   - order: emitters are ranked in slot order (the reference ranks them by
 *     block and shared-memory atomic order);
 *   - ids: every new photon and particle gets an id from the counter
 *     (the reference numbers tracked ones only), so the random stream of a
 *     secondary is its own;
 *   - capacity: emissions past the photon capacity are dropped with the
 *     parent unchanged (the reference writes past it); a pair whose second
 *     slot would be past the particle capacity is dropped with its photon
 *     (the reference checks the first slot only).
 */
#include "ap_rad.h"

#include <math.h>
#include <string.h>

#define RAD_PI 3.14159265358979323846 /* CONST_PI, src/core/constant_defs.h:11 */
#define FLAG_TRACKED (1u << 1)        /* ParticleFlag / PhotonFlag::tracked   */
#define FLAG_SECONDARY (1u << 7)      /* ParticleFlag::secondary              */

#define AT2(a, i, j) ((a)[(size_t)(i) + (size_t)(j) * (size_t)m->dims[0]])

void or_rad_uniforms(uint64_t seed, uint32_t tag, uint32_t call, uint64_t id, float u[4]) {
  const uint32_t ctr[4] = {call, (uint32_t)id, (uint32_t)(id >> 32), tag};
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t out[4];
  or_philox4x32_10(ctr, key, out);
  /* k * 2^-24 for k in [1, 2^24]: the range of curand_uniform, exact */
  for (int i = 0; i < 4; ++i) u[i] = (float)((out[i] >> 8) + 1u) * (1.0f / 16777216.0f);
}

/* Quadmesh (quadmesh.h): get_c1 / get_c2, pos, is_in_bulk. */
static inline int c1_of(const or_mesh *m, uint32_t c) { return (int)(c % (uint32_t)m->dims[0]); }
static inline int c2_of(const or_mesh *m, uint32_t c) {
  return (int)((c / (uint32_t)m->dims[0]) % (uint32_t)m->dims[1]);
}
/* pos(i, n, pos_in_cell): a dimension past the grid's gives x * delta. */
static inline float mpos(const or_mesh *m, int i, int n, float x) {
  if (i < m->dimension) return m->lower[i] + m->delta[i] * ((float)(n - m->guard[i]) + x);
  return x * m->delta[i];
}
static inline int in_bulk(const or_mesh *m, uint32_t c) {
  const int c1 = c1_of(m, c), c2 = c2_of(m, c);
  const uint32_t c3 = c / ((uint32_t)m->dims[0] * (uint32_t)m->dims[1]);
  return c1 >= m->guard[0] && c1 < m->dims[0] - m->guard[0] && c2 >= m->guard[1] &&
         c2 < m->dims[1] - m->guard[1] && c3 < (uint32_t)m->dims[2];
}

/* spline_t<1> and Interpolator2D (interpolation.cuh:28-37, 146-171);
 * st0 / st1 are the stagger bits of x and y. */
static inline float cic(float dx) {
  const float w = 1.0f - fabsf(dx);
  return w > 0.0f ? w : 0.0f;
}
static float interp2d(const or_mesh *m, const float *f, float x1, float x2, int c1, int c2,
                      int st0, int st1) {
  float r = 0.0f;
  for (int j = 0; j <= 2; j++) {
    const int jj = j + c2 - 1;
    const float wy = cic(((float)jj + (st1 == 0 ? 0.5f : 1.0f)) - (x2 + (float)c2));
    for (int i = 0; i <= 2; i++) {
      const int ii = i + c1 - 1;
      const float wx = cic(((float)ii + (st0 == 0 ? 0.5f : 1.0f)) - (x1 + (float)c1));
      r += AT2(f, ii, jj) * wx * wy;
    }
  }
  return r;
}
/* |B| at a position: B1 Stagger(0b001), B2 0b010, B3 0b100. */
static float b_mag(const or_mesh *m, const or_fields *f, float x1, float x2, int c1, int c2) {
  const float B1 = interp2d(m, f->B[0], x1, x2, c1, c2, 1, 0);
  const float B2 = interp2d(m, f->B[1], x1, x2, c1, c2, 0, 1);
  const float B3 = interp2d(m, f->B[2], x1, x2, c1, c2, 0, 0);
  return sqrtf(B1 * B1 + B2 * B2 + B3 * B3);
}
static void b_vec(const or_mesh *m, const or_fields *f, float x1, float x2, int c1, int c2,
                  float B[3]) {
  B[0] = interp2d(m, f->B[0], x1, x2, c1, c2, 1, 0);
  B[1] = interp2d(m, f->B[1], x1, x2, c1, c2, 0, 1);
  B[2] = interp2d(m, f->B[2], x1, x2, c1, c2, 0, 0);
}

/* cart2logsph / logsph2cart (ptc_updater_logsph.cu:26-44). */
static inline void cart2logsph(float *v1, float *v2, float *v3, float x2, float x3) {
  const float v1n = *v1, v2n = *v2, v3n = *v3;
  const float c2 = cosf(x2), s2 = sinf(x2), c3 = cosf(x3), s3 = sinf(x3);
  *v1 = v1n * s2 * c3 + v2n * s2 * s3 + v3n * c2;
  *v2 = v1n * c2 * c3 + v2n * c2 * s3 - v3n * s2;
  *v3 = -v1n * s3 + v2n * c3;
}
static inline void logsph2cart(float *v1, float *v2, float *v3, float x2, float x3) {
  const float v1n = *v1, v2n = *v2, v3n = *v3;
  const float c2 = cosf(x2), s2 = sinf(x2), c3 = cosf(x3), s3 = sinf(x3);
  *v1 = v1n * s2 * c3 + v2n * c2 * c3 - v3n * s3;
  *v2 = v1n * s2 * s3 + v2n * c2 * s3 + v3n * c3;
  *v3 = v1n * c2 - v2n * s2;
}

/* Zone wrap of one coordinate (find_zone + the cell shift of
 * copy_component_to_buffer, kernels.cu:134-142); 0 when the photon leaves
 * through a non-periodic side. */
static int wrap(int *c, int g, int n, int periodic) {
  const int red = n - 2 * g;
  if (*c < g) {
    if (!periodic) return 0;
    *c += red;
  } else if (*c >= n - g) {
    if (!periodic) return 0;
    *c -= red;
  }
  return 1;
}

void or_move_photons_cart(const or_mesh *m, or_photons *ph, size_t num, float dt,
                          const int periodic[3]) {
  for (size_t idx = 0; idx < num; ++idx) {
    const uint32_t c = ph->cell[idx];
    if (c == OR_MAX_CELL) continue;
    if (m->dimension == 1) {
      /* move_photons_cart_1d (ptc_updater.cu:627-656) */
      const float p1 = ph->p1[idx], p2 = ph->p2[idx], p3 = ph->p3[idx];
      const float E = sqrtf(p1 * p1 + p2 * p2 + p3 * p3);
      const float old_x1 = ph->x1[idx], old_x2 = ph->x2[idx], old_x3 = ph->x3[idx];
      float new_x1 = old_x1 + p1 / E * dt * m->inv_delta[0];
      const int dc1 = (int)floorf(new_x1);
      int cn = (int)c + dc1;
      new_x1 -= (float)dc1;
      ph->x1[idx] = new_x1;
      ph->x2[idx] = old_x2 + p2 * dt / E;
      ph->x3[idx] = old_x3 + p3 * dt / E;
      ph->path_left[idx] -= dt;
      ph->cell[idx] = wrap(&cn, m->guard[0], m->dims[0], periodic[0]) ? (uint32_t)cn
                                                                       : OR_MAX_CELL;
    } else {
      /* move_photons_cart_2d (ptc_updater.cu:658-690) */
      const int c1 = c1_of(m, c), c2 = c2_of(m, c);
      float v1 = ph->p1[idx], v2 = ph->p2[idx], v3 = ph->p3[idx];
      const float E = sqrtf(v1 * v1 + v2 * v2 + v3 * v3);
      v1 /= E;
      v2 /= E;
      v3 /= E;
      const float old_x1 = ph->x1[idx], old_x2 = ph->x2[idx], old_x3 = ph->x3[idx];
      float new_x1 = old_x1 + v1 * dt * m->inv_delta[0];
      float new_x2 = old_x2 + v2 * dt * m->inv_delta[1];
      const int dc1 = (int)floorf(new_x1);
      const int dc2 = (int)floorf(new_x2);
      int n1 = c1 + dc1, n2 = c2 + dc2;
      new_x1 -= (float)dc1;
      new_x2 -= (float)dc2;
      ph->x1[idx] = new_x1;
      ph->x2[idx] = new_x2;
      ph->x3[idx] = old_x3 + v3 * dt;
      ph->path_left[idx] -= dt;
      const int keep = wrap(&n1, m->guard[0], m->dims[0], periodic[0]) &&
                       wrap(&n2, m->guard[1], m->dims[1], periodic[1]);
      ph->cell[idx] = keep ? (uint32_t)(n1 + n2 * m->dims[0]) : OR_MAX_CELL;
    }
  }
}

void or_move_photons_logsph(const or_mesh *m, const or_rad_params *rp, or_photons *ph,
                            size_t num, float dt) {
  for (size_t idx = 0; idx < num; ++idx) {
    const uint32_t c = ph->cell[idx];
    if (c == OR_MAX_CELL) continue;
    const int c1 = c1_of(m, c), c2 = c2_of(m, c);
    float v1 = ph->p1[idx], v2 = ph->p2[idx], v3 = ph->p3[idx];
    const float E = sqrtf(v1 * v1 + v2 * v2 + v3 * v3);
    v1 = v1 / E;
    v2 = v2 / E;
    v3 = v3 / E;
    const float old_x1 = ph->x1[idx], old_x2 = ph->x2[idx], old_x3 = ph->x3[idx];
    const float r1 = mpos(m, 0, c1, old_x1);
    const float exp_r1 = expf(r1);
    /* censor photons outside the conversion radius (:83-87) */
    if (exp_r1 > rp->r_cutoff || (double)exp_r1 < 1.02) {
      ph->cell[idx] = OR_MAX_CELL;
      continue;
    }
    const float r2 = mpos(m, 1, c2, old_x2);
    float x = exp_r1 * sinf(r2) * cosf(old_x3);
    float y = exp_r1 * sinf(r2) * sinf(old_x3);
    float z = exp_r1 * cosf(r2);
    logsph2cart(&v1, &v2, &v3, r2, old_x3);
    x += v1 * dt;
    y += v2 * dt;
    z += v3 * dt;
    float r1p = sqrtf(x * x + y * y + z * z);
    const float r2p = acosf(z / r1p);
    r1p = logf(r1p);
    const float r3p = atan2f(y, x);
    cart2logsph(&v1, &v2, &v3, r2p, r3p);
    ph->p1[idx] = v1 * E;
    ph->p2[idx] = v2 * E;
    ph->p3[idx] = v3 * E;
    float new_x1 = old_x1 + (r1p - r1) / m->delta[0];
    float new_x2 = old_x2 + (r2p - r2) / m->delta[1];
    int dc1 = (int)floorf(new_x1);
    int dc2 = (int)floorf(new_x2);
    /* the cell is taken before the axis reflection below (:114) */
    const int n1 = c1 + dc1, n2 = c2 + dc2;
    new_x1 -= (float)dc1;
    new_x2 -= (float)dc2;
    if (mpos(m, 1, c2 + dc2, new_x2) < 0.0f) {
      dc2 += 1;
      new_x2 = 1.0f - new_x2;
    } else if ((double)mpos(m, 1, c2 + dc2, new_x2) >= RAD_PI) {
      dc2 -= 1;
      new_x2 = 1.0f - new_x2;
    }
    ph->x1[idx] = new_x1;
    ph->x2[idx] = new_x2;
    ph->x3[idx] = r3p;
    ph->path_left[idx] -= dt;
    /* send_particles + clear_guard_cells: nothing comes back through the
     * non-periodic sides of one rank */
    const int keep = n1 >= m->guard[0] && n1 < m->dims[0] - m->guard[0] && n2 >= m->guard[1] &&
                     n2 < m->dims[1] - m->guard[1];
    ph->cell[idx] = keep ? (uint32_t)(n1 + n2 * m->dims[0]) : OR_MAX_CELL;
  }
}

/* rho_c of the pulsar lab (user_radiative_functions.cu:18-24): the pow
 * takes a double exponent, so it and the division are done in double. */
static float rho_c(float r, float theta) {
  const float c = cosf(theta);
  const float c2 = c * c;
  const float s = sinf(theta);
  if ((double)fabsf(s) < 1.0e-5) return 1.0e10f;
  return (float)((double)r * pow((double)(1.0f + 3.0f * c2), 1.5) /
                 (double)(3.0f * s * (1.0f + c2)));
}

/* ---- the 1D GR lab's functions (labs/1dgr/src/cuda/radiation/
 * user_radiative_functions.cuh:19-189). A metric array at x1 in cell c is
 * interpolated between c - 1 and c. The photon energy draw is u1; the
 * emission and conversion tests draw u0 and u1. */
static inline float gr_at(const float *a, uint32_t c, float x1) {
  return a[c] * x1 + a[c - 1] * (1.0f - x1);
}
static inline float sgnf(float v) { return (float)((0.0f < v) - (v < 0.0f)); }

/* The Boyer-Lindquist r of the tortoise coordinate xi and Delta
 * (:38-45); r takes the reference's double division. */
static inline float gr_r(float xi, float a) {
  const float rp = 1.0f + sqrtf(1.0f - a * a);
  const float rm = 1.0f - sqrtf(1.0f - a * a);
  const float exp_xi = expf(xi * (rp - rm));
  return (float)((rp - rm * exp_xi) / (1.0 - exp_xi));
}

static int check_emit_gr(const or_rad_params *rp, const or_ptc *p, size_t tid, const float u[4]) {
  const or_rad_gr *g = rp->gr;
  const float alpha = gr_at(g->alpha, p->cell[tid], p->x1[tid]);
  const float gamma = alpha * p->E[tid];
  return u[0] < or_ic_rate(g->ic, gamma) * alpha * rp->delta_t;
}

static void emit_photon_gr(const or_mesh *m, const or_rad_params *rp, or_ptc *p, size_t tid,
                           or_photons *ph, size_t off, const float u[4]) {
  const or_rad_gr *g = rp->gr;
  const float x1 = p->x1[tid], p1 = p->p1[tid], u0_ptc = p->E[tid];
  const uint32_t c = p->cell[tid];
  const float xi = mpos(m, 0, c1_of(m, c), x1);
  const float a = g->a;
  const float r = gr_r(xi, a);
  const float Delta = (float)(r * r - 2.0 * r + a * a);
  const float alpha = gr_at(g->alpha, c, x1), D1 = gr_at(g->D1, c, x1);
  const float D2 = gr_at(g->D2, c, x1), D3 = gr_at(g->D3, c, x1);
  const float B3B1 = gr_at(g->B3B1, c, x1), g11 = gr_at(g->gamma_rr, c, x1);
  const float g33 = gr_at(g->gamma_ff, c, x1), beta = gr_at(g->beta_phi, c, x1);
  const float ur_ptc = u0_ptc * Delta * (p1 / u0_ptc - D1) / D2;
  const float gamma = alpha * p->E[tid];
  const float Eph = or_ic_photon_e(g->ic, gamma, u[1]);
  p->E[tid] = (gamma - Eph) / alpha;
  const float En = p->E[tid];
  float np1 = sgnf(p1) * sqrtf(En * En * (D2 * (alpha * alpha - D3) + D1 * D1) - D2);
  if (np1 != np1) np1 = 0.0f;
  p->p1[tid] = np1;
  if (fabsf(Eph) < 50.0f) return; /* energy taken, no photon kept */
  ph->x1[off] = x1;
  ph->x2[off] = ph->x3[off] = 0.0f;
  ph->p1[off] = Delta * (Eph / gamma) * ur_ptc / g11;
  ph->p2[off] = 0.0f;
  ph->p3[off] = (Eph / gamma) * (u0_ptc * (g->omega + beta) + B3B1 * ur_ptc) / g33;
  ph->E[off] = Eph / alpha;
  ph->weight[off] = p->weight[tid];
  ph->path_left[off] = 0.0f;
  ph->cell[off] = c;
}

static int check_pair_gr(const or_rad_params *rp, const or_photons *ph, size_t tid,
                         const float u[4]) {
  const or_rad_gr *g = rp->gr;
  const float alpha = gr_at(g->alpha, ph->cell[tid], ph->x1[tid]);
  const float u0_hat = alpha * fabsf(ph->E[tid]);
  const float prob = or_gg_rate(g->ic, u0_hat) * alpha * rp->delta_t;
  return u[1] < prob;
}

static void produce_pair_gr(const or_rad_params *rp, or_photons *ph, size_t tid, or_ptc *p,
                            size_t off) {
  const or_rad_gr *g = rp->gr;
  const float u0 = 0.5f * fabsf(ph->E[tid]);
  const uint32_t c = ph->cell[tid];
  const float x1 = ph->x1[tid];
  ph->cell[tid] = OR_MAX_CELL;
  const float alpha = gr_at(g->alpha, c, x1), D1 = gr_at(g->D1, c, x1);
  const float D2 = gr_at(g->D2, c, x1), D3 = gr_at(g->D3, c, x1);
  float p1 = sgnf(ph->p1[tid]) * sqrtf(u0 * u0 * (D2 * (alpha * alpha - D3) + D1 * D1) - D2);
  if (p1 != p1) p1 = 0.0f;
  for (int k = 0; k < 2; ++k) {
    const size_t o = off + (size_t)k;
    p->x1[o] = x1;
    p->x2[o] = p->x3[o] = 0.0f;
    p->p1[o] = p1;
    p->p2[o] = p->p3[o] = 0.0f;
    p->E[o] = u0;
    p->weight[o] = ph->weight[tid];
    p->cell[o] = c;
    p->flag[o] = FLAG_SECONDARY | ((uint32_t)k << 29);
  }
}

void or_move_photons_gr(const or_mesh *m, const or_rad_gr *g, or_photons *ph, size_t num,
                        float dt, uint32_t step, int data_interval) {
  const float inv = m->inv_delta[0];
  for (size_t idx = 0; idx < num; ++idx) {
    const uint32_t c = ph->cell[idx];
    if (c == OR_MAX_CELL) continue;
    if (!in_bulk(m, c)) {
      ph->cell[idx] = OR_MAX_CELL;
      continue;
    }
    float p1 = ph->p1[idx];
    const float p3 = ph->p3[idx], x1 = ph->x1[idx];
    float u0 = fabsf(ph->E[idx]);
    const float nx1 = 1.0f - x1;
    const float xi = mpos(m, 0, (int)c, x1);
    const float a = 0.99f; /* the reference fixes the spin here (:322) */
    const float r = gr_r(xi, a);
    const float alpha = g->alpha[c] * x1 + g->alpha[c - 1] * nx1;
    const float gamma11 = g->gamma_rr[c] * x1 + g->gamma_rr[c - 1] * nx1;
    const float gamma33 = g->gamma_ff[c] * x1 + g->gamma_ff[c - 1] * nx1;
    const float dDelta_dr = 2.0f * r - 2.0f;
    const float dl = r * r - 2.0f * r + a * a;
    const float Delta_sqr = dl * dl;
    u0 = sqrtf(gamma11 * p1 * p1 / Delta_sqr + gamma33 * p3 * p3) / alpha;
    const float da2dr = (g->alpha[c] * g->alpha[c] - g->alpha[c - 1] * g->alpha[c - 1]) * inv;
    const float dgamma11dxi = (g->gamma_rr[c] - g->gamma_rr[c - 1]) * inv;
    const float dgamma33dxi = (g->gamma_ff[c] - g->gamma_ff[c - 1]) * inv;
    const float dbetadxi = (g->beta_phi[c] - g->beta_phi[c - 1]) * inv;
    const float gr_term =
        (-0.5f * u0 * da2dr - (p1 * p1 * dgamma11dxi / Delta_sqr + p3 * p3 * dgamma33dxi) *
                                  0.5f / u0 +
         p3 * dbetadxi + gamma11 * p1 * p1 * dDelta_dr / (Delta_sqr * u0)) *
        dt;
    p1 += gr_term;
    u0 = sqrtf(gamma11 * p1 * p1 / Delta_sqr + gamma33 * p3 * p3) / alpha;
    ph->p1[idx] = p1;
    ph->E[idx] = u0;
    const float vr = gamma11 * p1 / (Delta_sqr * u0);
    if (step % (uint32_t)data_interval == 0 && (ph->flag[idx] & FLAG_TRACKED)) {
      const float theta = g->theta[c] * x1 + g->theta[c - 1] * nx1;
      const float ct = cosf(theta);
      const float Sigma = (r * r + a * a * (ct * ct));
      const float Delta = (r * r - 2.0f * r + a * a);
      const float g_00 = -(1.0f + 2.0f * r * (r * r + a * a) / Sigma / Delta);
      const float g_03 = -2.0f * r * a / Sigma / Delta;
      ph->p2[idx] = (u0 - g_03 * ph->p3[idx]) / g_00;
    }
    float new_x1 = x1 + vr * dt * inv;
    const int dc1 = (int)floorf(new_x1);
    new_x1 -= (float)dc1;
    ph->cell[idx] = c + (uint32_t)dc1;
    ph->x1[idx] = new_x1;
  }
}

/* ---- the 1D gap lab's functions (labs/1dgap/src/cuda/radiation/
 * user_radiative_functions.cuh:17-131): the 1D GR lab's tables on a flat
 * line. Draws as for the 1D GR model. */
static int check_emit_gap(const or_rad_params *rp, const or_ptc *p, size_t tid,
                          const float u[4]) {
  return u[0] < or_ic_rate(rp->gr->ic, p->E[tid]) * rp->delta_t;
}

static void emit_photon_gap(const or_rad_params *rp, or_ptc *p, size_t tid, or_photons *ph,
                            size_t off, const float u[4]) {
  const float x1 = p->x1[tid], p1 = p->p1[tid];
  const uint32_t c = p->cell[tid];
  const float gamma = p->E[tid];
  float Eph = or_ic_photon_e(rp->gr->ic, gamma, u[1]);
  if (Eph >= gamma - 1.01f) Eph = gamma - 1.01f;
  const float En = gamma - Eph;
  p->E[tid] = En;
  float np1 = En * p1 / gamma;
  if (np1 != np1) np1 = 0.0f;
  p->p1[tid] = np1;
  if (fabsf(Eph) < 0.001f / rp->e_min) return; /* energy taken, no photon kept */
  ph->x1[off] = x1;
  ph->x2[off] = ph->x3[off] = 0.0f;
  ph->p1[off] = sgnf(p1) * Eph;
  ph->p2[off] = ph->p3[off] = 0.0f;
  ph->E[off] = Eph;
  ph->weight[off] = p->weight[tid];
  ph->path_left[off] = 0.0f;
  ph->cell[off] = c;
}

static int check_pair_gap(const or_rad_params *rp, const or_photons *ph, size_t tid,
                          const float u[4]) {
  return u[1] < or_gg_rate(rp->gr->ic, ph->E[tid]) * rp->delta_t;
}

static void produce_pair_gap(const or_mesh *m, or_photons *ph, size_t tid, or_ptc *p,
                             size_t off) {
  const float Eph = fabsf(ph->p1[tid]);
  const uint32_t c = ph->cell[tid];
  const float x1 = ph->x1[tid];
  ph->cell[tid] = OR_MAX_CELL;
  float p1 = sgnf(ph->p1[tid]) * sqrtf(0.25f * Eph * Eph - 1.0f);
  if (p1 != p1) p1 = 0.0f;
  const float beta = mpos(m, 0, c1_of(m, c), x1);
  const float E = sqrtf(1.0f + p1 * p1 + beta * beta);
  for (int k = 0; k < 2; ++k) {
    const size_t o = off + (size_t)k;
    p->x1[o] = x1;
    p->x2[o] = p->x3[o] = 0.0f;
    p->p1[o] = p1;
    p->p2[o] = p->p3[o] = 0.0f;
    p->E[o] = E;
    p->weight[o] = ph->weight[tid];
    p->cell[o] = c;
    p->flag[o] = FLAG_SECONDARY | ((uint32_t)k << 29);
  }
}

void or_move_photons_gap(const or_mesh *m, or_photons *ph, size_t num, float dt) {
  for (size_t idx = 0; idx < num; ++idx) {
    const uint32_t c = ph->cell[idx];
    if (c == OR_MAX_CELL) continue;
    if (!in_bulk(m, c)) {
      ph->cell[idx] = OR_MAX_CELL;
      continue;
    }
    const float p1 = ph->p1[idx], x1 = ph->x1[idx];
    float new_x1 = x1 + sgnf(p1) * dt * m->inv_delta[0];
    const int dc1 = (int)floorf(new_x1);
    new_x1 -= (float)dc1;
    ph->cell[idx] = c + (uint32_t)dc1;
    ph->x1[idx] = new_x1;
  }
}

/* check_emit_photon of the model (default :13-17; pulsar :26-53). */
static int check_emit(const or_mesh *m, const or_rad_params *rp, const or_ptc *p, size_t tid,
                      const float u[4]) {
  const float gamma = p->E[tid];
  if (rp->model == OR_RAD_DEFAULT) return gamma > rp->gamma_thr;
  if (rp->model == OR_RAD_GR1D) return check_emit_gr(rp, p, tid, u);
  if (rp->model == OR_RAD_GAP1D) return check_emit_gap(rp, p, tid, u);
  const uint32_t c = p->cell[tid];
  const int c1 = c1_of(m, c), c2 = c2_of(m, c);
  const float r = expf(mpos(m, 0, c1, p->x1[tid]));
  if (r > 0.6f / rp->omega) return 0;
  if ((double)r < 1.05) return 0;
  const float theta = mpos(m, 1, c2, p->x2[tid]);
  const float rc = rho_c(r, theta);
  if (rc < 1.0f) return 0;
  const float rate = rp->delta_t * gamma / (rp->l_curv * rc);
  const float Eph = rp->e_curv * gamma * gamma * gamma / rc;
  return u[0] < rate && Eph > 2.1f;
}

/* emit_photon of the model (default :19-63; pulsar :55-131): updates the
 * parent and writes the photon at slot off, or leaves the slot a hole. */
static void emit_photon(const or_mesh *m, const or_rad_params *rp, or_ptc *p, size_t tid,
                        or_photons *ph, size_t off, const or_fields *f, const float u[4]) {
  if (rp->model == OR_RAD_GR1D) {
    emit_photon_gr(m, rp, p, tid, ph, off, u);
    return;
  }
  if (rp->model == OR_RAD_GAP1D) {
    emit_photon_gap(rp, p, tid, ph, off, u);
    return;
  }
  const uint32_t c = p->cell[tid];
  const int c1 = c1_of(m, c), c2 = c2_of(m, c);
  const float p1 = p->p1[tid], p2 = p->p2[tid], p3 = p->p3[tid];
  const float gamma = p->E[tid];
  if (rp->model == OR_RAD_DEFAULT) {
    const float pi = sqrtf(gamma * gamma - 1.0f);
    const float Eph = 2.5f + u[0] * (rp->E_secondary - 1.0f) * 2.0f;
    const float gr = gamma - Eph;
    const float pf = sqrtf(gr * gr - 1.0f);
    p->p1[tid] = p1 * pf / pi;
    p->p2[tid] = p2 * pf / pi;
    p->p3[tid] = p3 * pf / pi;
    p->E[tid] = gamma - Eph;
    const float theta = mpos(m, 1, c2, p->x2[tid]);
    const float l = (1.0f / sinf(theta) - 1.0f) * rp->photon_path;
    const float lph = l < 10.0f ? l : 10.0f; /* min(10.0f, l) */
    if (theta < 0.005f || (double)theta > RAD_PI - 0.005f) return;
    const float path = lph * (0.5f + 0.5f * u[1]);
    if (path > rp->r_cutoff) return;
    ph->x1[off] = p->x1[tid];
    ph->x2[off] = p->x2[tid];
    ph->x3[off] = p->x3[tid];
    ph->p1[off] = Eph * p1 / pi;
    ph->p2[off] = Eph * p2 / pi;
    ph->p3[off] = Eph * p3 / pi;
    ph->E[off] = 0.0f; /* not set by the reference's default model */
    ph->weight[off] = p->weight[tid];
    ph->path_left[off] = path;
    ph->cell[off] = c;
    return;
  }
  const float x1 = p->x1[tid], x2 = p->x2[tid];
  const float pi = sqrtf(p1 * p1 + p2 * p2 + p3 * p3);
  const float r = expf(mpos(m, 0, c1, x1));
  const float theta = mpos(m, 1, c2, x2);
  const float a = gamma - 1.0f;
  const float b = rp->e_curv * gamma * gamma * gamma / rho_c(r, theta);
  const float Eph = b < a ? b : a; /* std::min(a, b) */
  if (Eph < 2.1f) return;
  const float gr = gamma - Eph;
  const float pf = sqrtf(gr * gr - 1.0f);
  p->p1[tid] = p1 * pf / pi;
  p->p2[tid] = p2 * pf / pi;
  p->p3[tid] = p3 * pf / pi;
  p->E[tid] = gamma - Eph;
  const float B = b_mag(m, f, x1, x2, c1, c2);
  if (Eph * B / rp->BQ < 2.1f && p1 > 0.0f) return;
  ph->x1[off] = p->x1[tid];
  ph->x2[off] = p->x2[tid];
  ph->x3[off] = p->x3[tid];
  ph->p1[off] = Eph * p1 / pi;
  ph->p2[off] = Eph * p2 / pi;
  ph->p3[off] = Eph * p3 / pi;
  ph->E[off] = Eph;
  ph->weight[off] = p->weight[tid];
  ph->path_left[off] = 0.0f;
  ph->cell[off] = c;
}

/* check_produce_pair of the model (default :65-68; pulsar :134-171); the
 * pulsar checks may remove the photon. */
static int check_pair(const or_mesh *m, const or_rad_params *rp, or_photons *ph, size_t tid,
                      const or_fields *f) {
  if (rp->model == OR_RAD_DEFAULT) return ph->path_left[tid] <= 0.0f;
  const uint32_t cell = ph->cell[tid];
  const int c1 = c1_of(m, cell), c2 = c2_of(m, cell);
  const float x1 = ph->x1[tid], x2 = ph->x2[tid];
  const float p1 = ph->p1[tid], p2 = ph->p2[tid], p3 = ph->p3[tid];
  const float Eph = ph->E[tid];
  const float theta = mpos(m, 1, c2, x2);
  if (theta < m->delta[1] || (double)theta > RAD_PI - (double)m->delta[1]) {
    ph->cell[tid] = OR_MAX_CELL;
    return 0;
  }
  const float r0 = AT2(f->Rho[0], c1, c2), r1 = AT2(f->Rho[1], c1, c2);
  const float s = fabsf(r0 + r1);
  const float rho = s < 0.0001f ? 0.0001f : s; /* max(s, 0.0001f) */
  const float N = fabsf(r0) + fabsf(r1);
  const float multiplicity = N / rho;
  if (multiplicity > 50.0f) {
    ph->cell[tid] = OR_MAX_CELL;
    return 0;
  }
  float B[3];
  b_vec(m, f, x1, x2, c1, c2, B);
  const float Bm = sqrtf(B[0] * B[0] + B[1] * B[1] + B[2] * B[2]);
  const float cth = (B[0] * p1 + B[1] * p2 + B[2] * p3) / (Bm * Eph);
  const float chi =
      (float)((double)(Eph * Bm) * sqrt(1.0 - (double)(cth * cth)) / (double)rp->BQ);
  return (double)chi > 0.12;
}

/* produce_pair (default :70-121; the pulsar lab's is the same). */
static void produce_pair(or_photons *ph, size_t tid, or_ptc *p, size_t off) {
  const float p1 = ph->p1[tid], p2 = ph->p2[tid], p3 = ph->p3[tid];
  float E_ph2 = p1 * p1 + p2 * p2 + p3 * p3;
  if (E_ph2 <= 4.01f) E_ph2 = 4.01f;
  const float ratio = sqrtf(0.25f - 1.0f / E_ph2);
  const float gamma = sqrtf(1.0f + ratio * ratio * E_ph2);
  if (gamma != gamma) {
    ph->cell[tid] = OR_MAX_CELL;
    return;
  }
  for (int k = 0; k < 2; ++k) {
    const size_t o = off + (size_t)k;
    p->x1[o] = ph->x1[tid];
    p->x2[o] = ph->x2[tid];
    p->x3[o] = ph->x3[tid];
    p->p1[o] = ratio * p1;
    p->p2[o] = ratio * p2;
    p->p3[o] = ratio * p3;
    p->E[o] = gamma;
    p->weight[o] = ph->weight[tid];
    p->cell[o] = ph->cell[tid];
    p->flag[o] = FLAG_SECONDARY | ((uint32_t)k << 29); /* electron, then positron */
  }
  ph->cell[tid] = OR_MAX_CELL;
}

void or_emit_photons(const or_mesh *m, const or_rad_params *rp, or_ptc *p, size_t ptc_num,
                     or_photons *ph, size_t *ph_num, size_t ph_cap, const or_fields *f,
                     float *photon_produced, uint32_t call, uint64_t first_id,
                     or_rad_counts *out) {
  const size_t base = *ph_num;
  size_t rank = 0, written = 0;
  for (size_t tid = 0; tid < ptc_num; ++tid) {
    const uint32_t cell = p->cell[tid];
    if (cell == OR_MAX_CELL || !in_bulk(m, cell)) continue;
    if ((p->flag[tid] >> 29) == 2u) continue; /* ions do not emit */
    float u[4];
    or_rad_uniforms(rp->seed, 1u, call, p->id[tid], u);
    if (!check_emit(m, rp, p, tid, u)) continue;
    if (photon_produced) AT2(photon_produced, c1_of(m, cell), c2_of(m, cell)) += p->weight[tid];
    const size_t off = base + rank;
    const uint64_t id = first_id + rank;
    rank++;
    if (off >= ph_cap) continue;
    ph->cell[off] = OR_MAX_CELL;
    emit_photon(m, rp, p, tid, ph, off, f, u);
    ph->flag[off] = u[2] < rp->track_percent ? FLAG_TRACKED : 0u;
    ph->id[off] = id;
    written++;
  }
  size_t n = base + rank + 1;
  *ph_num = n < ph_cap ? n : ph_cap;
  if (out) {
    out->marked = rank;
    out->written = written;
    out->dropped = rank - written;
  }
}

void or_produce_pairs(const or_mesh *m, const or_rad_params *rp, or_photons *ph, size_t ph_num,
                      or_ptc *p, size_t *ptc_num, size_t ptc_cap, const or_fields *f,
                      float *pair_produced, uint32_t call, uint64_t first_id,
                      or_rad_counts *out) {
  const size_t base = *ptc_num + 20;
  size_t rank = 0, written = 0;
  for (size_t tid = 0; tid < ph_num; ++tid) {
    const uint32_t cell = ph->cell[tid];
    if (cell == OR_MAX_CELL || !in_bulk(m, cell)) continue;
    if (rp->model == OR_RAD_GR1D || rp->model == OR_RAD_GAP1D) {
      float ug[4];
      or_rad_uniforms(rp->seed, 2u, call, ph->id[tid], ug);
      if (!(rp->model == OR_RAD_GR1D ? check_pair_gr(rp, ph, tid, ug)
                                     : check_pair_gap(rp, ph, tid, ug)))
        continue;
    } else if (!check_pair(m, rp, ph, tid, f)) {
      continue;
    }
    if (pair_produced) AT2(pair_produced, c1_of(m, cell), c2_of(m, cell)) += ph->weight[tid];
    const size_t off = base + 2 * rank;
    const uint64_t id = first_id + 2 * (uint64_t)rank;
    rank++;
    if (off + 1 >= ptc_cap) {
      ph->cell[tid] = OR_MAX_CELL;
      continue;
    }
    float u[4];
    or_rad_uniforms(rp->seed, 2u, call, ph->id[tid], u);
    p->cell[off] = p->cell[off + 1] = OR_MAX_CELL;
    p->flag[off] = p->flag[off + 1] = 0u;
    if (rp->model == OR_RAD_GR1D)
      produce_pair_gr(rp, ph, tid, p, off);
    else if (rp->model == OR_RAD_GAP1D)
      produce_pair_gap(m, ph, tid, p, off);
    else
      produce_pair(ph, tid, p, off);
    const int tracked = u[0] < rp->track_percent;
    for (int k = 0; k < 2; ++k) {
      if (tracked) p->flag[off + k] |= FLAG_TRACKED;
      p->id[off + k] = id + (uint64_t)k;
    }
    written++;
  }
  size_t n = *ptc_num + 2 * rank + 50;
  *ptc_num = n < ptc_cap ? n : ptc_cap;
  if (out) {
    out->marked = rank;
    out->written = written;
    out->dropped = rank - written;
  }
}

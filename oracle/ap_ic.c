/*
 * CPU oracle, inverse-Compton tables (TEST INFRASTRUCTURE ONLY).
 *
 * Restates inverse_compton (src/cuda/radiation/rt_ic.cu) and the background
 * spectra (src/radiation/spectra.h). The reference builds its tables in
 * host code of a .cu file, where a float argument selects the float
 * overload of log / exp / pow (logf, expf, powf) and a double argument the
 * double function; the types below follow the reference's declarations
 * (Scalar = float parameters of x_ic, sigma_ic, sigma_lab, beta and of the
 * spectra's operator(), double locals of init). Built with
 * -ffp-contract=off. The library computes the same sums on the GPU with
 * CUDA's functions, so the two agree to the last bits of those functions.
 *
 * Pinned: oracle/ref_build compiles the reference's own integrands and
 * inverse_compton::init for the host (libapref_ic.so, with the
 * constructor's few grid lines restated around them), and
 * tests/test_ic_oracle.py requires every table entry to be equal bit for
 * bit for each spectrum; the lookups are pinned through the 1D GR pin
 * (tests/test_rad_gr_pin.py), which runs the reference's own find_ic_rate,
 * find_gg_rate and gen_photon_e.
 */
#include "ap_ic.h"

#include <math.h>

#define IC_MIN_GAMMA 1.01f  /* rt_ic.cu:14 */
#define IC_MAX_GAMMA 1.0e15 /* rt_ic.cu:15 */
#define IC_MIN_EP 1.0e-10   /* rt_ic.cu:18 */
#define IC_N_MU 100         /* init: N_mu (rt_ic.cu:297) */
#define IC_N_E 800          /* init: N_e */
#define IC_RE_SQUARE 7.91402e-26          /* src/core/constant_defs.h:36 */
#define IC_PI 3.14159265358979323846      /* CONST_PI, constant_defs.h:11 */

/* Spectra (spectra.h:10-118): operator() of a float energy, except the
 * black body's (double). */
double or_spectrum_ne(const or_spectrum *s, double e_d) {
  const float e = (float)e_d;
  switch (s->kind) {
    case OR_SPEC_POWER_LAW_HARD:
      if (e < s->p[2] && e > s->p[1]) return (float)(powf(e / s->p[2], s->p[0]) / e);
      return 0.0f;
    case OR_SPEC_POWER_LAW_SOFT:
      if (e < s->p[2] && e > s->p[1]) return (float)(powf(e / s->p[1], -s->p[0]) / e);
      return 0.0f;
    case OR_SPEC_BROKEN_POWER_LAW:
      if (e < s->p[2] && e > s->p[3]) return (float)(powf(e / s->p[2], s->p[1]) / e);
      if (e > s->p[2] && e < s->p[4]) return (float)(powf(e / s->p[2], -s->p[0]) / e);
      return 0.0f;
    case OR_SPEC_BLACK_BODY:
      return 1.75464e30 * e_d * e_d / (exp(e_d / (double)s->p[0]) - 1.0);
    case OR_SPEC_MONO_ENERGETIC:
      if (e < s->p[0] + s->p[1] && e > s->p[0] - s->p[1]) return (float)(1.0 / (2.0 * s->p[1]));
      return 0.0f;
  }
  return 0.0;
}

double or_spectrum_emin(const or_spectrum *s) {
  switch (s->kind) {
    case OR_SPEC_POWER_LAW_HARD:
    case OR_SPEC_POWER_LAW_SOFT: return s->p[1];
    case OR_SPEC_BROKEN_POWER_LAW: return s->p[3];
    case OR_SPEC_BLACK_BODY: return (float)(1e-10 * s->p[0]);
    case OR_SPEC_MONO_ENERGETIC: return (float)(s->p[0] * 1e-2);
  }
  return 0.0;
}

double or_spectrum_emax(const or_spectrum *s) {
  switch (s->kind) {
    case OR_SPEC_POWER_LAW_HARD:
    case OR_SPEC_POWER_LAW_SOFT: return s->p[2];
    case OR_SPEC_BROKEN_POWER_LAW: return s->p[4];
    case OR_SPEC_BLACK_BODY: return (float)(1e3 * s->p[0]);
    case OR_SPEC_MONO_ENERGETIC: return (float)(s->p[0] * 1e2);
  }
  return 0.0;
}

/* beta, sigma_ic, sigma_gg, x_ic, sigma_lab (rt_ic.cu:21-60); square and
 * cube keep their argument's type. */
static double ic_beta(float gamma) { return 1.0 / sqrt(1.0 - 1.0 / (gamma * gamma)); }

static double ic_sigma(float x) {
  if (x < 1.0e-3) return 1.0f - 2.0f * x + 26.0f * x * x / 5.0f;
  const double l = log(1.0 + 2.0 * x);
  const double sq = (1.0 + 2.0 * x) * (1.0 + 2.0 * x);
  return 0.75 * ((1.0 + x) * (2.0 * x * (1.0 + x) / (1.0 + 2.0 * x) - l) / (x * x * x) +
                 0.5 * l / x - (1.0 + 3.0 * x) / sq);
}

static double gg_sigma(double b) {
  return (1.0 - b * b) *
         ((3.0 - b * b * b * b) * log((1.0 + b) / (1.0 - b)) - 2.0 * b * (2.0 - b * b));
}

static double ic_x(float gamma, float e, float mu) {
  return gamma * e * (1.0 - mu * ic_beta(gamma));
}

static double lab_sigma(float q, float ge) {
  const float gq = ge * q;
  return 2.0 * q * logf(q) + (1.0 + 2.0 * q) * (1.0 - q) +
         0.5 * (gq * gq) * (1.0 - q) / (1.0 + q * ge);
}

void or_ic_init(const or_spectrum *s, double emin_d, double emax_d, double n0,
                or_ic_tables *t) {
  const int ng = t->n_gamma, ne = t->n_ep;
  const float emin = (float)emin_d, emax = (float)emax_d;
  /* constructor (rt_ic.cu:223-246) */
  t->dep = (float)(1.0 / ((float)ne - 1.0));
  t->dlep = (float)((-log(IC_MIN_EP)) / ((float)ne - 1.0));
  t->dg = (float)((log(IC_MAX_GAMMA) - logf(IC_MIN_GAMMA)) / ((float)ng - 1.0));
  for (int n = 0; n < ng; ++n) t->gammas[n] = expf(logf(IC_MIN_GAMMA) + t->dg * (float)n);
  /* init (rt_ic.cu:292-435) */
  const double dmu = 2.0 / (IC_N_MU - 1.0);
  const double de = (logf(emax) - logf(emin)) / (IC_N_E - 1.0);
  const double loge = logf(emin);
  for (int n = 0; n < ng; ++n) {
    const double gamma = t->gammas[n];
    double result = 0.0;
    for (int i_mu = 0; i_mu < IC_N_MU; i_mu++) {
      const double mu = i_mu * dmu - 1.0;
      for (int i_e = 0; i_e < IC_N_E; i_e++) {
        const double e = exp(loge + i_e * de);
        const double x = ic_x((float)gamma, (float)e, (float)mu);
        const double sigma = ic_sigma((float)x);
        /* n_e(e) is float for every spectrum but the black body; half of
           it is exact in either type */
        result += 0.5 * or_spectrum_ne(s, e) * sigma * (1.0f - ic_beta((float)gamma) * mu) * e;
      }
    }
    t->ic_rate[n] = (float)(result * dmu * de * (IC_RE_SQUARE * n0) * 8.0 * IC_PI / 3.0);
  }
  for (int n = 0; n < ng; ++n) {
    const double eph = t->gammas[n];
    if (eph < 2.0) {
      t->gg_rate[n] = 0.0f;
      continue;
    }
    double result = 0.0;
    for (int i_mu = 0; i_mu < IC_N_MU; i_mu++) {
      const double mu = i_mu * dmu - 1.0;
      for (int i_e = 0; i_e < IC_N_E; i_e++) {
        const double e = exp(loge + i_e * de);
        const double sv = eph * e * (1.0 - mu) * 0.5;
        if (sv <= 1.0) continue;
        const double b = sqrt(1.0 - 1.0 / sv);
        if (b == 1.0) continue;
        result += gg_sigma(b) * (1.0 - mu) * or_spectrum_ne(s, e) * e;
      }
    }
    t->gg_rate[n] = (float)(0.25 * result * dmu * de * IC_PI * (n0 * IC_RE_SQUARE));
  }
  for (int tab = 0; tab < 2; ++tab) {
    float *d = tab == 0 ? t->dNde : t->dNde_thomson;
    for (int n = 0; n < ng; ++n) {
      const double gamma = t->gammas[n];
      float *row = d + (size_t)n * ne;
      for (int i = 0; i < ne; ++i) {
        /* m_ep[i] = dep * i; m_log_ep[i] = exp(dlep * i + log(MIN_EP)) */
        const double e1 = tab == 0 ? (double)(t->dep * (float)i)
                                   : (double)(float)exp(t->dlep * (float)i + log(IC_MIN_EP));
        double result = 0.0;
        for (int i_e = 0; i_e < IC_N_E; i_e++) {
          const double e = exp(loge + i_e * de);
          const double nev = or_spectrum_ne(s, e);
          const double ge = gamma * e * 4.0;
          const double q = e1 / (ge * (1.0 - e1));
          if (e1 < ge / (1.0 + ge) && e1 > e / gamma)
            result += nev * lab_sigma((float)q, (float)ge) / gamma;
        }
        row[i] = tab == 0 ? (float)(result * de) : (float)(result * de * e1);
      }
      for (int i = 1; i < ne; ++i) row[i] += row[i - 1];
      for (int i = 0; i < ne; ++i) row[i] /= row[ne - 1];
    }
  }
}

/* find_n_gamma (rt_ic.cu:77-81); the index is clamped to the table. */
static int n_gamma_of(const or_ic_tables *t, float gamma) {
  if (gamma < IC_MIN_GAMMA) return 0;
  if (gamma > IC_MAX_GAMMA) return t->n_gamma - 1;
  int n = (int)((logf(gamma) - logf(IC_MIN_GAMMA)) / t->dg);
  return n < t->n_gamma - 1 ? n : t->n_gamma - 1;
}

/* find_ic_rate / find_gg_rate (rt_ic.cu:155-170): linear in log gamma
 * between gammas[n] and gammas[n + 1]; at the last entry the reference
 * reads one past the table, here the last entry is used for both. */
static float rate_of(const or_ic_tables *t, const float *rate, float g) {
  const int n = n_gamma_of(t, g);
  if (g > IC_MAX_GAMMA) return rate[n];
  const float x = (logf(g) - logf(t->gammas[n])) / t->dg;
  const int n1 = n + 1 < t->n_gamma ? n + 1 : n;
  return rate[n] * (1.0f - x) + rate[n1] * x;
}

float or_ic_rate(const or_ic_tables *t, float gamma) { return rate_of(t, t->ic_rate, gamma); }

float or_gg_rate(const or_ic_tables *t, float eph) {
  if (eph < 2.0) return 0.0f;
  return rate_of(t, t->gg_rate, eph);
}

/* binary_search (rt_ic.cu:89-117) over one row of `size` entries. */
static int bsearch_row(float u, const float *a, int size, float *l, float *h) {
  int lo = 0, hi = size - 1, tmp = 0;
  float v = 0.0f;
  while (lo < hi) {
    tmp = (lo + hi) / 2;
    v = a[tmp];
    if (v < u) {
      lo = tmp + 1;
    } else if (v > u) {
      hi = tmp - 1;
    } else {
      hi = tmp;
      *l = *h = v;
      return hi;
    }
  }
  if (v < u) {
    *l = v;
    *h = (lo < size ? a[lo] : v);
    return tmp;
  }
  *h = v;
  *l = (hi >= 0 ? a[hi] : v);
  return hi > 0 ? hi : 0;
}

/* gen_photon_e (rt_ic.cu:128-153). */
float or_ic_photon_e(const or_ic_tables *t, float gamma, float u) {
  const int gn = n_gamma_of(t, gamma);
  float l, h, bb;
  double result;
  int b = bsearch_row(u, t->dNde + (size_t)gn * t->n_ep, t->n_ep, &l, &h);
  if (b < 2) {
    b = bsearch_row(u, t->dNde_thomson + (size_t)gn * t->n_ep, t->n_ep, &l, &h);
    bb = (l == h ? (float)b : (u - l) / (h - l) + (float)b);
    result = exp(t->dlep * bb + log(IC_MIN_EP));
  } else {
    bb = (l == h ? (float)b : (u - l) / (h - l) + (float)b);
    result = t->dep * bb;
  }
  /* the device min / max of doubles: fmin / fmax */
  return (float)fmax(fmin(result * gamma, gamma - 1.01), 0.0);
}

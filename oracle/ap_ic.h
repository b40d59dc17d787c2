/*
 * CPU oracle, inverse-Compton tables (TEST INFRASTRUCTURE ONLY); see ap_ic.c
 * for the reference lines each function restates.
 */
#ifndef AP_IC_H_
#define AP_IC_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Background photon spectra (src/radiation/spectra.h). */
enum {
  OR_SPEC_POWER_LAW_HARD = 0,   /* p = {delta, emin, emax}                     */
  OR_SPEC_POWER_LAW_SOFT = 1,   /* p = {alpha, emin, emax}                     */
  OR_SPEC_BROKEN_POWER_LAW = 2, /* p = {alpha, delta, epeak, emin, emax}       */
  OR_SPEC_BLACK_BODY = 3,       /* p = {kT}                                    */
  OR_SPEC_MONO_ENERGETIC = 4    /* p = {e0, de}                                */
};
typedef struct {
  int kind;
  float p[5];
} or_spectrum;

/* The tables of inverse_compton (src/cuda/radiation/rt_ic.cu): per Lorentz
 * factor gammas[n] (n < n_gamma) the scattering rate, the gamma-gamma pair
 * rate, and two cumulative, normalised photon-energy distributions of
 * n_ep entries each (row n at n * n_ep): over e1 = dep * i (dNde) and over
 * e1 = exp(dlep * i + log(1e-10)) (dNde_thomson). Caller-allocated. */
typedef struct {
  int n_gamma, n_ep;
  float dep, dg, dlep;
  float *ic_rate, *gg_rate, *gammas;
  float *dNde, *dNde_thomson;
} or_ic_tables;

/* The spectrum's density n_e(e) as the reference's functor returns it. */
double or_spectrum_ne(const or_spectrum *s, double e);
/* emin() / emax() of the spectrum. */
double or_spectrum_emin(const or_spectrum *s);
double or_spectrum_emax(const or_spectrum *s);

/* inverse_compton's constructor and init(n_e, emin, emax, n0). */
void or_ic_init(const or_spectrum *s, double emin, double emax, double n0, or_ic_tables *t);

/* find_ic_rate, find_gg_rate and gen_photon_e (rt_ic.cu:77-170) with the
 * uniform u of the photon energy draw. */
float or_ic_rate(const or_ic_tables *t, float gamma);
float or_gg_rate(const or_ic_tables *t, float eph);
float or_ic_photon_e(const or_ic_tables *t, float gamma, float u);

#ifdef __cplusplus
}
#endif

#endif /* AP_IC_H_ */

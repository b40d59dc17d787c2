/*
 * Oracle pin build, inverse-Compton tables (TEST INFRASTRUCTURE ONLY): runs
 * the reference's own inverse_compton::init on the host.
 *
 * The Makefile copies beta, sigma_ic, sigma_gg, x_ic, sigma_lab and the
 * member template inverse_compton::init from src/cuda/radiation/rt_ic.cu
 * into oracle/_ref/ic_kernels.inc (extract_kernels.py; the rest of that file
 * launches kernels and fills device arrays) and includes them unmodified.
 * The class around them keeps the members init names, on host vectors
 * (copy_to_device does nothing); the spectra are src/radiation/spectra.h
 * unmodified. As in the reference's .cu host code, unqualified log, exp,
 * sqrt and pow of float arguments are the float functions (ls_host_math.h
 * and the using-declaration below).
 *
 * The constructor's grid (rt_ic.cu:223-246: dep, dlep, dg, the Lorentz
 * factors and the two energy axes) sets device symbols and cuRAND states
 * around a few lines of arithmetic; those lines are restated in
 * ref_ic_init below, with the reference's expressions.
 */
#include "ls_host_math.h"
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <vector>
using std::pow;

#include "cuda/cuda_control.h"
#include "core/constant_defs.h"
#include "core/typedefs.h"
#include "utils/util_functions.h"
#include "radiation/spectra.h"

#define MIN_GAMMA 1.01f  /* rt_ic.cu:14-18 */
#define MAX_GAMMA 1.0e15
#define MIN_EP 1.0e-10

namespace Aperture {

struct Logger {
  template <typename... Args>
  static void print_info(const char *, const Args &...) {}
};

template <typename T>
struct host_array {
  std::vector<T> v;
  T &operator[](size_t i) { return v[i]; }
  const T &operator[](size_t i) const { return v[i]; }
  size_t size() const { return v.size(); }
  void copy_to_device() {}
};

template <typename T>
struct host_multi_array {
  std::vector<T> v;
  size_t nx = 0;
  T &operator()(size_t i, size_t j) { return v[i + j * nx]; }
  void copy_to_device() {}
};

class inverse_compton {
 public:
  template <typename F>
  void init(const F &n_e, Scalar emin, Scalar emax, double n0 = 1.0);

  host_multi_array<Scalar> m_dNde, m_dNde_thomson;
  host_array<Scalar> m_ic_rate, m_gg_rate, m_gammas, m_log_ep, m_ep;
  Scalar m_dep, m_dg, m_dlep;
};

#include "ic_kernels.inc"

}  // namespace Aperture

using namespace Aperture;

template <typename F>
static void run(inverse_compton &ic, const F &ne, float emin, float emax, double n0) {
  ic.init(ne, emin, emax, n0);
}

extern "C" {

/* inverse_compton(params) with n_gamma x n_ep, then init(n_e, emin, emax,
 * n0) for spectrum `kind` (0 power_law_hard, 1 power_law_soft,
 * 2 broken_power_law, 3 black_body, 4 mono_energetic; p = the constructor's
 * arguments). Copies the tables out; steps = {dep, dg, dlep}. */
int ref_ic_init(int kind, const float p[5], float emin, float emax, double n0, int ng, int ne,
                float *ic_rate, float *gg_rate, float *gammas, float *dNde, float *dNde_th,
                float *steps) {
  inverse_compton ic;
  ic.m_dNde.v.assign((size_t)ng * ne, 0.0f);
  ic.m_dNde.nx = (size_t)ne;
  ic.m_dNde_thomson.v.assign((size_t)ng * ne, 0.0f);
  ic.m_dNde_thomson.nx = (size_t)ne;
  for (auto *a : {&ic.m_ic_rate, &ic.m_gg_rate, &ic.m_gammas}) a->v.assign((size_t)ng, 0.0f);
  for (auto *a : {&ic.m_log_ep, &ic.m_ep}) a->v.assign((size_t)ne, 0.0f);
  // the constructor's grid (rt_ic.cu:230-246)
  ic.m_dep = 1.0 / ((Scalar)ic.m_ep.size() - 1.0);
  for (uint32_t n = 0; n < ic.m_ep.size(); n++) ic.m_ep[n] = ic.m_dep * n;
  ic.m_dlep = (-log(MIN_EP)) / ((Scalar)ic.m_log_ep.size() - 1.0);
  for (uint32_t n = 0; n < ic.m_ep.size(); n++)
    ic.m_log_ep[n] = exp(ic.m_dlep * n + log(MIN_EP));
  ic.m_dg = (log(MAX_GAMMA) - log(MIN_GAMMA)) / ((Scalar)ng - 1.0);
  for (uint32_t n = 0; n < ic.m_gammas.size(); n++)
    ic.m_gammas[n] = exp(log(MIN_GAMMA) + ic.m_dg * (Scalar)n);
  switch (kind) {
    case 0: run(ic, Spectra::power_law_hard(p[0], p[1], p[2]), emin, emax, n0); break;
    case 1: run(ic, Spectra::power_law_soft(p[0], p[1], p[2]), emin, emax, n0); break;
    case 2: run(ic, Spectra::broken_power_law(p[0], p[1], p[2], p[3], p[4]), emin, emax, n0); break;
    case 3: run(ic, Spectra::black_body(p[0]), emin, emax, n0); break;
    case 4: run(ic, Spectra::mono_energetic(p[0], p[1]), emin, emax, n0); break;
    default: return -1;
  }
  for (int n = 0; n < ng; ++n) {
    ic_rate[n] = ic.m_ic_rate[n];
    gg_rate[n] = ic.m_gg_rate[n];
    gammas[n] = ic.m_gammas[n];
  }
  for (size_t k = 0; k < (size_t)ng * ne; ++k) {
    dNde[k] = ic.m_dNde.v[k];
    dNde_th[k] = ic.m_dNde_thomson.v[k];
  }
  steps[0] = ic.m_dep;
  steps[1] = ic.m_dg;
  steps[2] = ic.m_dlep;
  return 0;
}

}  // extern "C"

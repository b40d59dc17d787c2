// inverse_compton (src/cuda/radiation/rt_ic.cu:207-435): the rate and
// photon-energy tables for a background spectrum (src/radiation/spectra.h).
//
// The reference fills them in host code, entry after entry: 100 angles x
// 800 energies for each of the n_gamma scattering and pair rates, 800
// energies for each of the 2 x n_gamma x n_ep spectrum entries (about
// 0.7 G integrand evaluations at the default 600 x 600). Here:
//   k_ic_rates: one CTA per Lorentz factor sums both rates' 80,000 terms
//               over its threads and reduces them in a fixed order;
//   k_ic_dnde:  one thread per spectrum entry, its 800 terms in order;
//   k_ic_cumsum: one thread per row, the float cumulative sum and the
//               normalisation in the reference's order.
// The integrands keep the reference's expressions and types (Scalar =
// float parameters, double locals; in its .cu host code a float argument
// selects logf / expf / powf). The grid constants (dep, dg, dlep, the
// Lorentz factors) are computed on the host exactly as the reference's
// constructor does.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "ap_internal.h"

namespace apb {

namespace {

constexpr int kIcNmu = 100;                   // init: N_mu (rt_ic.cu:297)
constexpr int kIcNe = 800;                    // init: N_e
constexpr double kIcReSquare = 7.91402e-26;   // RE_SQUARE (src/core/constant_defs.h:36)
constexpr double kIcPi = 3.14159265358979323846;
constexpr float kMinGamma = 1.01f;            // MIN_GAMMA
constexpr double kMaxGamma = 1.0e15;          // MAX_GAMMA
constexpr double kMinEp = 1.0e-10;            // MIN_EP
constexpr int kRateThreads = 256;

// n_e(e) of the spectra: operator() of a float energy (the black body's of
// a double), returned in its type.
__device__ double spec_ne(const ap_spectrum &s, double e_d) {
  const float e = (float)e_d;
  switch (s.kind) {
    case AP_SPEC_POWER_LAW_HARD:
      if (e < s.p[2] && e > s.p[1]) return powf(e / s.p[2], s.p[0]) / e;
      return 0.0f;
    case AP_SPEC_POWER_LAW_SOFT:
      if (e < s.p[2] && e > s.p[1]) return powf(e / s.p[1], -s.p[0]) / e;
      return 0.0f;
    case AP_SPEC_BROKEN_POWER_LAW:
      if (e < s.p[2] && e > s.p[3]) return powf(e / s.p[2], s.p[1]) / e;
      if (e > s.p[2] && e < s.p[4]) return powf(e / s.p[2], -s.p[0]) / e;
      return 0.0f;
    case AP_SPEC_BLACK_BODY:
      return 1.75464e30 * e_d * e_d / (exp(e_d / (double)s.p[0]) - 1.0);
    default:  // AP_SPEC_MONO_ENERGETIC
      if (e < s.p[0] + s.p[1] && e > s.p[0] - s.p[1]) return (float)(1.0 / (2.0 * s.p[1]));
      return 0.0f;
  }
}

// beta, sigma_ic, sigma_gg, x_ic, sigma_lab (rt_ic.cu:21-60).
__device__ __forceinline__ double ic_beta(float gamma) {
  return 1.0 / sqrt(1.0 - 1.0 / (gamma * gamma));
}
__device__ double ic_sigma(float x) {
  if ((double)x < 1.0e-3) return 1.0f - 2.0f * x + 26.0f * x * x / 5.0f;
  const double l = log(1.0 + 2.0 * x);
  const double sq = (1.0 + 2.0 * x) * (1.0 + 2.0 * x);
  return 0.75 * ((1.0 + x) * (2.0 * x * (1.0 + x) / (1.0 + 2.0 * x) - l) / (x * x * x) +
                 0.5 * l / x - (1.0 + 3.0 * x) / sq);
}
__device__ __forceinline__ double gg_sigma(double b) {
  return (1.0 - b * b) *
         ((3.0 - b * b * b * b) * log((1.0 + b) / (1.0 - b)) - 2.0 * b * (2.0 - b * b));
}
__device__ __forceinline__ double ic_x(float gamma, float e, float mu) {
  return gamma * e * (1.0 - mu * ic_beta(gamma));
}
__device__ __forceinline__ double lab_sigma(float q, float ge) {
  const float gq = ge * q;
  return 2.0 * q * logf(q) + (1.0 + 2.0 * q) * (1.0 - q) +
         0.5 * (gq * gq) * (1.0 - q) / (1.0 + q * ge);
}

struct IcGrid {
  double loge, de, dmu, n0;  // log(emin) (float log), energy and angle steps
  int n_gamma, n_ep;
  float dep, dlep;
};

// Both rates of Lorentz factor blockIdx.x (init, rt_ic.cu:299-354).
__global__ void __launch_bounds__(kRateThreads)
    k_ic_rates(ap_spectrum s, IcGrid G, const float *gammas, float *ic_rate, float *gg_rate) {
  __shared__ double s_ic[kRateThreads], s_gg[kRateThreads];
  const int n = blockIdx.x;
  const double gamma = gammas[n];
  const bool gg = gamma >= 2.0;
  double ric = 0.0, rgg = 0.0;
  for (int k = threadIdx.x; k < kIcNmu * kIcNe; k += kRateThreads) {
    const int i_mu = k / kIcNe, i_e = k - i_mu * kIcNe;
    const double mu = i_mu * G.dmu - 1.0;
    const double e = exp(G.loge + i_e * G.de);
    const double ne = spec_ne(s, e);
    const double x = ic_x((float)gamma, (float)e, (float)mu);
    const double sigma = ic_sigma((float)x);
    // n_e is float for every spectrum but the black body; half of it is
    // exact in either type
    ric += 0.5 * ne * sigma * (1.0f - ic_beta((float)gamma) * mu) * e;
    if (gg) {
      const double sv = gamma * e * (1.0 - mu) * 0.5;
      if (sv > 1.0) {
        const double b = sqrt(1.0 - 1.0 / sv);
        if (b != 1.0) rgg += gg_sigma(b) * (1.0 - mu) * ne * e;
      }
    }
  }
  s_ic[threadIdx.x] = ric;
  s_gg[threadIdx.x] = rgg;
  __syncthreads();
  for (int w = kRateThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s_ic[threadIdx.x] += s_ic[threadIdx.x + w];
      s_gg[threadIdx.x] += s_gg[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    ic_rate[n] = (float)(s_ic[0] * G.dmu * G.de * (kIcReSquare * G.n0) * 8.0 * kIcPi / 3.0);
    gg_rate[n] = gg ? (float)(0.25 * s_gg[0] * G.dmu * G.de * kIcPi * (G.n0 * kIcReSquare))
                    : 0.0f;
  }
}

// One entry of the lab-frame spectrum (rt_ic.cu:381-432): table 0 over
// e1 = dep * i, table 1 (Thomson) over e1 = exp(dlep * i + log(MIN_EP)),
// times e1. The float entries before the cumulative sum.
__global__ void k_ic_dnde(ap_spectrum s, IcGrid G, const float *gammas, float *dNde,
                          float *dNde_th) {
  const size_t per = (size_t)G.n_gamma * G.n_ep;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < 2 * per;
       t += (size_t)gridDim.x * blockDim.x) {
    const int tab = t < per ? 0 : 1;
    const size_t k = t - (size_t)tab * per;
    const int n = (int)(k / G.n_ep), i = (int)(k - (size_t)n * G.n_ep);
    const double gamma = gammas[n];
    const double e1 = tab == 0 ? (double)(G.dep * (float)i)
                               : (double)(float)exp(G.dlep * (float)i + log(kMinEp));
    double result = 0.0;
    for (int i_e = 0; i_e < kIcNe; i_e++) {
      const double e = exp(G.loge + i_e * G.de);
      const double ne = spec_ne(s, e);
      const double ge = gamma * e * 4.0;
      const double q = e1 / (ge * (1.0 - e1));
      if (e1 < ge / (1.0 + ge) && e1 > e / gamma) result += ne * lab_sigma((float)q, (float)ge) / gamma;
    }
    if (tab == 0)
      dNde[k] = (float)(result * G.de);
    else
      dNde_th[k] = (float)(result * G.de * e1);
  }
}

// Cumulative sum along each row and the division by its last entry, in
// float and in the reference's order.
__global__ void k_ic_cumsum(float *dNde, float *dNde_th, int n_gamma, int n_ep) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * n_gamma) return;
  float *row = (t < n_gamma ? dNde : dNde_th) + (size_t)(t % n_gamma) * n_ep;
  for (int i = 1; i < n_ep; ++i) row[i] += row[i - 1];
  const float last = row[n_ep - 1];
  for (int i = 0; i < n_ep; ++i) row[i] /= last;
}

}  // namespace

int ic_init(Ctx &c, const ap_spectrum &s, double emin_d, double emax_d, double n0, int ng,
            int ne) {
  if (ng < 2 || ne < 2 || ng > (1 << 16) || ne > (1 << 16)) return AP_ERR_INVALID;
  const size_t words = 3 * (size_t)ng + 2 * (size_t)ng * ne;
  if (!c.ic_buf || c.ic_n_gamma != ng || c.ic_n_ep != ne) {
    cudaFree(c.ic_buf);
    c.ic_buf = nullptr;
    if (cudaMalloc(&c.ic_buf, words * sizeof(float)) != cudaSuccess) return AP_ERR_NOMEM;
  }
  c.ic_ready = false;
  // the constructor's grid (rt_ic.cu:223-246), on the host as there
  const float dep = (float)(1.0 / ((float)ne - 1.0));
  const float dlep = (float)((-std::log(kMinEp)) / ((float)ne - 1.0));
  const float dg = (float)((std::log(kMaxGamma) - std::log(kMinGamma)) / ((float)ng - 1.0));
  std::vector<float> gammas((size_t)ng);
  for (int n = 0; n < ng; ++n) gammas[n] = std::exp(std::log(kMinGamma) + dg * (float)n);
  float *ic_rate = c.ic_buf, *gg_rate = ic_rate + ng, *g = gg_rate + ng;
  float *dNde = g + ng, *dNde_th = dNde + (size_t)ng * ne;
  cudaError_t e =
      cudaMemcpyAsync(g, gammas.data(), sizeof(float) * ng, cudaMemcpyHostToDevice, c.stream);
  if (e != cudaSuccess) return AP_ERR_CUDA;
  const float emin = (float)emin_d, emax = (float)emax_d;
  IcGrid G;
  G.dmu = 2.0 / (kIcNmu - 1.0);
  G.de = (std::log(emax) - std::log(emin)) / (kIcNe - 1.0);
  G.loge = std::log(emin);
  G.n0 = n0;
  G.n_gamma = ng;
  G.n_ep = ne;
  G.dep = dep;
  G.dlep = dlep;
  k_ic_rates<<<ng, kRateThreads, 0, c.stream>>>(s, G, g, ic_rate, gg_rate);
  const size_t entries = 2 * (size_t)ng * ne;
  const int grid = (int)((entries + 255) / 256 < (size_t)c.num_sms * 32 ? (entries + 255) / 256
                                                                        : (size_t)c.num_sms * 32);
  k_ic_dnde<<<grid, 256, 0, c.stream>>>(s, G, g, dNde, dNde_th);
  k_ic_cumsum<<<(2 * ng + 127) / 128, 128, 0, c.stream>>>(dNde, dNde_th, ng, ne);
  c.launches += 3;
  if (cudaGetLastError() != cudaSuccess) return AP_ERR_CUDA;
  c.ic_n_gamma = ng;
  c.ic_n_ep = ne;
  c.ic_dep = dep;
  c.ic_dg = dg;
  c.ic_dlep = dlep;
  c.ic_spec = s;
  c.ic_emin = emin_d;
  c.ic_emax = emax_d;
  c.ic_n0 = n0;
  c.ic_ready = true;
  return AP_OK;
}

void ic_free(Ctx &c) {
  cudaFree(c.ic_buf);
  c.ic_buf = nullptr;
  c.ic_ready = false;
}

}  // namespace apb

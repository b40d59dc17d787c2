// Inverse-Compton table lookups on the device: find_n_gamma, find_ic_rate,
// find_gg_rate, binary_search and gen_photon_e of src/cuda/radiation/
// rt_ic.cu:77-170, over the tables that k_ic.cu builds (ap_ic_init).
#pragma once

#include <cuda_runtime.h>

namespace apb {

constexpr float kIcMinGamma = 1.01f;  // MIN_GAMMA (rt_ic.cu:14)
constexpr double kIcMaxGamma = 1.0e15;  // MAX_GAMMA (:15)
constexpr double kIcMinEp = 1.0e-10;    // MIN_EP (:18)

struct IcK {
  const float *ic_rate, *gg_rate, *gammas;  // n_gamma each
  const float *dNde, *dNde_th;              // n_gamma rows of n_ep
  int n_gamma, n_ep;
  float dep, dg, dlep;
};

// find_n_gamma; the index is clamped to the table (the reference's can
// reach n_gamma through float rounding just below MAX_GAMMA).
__device__ __forceinline__ int ic_n_gamma(const IcK &T, float gamma) {
  if (gamma < kIcMinGamma) return 0;
  if ((double)gamma > kIcMaxGamma) return T.n_gamma - 1;
  const int n = (int)((logf(gamma) - logf(kIcMinGamma)) / T.dg);
  return n < T.n_gamma - 1 ? n : T.n_gamma - 1;
}

// find_ic_rate / find_gg_rate: linear in log gamma between gammas[n] and
// gammas[n + 1]; where the reference reads one past the table (the last
// entry), the last entry is used for both ends.
__device__ __forceinline__ float ic_interp(const IcK &T, const float *rate, float g) {
  const int n = ic_n_gamma(T, g);
  if ((double)g > kIcMaxGamma) return rate[n];
  const float x = (logf(g) - logf(T.gammas[n])) / T.dg;
  const int n1 = n + 1 < T.n_gamma ? n + 1 : n;
  return rate[n] * (1.0f - x) + rate[n1] * x;
}
__device__ __forceinline__ float ic_rate(const IcK &T, float gamma) {
  return ic_interp(T, T.ic_rate, gamma);
}
__device__ __forceinline__ float gg_rate(const IcK &T, float eph) {
  if ((double)eph < 2.0) return 0.0f;
  return ic_interp(T, T.gg_rate, eph);
}

// binary_search over one row of `size` entries (rt_ic.cu:89-117): the
// entry index and the bracketing values l <= u <= h.
__device__ __forceinline__ int ic_bsearch(float u, const float *a, int size, float &l, float &h) {
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
      l = h = v;
      return hi;
    }
  }
  if (v < u) {
    l = v;
    h = (lo < size ? a[lo] : v);
    return tmp;
  }
  h = v;
  l = (hi >= 0 ? a[hi] : v);
  return hi > 0 ? hi : 0;
}

// gen_photon_e (rt_ic.cu:128-153) with the uniform u of the draw.
__device__ __forceinline__ float ic_photon_e(const IcK &T, float gamma, float u) {
  const int gn = ic_n_gamma(T, gamma);
  float l, h, bb;
  double result;
  int b = ic_bsearch(u, T.dNde + (size_t)gn * T.n_ep, T.n_ep, l, h);
  if (b < 2) {
    b = ic_bsearch(u, T.dNde_th + (size_t)gn * T.n_ep, T.n_ep, l, h);
    bb = (l == h ? (float)b : (u - l) / (h - l) + (float)b);
    result = exp(T.dlep * bb + log(kIcMinEp));
  } else {
    bb = (l == h ? (float)b : (u - l) / (h - l) + (float)b);
    result = T.dep * bb;
  }
  return (float)fmax(fmin(result * gamma, gamma - 1.01), 0.0);
}

}  // namespace apb

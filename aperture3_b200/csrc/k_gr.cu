// 1D GR lab path (src/cuda/algorithms/ptc_updater_1dgr.cu,
// field_solver_1dgr.cu, src/grids/grid_1dgr.cpp): the radial pusher along
// a field line of a Kerr black hole's magnetosphere (GR terms from the
// metric coefficients D1, D2, D3, alpha and the smoothed E3), its current /
// charge deposit weighted by the flux-tube factors K1_j and K1, the
// K1-weighted 1-2-1 filter, and the E1 update E1 += (j0 - J1) dt.
//
// The push keeps the reference's float / double mix operation by operation
// (-fmad=false, IEEE float division and square root); its one transcendental
// is the float exp of the tortoise coordinate, evaluated with CUDA's expf as
// the reference's device code does, so particles agree with an FP32 CPU
// evaluation to the last bits of that exponential. The deposit accumulates
// exact fixed-point sums in a shared-memory window over each chunk's cells,
// as the other 1D kernels do. The metric coefficients are computed on the
// host exactly as Grid_1dGR::compute_coef does (host_gr_coef).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

#include "ap_device.cuh"
#include "ap_internal.h"

namespace apb {

namespace {

constexpr int kGrThreads = 256;
constexpr int kGrItems = 8;
constexpr int kGrChunk = kGrThreads * kGrItems;  // 2048 particle slots
constexpr int kGrWin = 6000;                     // cell-components per window
constexpr uint32_t kFlagTracked = 1u << 1;  // ParticleFlag::tracked (enum_types.h:76-87)

__device__ __forceinline__ int bits_of_u32(uint32_t v) { return 32 - __clz(v | 1u); }

__device__ __forceinline__ void win_add(int *hi, unsigned *lo, int o, float v, float scale,
                                        int L) {
  const long long X = __float2ll_rn(v * scale);  // exact scaling by a power of two
  atomicAdd(hi + o, (int)(X >> L));
  atomicAdd(lo + o, (unsigned)X & ((1u << L) - 1u));
}

// One chunk of slots: update_ptc_1dgr (ptc_updater_1dgr.cu:137-300) per
// live particle. Window components: 0 = J1, 1 + sp = Rho[sp].
__device__ void gr_chunk(const PushDepositParams &P, const GrK &G, size_t ch, int *sWhi,
                         unsigned *sWlo, int &s_lo, int &s_hi) {
  const int tid = threadIdx.x;
  const int n0 = P.m.dims[0], g0 = P.m.guard[0];
  const int ns = P.num_species;
  const int ncomp = 1 + ns;
  const int win_comp = kGrWin / ncomp;
  const int lgw = bits_of_u32(kGrChunk);
  const int lgn = bits_of_u32((uint32_t)min(P.number, (size_t)0x7fffffff));
  const int B = min(63 - 2 * lgw, 62 - lgn);
  const float qw = P.qmax * *P.wmax;
  int S = B - 2;
  if (qw > 0.0f) S -= ilogbf(qw);
  S = max(-100, min(100, S));
  const int L = 32 - lgw;
  const float fscale = ldexpf(1.0f, S);
  if (ch == 0 && tid == 0) *P.fx_used = FixedFmt{S, L};
  const size_t first = ch * kGrChunk;
  if (tid == 0) {
    s_lo = INT_MAX;
    s_hi = INT_MIN;
  }
  __syncthreads();
  uint32_t cells[kGrItems];
  int lo = INT_MAX, hi = INT_MIN;
#pragma unroll
  for (int k = 0; k < kGrItems; ++k) {
    const size_t idx = first + (size_t)k * kGrThreads + tid;
    cells[k] = idx < P.number ? P.p.cell[idx] : AP_MAX_CELL;
    if (cells[k] != AP_MAX_CELL) {
      lo = min(lo, (int)cells[k]);
      hi = max(hi, (int)cells[k]);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((tid & 31) == 0 && lo <= hi) {
    atomicMin(&s_lo, lo);
    atomicMax(&s_hi, hi);
  }
  __syncthreads();
  const int wlo = s_lo - 2;
  const int wlen = s_hi - s_lo + 5;
  const bool use_smem = (s_lo <= s_hi) && wlen <= win_comp;
  if (use_smem)
    for (int i = tid; i < ncomp * win_comp; i += kGrThreads) {
      sWhi[i] = 0;
      sWlo[i] = 0u;
    }
  __syncthreads();

  const float *E3 = P.F[2].ptr;
  const float lower = P.m.lower[0], delta = P.m.delta[0], inv_delta = P.m.inv_delta[0];
  const float dt = P.dt, a = G.a;
#pragma unroll 1
  for (int k = 0; k < kGrItems; ++k) {
    const size_t idx = first + (size_t)k * kGrThreads + tid;
    const uint32_t c = cells[k];
    if (c == AP_MAX_CELL) continue;
    if ((int)c < g0 || (int)c >= n0 - g0) {  // is_in_bulk
      P.p.cell[idx] = AP_MAX_CELL;
      continue;
    }
    float p1 = P.p.p1[idx];
    const float x1 = P.p.x1[idx];
    float u0 = P.p.E[idx];
    float nx1 = 1.0f - x1;
    const uint32_t flag = P.p.flag[idx];
    const int sp = ptc_type(flag);
    const float xi = mesh_pos(lower, delta, (int)c, g0, x1);
    const float rp = 1.0f + sqrtf(1.0f - a * a);
    const float rm = 1.0f - sqrtf(1.0f - a * a);
    const float exp_xi = expf(xi * (rp - rm));
    const float r = (float)((double)(rp - rm * exp_xi) / (1.0 - (double)exp_xi));
    // interpolated coefficients (:173-191)
    float alpha = G.alpha[c] * x1 + G.alpha[c - 1] * nx1;
    float D1 = G.D1[c] * x1 + G.D1[c - 1] * nx1;
    float D2 = G.D2[c] * x1 + G.D2[c - 1] * nx1;
    float D3 = G.D3[c] * x1 + G.D3[c - 1] * nx1;
    const float Dxi = (x1 < 0.5f ? E3[c] * (0.5f + x1) + E3[c - 1] * (0.5f - x1)
                                 : E3[c] * (1.5f - x1) + E3[c + 1] * (x1 - 0.5f));
    const float agrr = G.agrr[c] * x1 + G.agrr[c - 1] * nx1;
    const float Er = agrr * Dxi;
    float vr = (p1 / u0 - D1) / D2;
    const float da2dr = (G.alpha[c] * G.alpha[c] - G.alpha[c - 1] * G.alpha[c - 1]) * inv_delta;
    const float dD1dr = (G.D1[c] - G.D1[c - 1]) * inv_delta;
    const float dD2dr = (G.D2[c] - G.D2[c - 1]) * inv_delta;
    const float dD3dr = (G.D3[c] - G.D3[c - 1]) * inv_delta;
    const float dDelta_dr = (float)((double)(2.0f * r) - 2.0);
    // momentum (:213-226)
    const float gr_term = -0.5f * u0 *
                              (da2dr - (dD3dr + 2.0f * (dD1dr - D1 * dDelta_dr) * vr +
                                        (dD2dr - 2.0f * D2 * dDelta_dr) * vr * vr)) *
                              dt +
                          dDelta_dr * p1 * vr * dt;
    p1 += gr_term;
    const float E_term = Er * P.charge[sp] / P.mass[sp] * dt;
    p1 += E_term;
    u0 = sqrtf((D2 + p1 * p1) / (D2 * (alpha * alpha - D3) + D1 * D1));
    P.p.p1[idx] = p1;
    vr = (p1 / u0 - D1) / D2;
    if (G.step % (uint32_t)G.data_interval == 0 && (flag & kFlagTracked)) {
      // lower u_0 of tracked particles into p2 (:232-246)
      const float theta = G.theta[c] * x1 + G.theta[c - 1] * nx1;
      const float ct = cosf(theta), st = sinf(theta);
      const float Sigma = (r * r + a * a * (ct * ct));
      const float Delta = (r * r - 2.0f * r + a * a);
      const float g_00 = -(1.0f - 2.0f * r / Sigma);
      const float g_03 = (float)(-4.0 * (double)r * (double)a * (double)(st * st) / (double)Sigma);
      const float B31 = G.B3B1[c] * x1 + G.B3B1[c - 1] * nx1;
      P.p.p2[idx] = (g_00 + g_03 * G.omega) * u0 + g_03 * B31 * Delta * u0 * vr;
    }
    // move (:249-264); a move of more than one cell, which the reference
    // reports and continues past the coefficient arrays, empties the slot
    float new_x1 = x1 + vr * dt * inv_delta;
    const int dc1 = (int)floorf(new_x1);
    if (dc1 > 1 || dc1 < -1) {
      atomicAdd(&P.status->moved_far, 1ull);
      P.p.cell[idx] = AP_MAX_CELL;
      continue;
    }
    new_x1 -= (float)dc1;
    const uint32_t cn = c + dc1;
    P.p.cell[idx] = cn;
    P.p.x1[idx] = new_x1;
    nx1 = 1.0f - new_x1;
    alpha = G.alpha[cn] * new_x1 + G.alpha[cn - 1] * nx1;
    D1 = G.D1[cn] * new_x1 + G.D1[cn - 1] * nx1;
    D2 = G.D2[cn] * new_x1 + G.D2[cn - 1] * nx1;
    D3 = G.D3[cn] * new_x1 + G.D3[cn - 1] * nx1;
    u0 = sqrtf((D2 + p1 * p1) / (D2 * (alpha * alpha - D3) + D1 * D1));
    P.p.E[idx] = u0;
    // deposit (:266-293): J1 through K1_j, Rho through K1, every step
    if (!(flag & kFlagIgnoreCurrent)) {
      const float weight = -P.charge[sp] * P.p.w[idx];
      const int i0 = (dc1 == -1 ? -2 : -1), i1 = (dc1 == 1 ? 1 : 0);
      const bool rho = sp < ns;
      float djx = 0.0f;
#pragma unroll
      for (int j = 0; j < 3; ++j) {  // the 2 or 3 nodes i0 .. i1, in order
        const int i = i0 + j;
        if (i > i1) continue;
        const float sx0 = cic(-x1 + i + 1);
        const float sx1 = cic(-new_x1 + (i + 1 - dc1));
        djx += sx1 - sx0;
        const int o = i + (int)c;
        const float a1 = weight * djx / G.K1_j[o + 1] * delta / dt;
        const float rr = -weight * sx1 / G.K1[o];
        if (use_smem) {
          win_add(sWhi, sWlo, o + 1 - wlo, a1, fscale, L);
          if (rho) win_add(sWhi, sWlo, (1 + sp) * win_comp + o - wlo, rr, fscale, L);
        } else {
          atomicAdd(P.acc + o + 1, (unsigned long long)__float2ll_rn(a1 * fscale));
          if (rho)
            atomicAdd(P.acc + (3 + sp) * P.acc_comp + o,
                      (unsigned long long)__float2ll_rn(rr * fscale));
        }
      }
    }
  }
  __syncthreads();
  if (use_smem) {
    for (int i = tid; i < ncomp * wlen; i += kGrThreads) {
      const int comp = i / wlen, o = i % wlen;
      const int si = comp * win_comp + o;
      const long long v = (long long)sWhi[si] * (1ll << L) + (long long)sWlo[si];
      if (v == 0) continue;
      const int gx = wlo + o;
      if (gx < 0 || gx >= n0) continue;
      const int gcomp = comp == 0 ? 0 : 2 + comp;  // J1, then Rho[sp] at 3 + sp
      atomicAdd(P.acc + gcomp * P.acc_comp + gx, (unsigned long long)v);
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kGrThreads)
    k_gr_push_deposit(const __grid_constant__ PushDepositParams P, const __grid_constant__ GrK G) {
  __shared__ int sWhi[kGrWin];
  __shared__ unsigned sWlo[kGrWin];
  __shared__ int s_lo, s_hi;
  const size_t nchunks = (P.number + kGrChunk - 1) / kGrChunk;
  for (size_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x)
    gr_chunk(P, G, ch, sWhi, sWlo, s_lo, s_hi);
}

// filter_current1d of the GR lab (ptc_updater_1dgr.cu:388-404): cells
// [0, n), each neighbour weighted by k1, the sum divided by k1 of the cell;
// the reference reads one element past each end of the row, which counts
// as 0 here.
__global__ void k_gr_filter(const float *__restrict__ src, float *__restrict__ dst,
                            const float *__restrict__ k1, int n, int g, int bnd_lower,
                            int bnd_upper) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int dp = (bnd_upper && i == n - g - 1) ? 0 : 1;
    const int dm = (bnd_lower && i == g) ? 0 : 1;
    const int ip = i + dp, im = i - dm;
    const float jp = ip < n ? src[ip] : 0.0f, kp = ip < n ? k1[ip] : 0.0f;
    const float jm = im >= 0 ? src[im] : 0.0f, km = im >= 0 ? k1[im] : 0.0f;
    float t = 0.5f * src[i] * k1[i];
    t += 0.25f * jp * kp;
    t += 0.25f * jm * km;
    t /= k1[i];
    dst[i] = t;
  }
}

// update_e_1dgr (field_solver_1dgr.cu:14-24).
__global__ void k_gr_update_e(float *__restrict__ e1, const float *__restrict__ j1,
                              const float *__restrict__ j0, int n, int g, float dt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x + g + 1; i < n - g - 5;
       i += gridDim.x * blockDim.x)
    e1[i] += (j0[i] - j1[i]) * dt;
}

int grid_for_cells(const Ctx &c, size_t n, int block) {
  size_t g = (n + block - 1) / block;
  const size_t cap = (size_t)c.num_sms * 8;
  if (g > cap) g = cap;
  return g < 1 ? 1 : (int)g;
}

float sqf(float x) { return x * x; }
double sqd(double x) { return x * x; }

}  // namespace

// Grid_1dGR::compute_coef (grid_1dgr.cpp:21-187), host side: the metric
// coefficients of each cell from the tabulated field-line data the
// reference reads from coef.h5. Every expression keeps the reference's
// float / double types (a, omega and B0 are floats; double literals promote).
void host_gr_coef(const ap_mesh &m, const ap_gr_params &gp, const ap_gr_table &t,
                  std::vector<float> *co) {
  const int n_size = m.dims[0];
  for (int k = 0; k < AP_GR_NCOEF; ++k) co[k].assign((size_t)n_size, 0.0f);
  const float a = gp.a, omega = gp.omega, B0 = gp.B0;
  const float *v_r = t.r;
  size_t n_data = 0, n_mid = 0;
  for (int n = 0; n < n_size; ++n) {
    const double xi = m.lower[0] + (float)(n - m.guard[0] + 1) * m.delta[0];
    const double rp = 1.0 + std::sqrt(1.0 - a * a);
    const double rm = 1.0 - std::sqrt(1.0 - a * a);
    const double exp_xi = std::exp(xi * (rp - rm));
    const double r = (rp - rm * exp_xi) / (1.0 - exp_xi);
    while (n_data + 2 < t.n && v_r[n_data + 1] < r) n_data += 1;
    const double x = (r - v_r[n_data]) / (float)(v_r[n_data + 1] - v_r[n_data]);
    const float B1 = t.B1[n_data] * (1.0 - x) + t.B1[n_data + 1] * x;
    const float B3 = t.B3[n_data] * (1.0 - x) + t.B3[n_data + 1] * x;
    const float theta = t.theta[n_data] * (1.0 - x) + t.theta[n_data + 1] * x;
    const float b31 = B3 / B1;
    co[AP_GR_B3B1][n] = b31;
    co[AP_GR_RHO0][n] = B0 * (t.rho[n_data] * (1.0 - x) + t.rho[n_data + 1] * x);
    float Sigma = r * r + (float)(a * a * sqf(std::cos(theta)));
    float Delta = r * r - 2.0 * r + a * a;
    float A = sqd(r * r + a * a) - (float)(Delta * a * a * sqf(std::sin(theta)));
    const float w = 2.0 * a * r / A;
    float g11 = Sigma / Delta;
    float g22 = Sigma;
    float g33 = A * sqf(std::sin(theta)) / Sigma;
    float sqrt_gamma = std::sqrt(g11 * g22 * g33);
    co[AP_GR_K1][n] =
        (Delta * sqrt_gamma) / (t.dpsidth[n_data] * (1.0 - x) + t.dpsidth[n_data + 1] * x);
    co[AP_GR_D1][n] = (b31 * g33 * (omega - w)) * Delta;
    co[AP_GR_D2][n] = (g11 + b31 * b31 * g33) * Delta * Delta;
    co[AP_GR_D3][n] = g33 * sqf(omega - w);
    co[AP_GR_ALPHA][n] = std::sqrt(Delta * Sigma / A);
    co[AP_GR_GAMMA_RR][n] = 1.0 / g11;
    co[AP_GR_GAMMA_FF][n] = 1.0 / g33;
    co[AP_GR_BETA_PHI][n] = -2.0 * a * r / A;
    // cell-face quantities; the interpolation weight y uses r, as the
    // reference does
    const double xi_mid = m.lower[0] + ((n - m.guard[0]) + 0.5) * m.delta[0];
    const double exp_xi_mid = std::exp(xi_mid * (rp - rm));
    const double r_mid = (rp - rm * exp_xi_mid) / (1.0 - exp_xi_mid);
    while (n_mid + 2 < t.n && v_r[n_mid + 1] < r_mid) n_mid += 1;
    const double y = (r - v_r[n_mid]) / (float)(v_r[n_mid + 1] - v_r[n_mid]);
    co[AP_GR_J0][n] = B0 * (t.jr[n_mid] * (1.0 - y) + t.jr[n_mid + 1] * y) / Delta;
    const float theta_mid = t.theta[n_mid] * (1.0 - y) + t.theta[n_mid + 1] * y;
    Sigma = r_mid * r_mid + (float)(a * a * sqf(std::cos(theta_mid)));
    Delta = r_mid * r_mid - 2.0 * r_mid + a * a;
    A = sqd(r_mid * r_mid + a * a) - (float)(Delta * a * a * sqf(std::sin(theta_mid)));
    g11 = Sigma / Delta;
    g22 = Sigma;
    g33 = A * sqf(std::sin(theta_mid)) / Sigma;
    sqrt_gamma = std::sqrt(g11 * g22 * g33);
    co[AP_GR_K1_J][n] =
        (Delta * sqrt_gamma) / (t.dpsidth[n_mid] * (1.0 - y) + t.dpsidth[n_mid + 1] * y);
    co[AP_GR_AGRR][n] = Delta * Delta * std::sqrt(Delta * Sigma / A) * g11;
  }
}

cudaError_t launch_gr_push_deposit(Ctx &c, const PushDepositParams &P, const GrK &G) {
  const size_t nchunks = (P.number + kGrChunk - 1) / kGrChunk;
  if (nchunks == 0) return cudaSuccess;
  const int grid = (int)(nchunks < (size_t)c.num_sms * 8 ? nchunks : (size_t)c.num_sms * 8);
  k_gr_push_deposit<<<grid, kGrThreads, 0, c.stream>>>(P, G);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_gr_filter(Ctx &c, const float *src, float *dst, const float *k1,
                             int bnd_lower, int bnd_upper) {
  const int n = c.mesh.dims[0];
  k_gr_filter<<<grid_for_cells(c, n, 256), 256, 0, c.stream>>>(src, dst, k1, n, c.mesh.guard[0],
                                                               bnd_lower, bnd_upper);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_gr_update_e(Ctx &c, const float *j0, float dt) {
  const int n = c.mesh.dims[0];
  k_gr_update_e<<<grid_for_cells(c, n, 256), 256, 0, c.stream>>>(
      static_cast<float *>(c.fields.E[0].ptr), static_cast<const float *>(c.fields.J[0].ptr), j0,
      n, c.mesh.guard[0], dt);
  c.launches++;
  return cudaGetLastError();
}

}  // namespace apb

// 1D gap lab path (src/cuda/algorithms/ptc_updater_1dgap.cu,
// field_solver_1dgap.cu): the radial-gap pusher with beta_phi(x) = x, its
// current / charge deposit (J1 scaled by delta / dt, Rho every step), the
// 1-2-1 filter of that lab over whole rows, and the E1 update
// E1 += (j0 - J1) dt.
//
// The push keeps the reference's float / double mix operation by operation
// (the library is built with -fmad=false and IEEE float division and square
// root; double arithmetic is IEEE), so particles match an FP32/FP64 CPU
// evaluation of the reference bit for bit. The deposit accumulates exact
// fixed-point sums in a shared-memory window over the chunk's cells, as
// the Cartesian 1D kernel does.
#include <cuda_runtime.h>
#include <stdint.h>

#include <climits>

#include "ap_device.cuh"
#include "ap_internal.h"

namespace apb {

namespace {

constexpr int kGapThreads = 256;
constexpr int kGapItems = 8;
constexpr int kGapChunk = kGapThreads * kGapItems;  // 2048 particle slots
constexpr int kGapWin = 6000;                       // cell-components per window

__device__ __forceinline__ int bits_of_u32(uint32_t v) { return 32 - __clz(v | 1u); }

struct GapAcc {
  int *hi;
  unsigned *lo;
};

__device__ __forceinline__ void gap_add(const GapAcc &a, int o, float v, float scale, int L) {
  const long long X = __float2ll_rn(v * scale);  // exact scaling by a power of two
  atomicAdd(a.hi + o, (int)(X >> L));
  atomicAdd(a.lo + o, (unsigned)X & ((1u << L) - 1u));
}

// One chunk of slots: update_ptc_1dgap (ptc_updater_1dgap.cu:75-161) per
// live particle. Window components: 0 = J1, 1 + sp = Rho[sp].
__device__ void gap_chunk(const PushDepositParams &P, size_t ch, int *sWhi, unsigned *sWlo,
                          int &s_lo, int &s_hi) {
  const int tid = threadIdx.x;
  const int n0 = P.m.dims[0], g0 = P.m.guard[0];
  const int ns = P.num_species;
  const int ncomp = 1 + ns;
  const int win_comp = kGapWin / ncomp;
  // scale: a window sums at most kGapChunk contributions per cell, the
  // global accumulators at most `number`
  const int lgw = bits_of_u32(kGapChunk);
  const int lgn = bits_of_u32((uint32_t)min(P.number, (size_t)0x7fffffff));
  int B = min(63 - 2 * lgw, 62 - lgn);
  const float qw = P.qmax * *P.wmax;
  int S = B - 2;
  if (qw > 0.0f) S -= ilogbf(qw);
  S = max(-100, min(100, S));
  const int L = 32 - lgw;
  const float fscale = ldexpf(1.0f, S);
  if (ch == 0 && tid == 0) *P.fx_used = FixedFmt{S, L};
  const size_t first = ch * kGapChunk;
  if (tid == 0) {
    s_lo = INT_MAX;
    s_hi = INT_MIN;
  }
  __syncthreads();
  uint32_t cells[kGapItems];
  int lo = INT_MAX, hi = INT_MIN;
#pragma unroll
  for (int k = 0; k < kGapItems; ++k) {
    const size_t idx = first + (size_t)k * kGapThreads + tid;
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
    for (int i = tid; i < ncomp * win_comp; i += kGapThreads) {
      sWhi[i] = 0;
      sWlo[i] = 0u;
    }
  __syncthreads();

  const float *E3 = P.F[2].ptr;
  const float lower = P.m.lower[0], delta = P.m.delta[0];
#pragma unroll 1
  for (int k = 0; k < kGapItems; ++k) {
    const size_t idx = first + (size_t)k * kGapThreads + tid;
    const uint32_t c = cells[k];
    if (c == AP_MAX_CELL) continue;
    if ((int)c < g0 || (int)c >= n0 - g0) {  // is_in_bulk
      P.p.cell[idx] = AP_MAX_CELL;
      continue;
    }
    float p1 = P.p.p1[idx];
    const float x1 = P.p.x1[idx];
    float gamma = P.p.E[idx];
    const uint32_t flag = P.p.flag[idx];
    const int sp = ptc_type(flag);
    float beta = mesh_pos(lower, delta, (int)c, g0, x1);  // beta_phi(x) = x
    const float Dr = (x1 < 0.5f ? E3[c] * (0.5f + x1) + E3[c - 1] * (0.5f - x1)
                                : E3[c] * (1.5f - x1) + E3[c + 1] * (x1 - 0.5f));
    const float E_term = Dr * P.charge[sp] / P.mass[sp] * P.dt;
    p1 += E_term;
    const double sgn = beta < 0.0f ? -1.0 : 1.0;
    const double f = ((double)gamma - sgn * (double)p1) / (1.0 + (double)(beta * beta));
    p1 = (float)((double)p1 + (double)(beta / gamma) * f * f * (double)P.dt);
    P.p.p1[idx] = p1;
    gamma = sqrtf(1.0f + p1 * p1 + beta * beta);
    float vr = (float)((sgn * (double)p1 / (double)gamma + (double)(beta * beta)) /
                       (1.0 + (double)(beta * beta)));
    if (beta < 0.0f) vr *= -1.0f;
    float new_x1 = x1 + vr * P.dt * P.m.inv_delta[0];
    const int dc1 = (int)floorf(new_x1);
    // the reference reports a move of more than one cell and goes on
    if (dc1 > 1 || dc1 < -1) atomicAdd(&P.status->moved_far, 1ull);
    new_x1 -= (float)dc1;
    P.p.cell[idx] = (uint32_t)((int)c + dc1);
    P.p.x1[idx] = new_x1;
    beta = mesh_pos(lower, delta, (int)c + dc1, g0, new_x1);
    gamma = sqrtf(1.0f + p1 * p1 + beta * beta);
    P.p.E[idx] = gamma;
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
        const float a1 = weight * djx * delta / P.dt;
        const float r = -weight * sx1;
        const int o = i + (int)c;
        if (use_smem) {
          const GapAcc W{sWhi, sWlo};
          gap_add(W, o + 1 - wlo, a1, fscale, L);
          if (rho) gap_add(W, (1 + sp) * win_comp + o - wlo, r, fscale, L);
        } else {
          atomicAdd(P.acc + o + 1, (unsigned long long)__float2ll_rn(a1 * fscale));
          if (rho)
            atomicAdd(P.acc + (3 + sp) * P.acc_comp + o,
                      (unsigned long long)__float2ll_rn(r * fscale));
        }
      }
    }
  }
  __syncthreads();
  if (use_smem) {
    for (int i = tid; i < ncomp * wlen; i += kGapThreads) {
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

__global__ void __launch_bounds__(kGapThreads) k_gap_push_deposit(const __grid_constant__ PushDepositParams P) {
  __shared__ int sWhi[kGapWin];
  __shared__ unsigned sWlo[kGapWin];
  __shared__ int s_lo, s_hi;
  const size_t nchunks = (P.number + kGapChunk - 1) / kGapChunk;
  for (size_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x)
    gap_chunk(P, ch, sWhi, sWlo, s_lo, s_hi);
}

// filter_current1d (ptc_updater_1dgap.cu:196-213) over cells [0, n): the
// reference reads one element past each end of the row, which counts as 0.
__global__ void k_gap_filter(const float *__restrict__ src, float *__restrict__ dst, int n, int g,
                             int bnd_lower, int bnd_upper) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int dp = (bnd_upper && i == n - g - 1) ? 0 : 1;
    const int dm = (bnd_lower && i == g) ? 0 : 1;
    const float jp = (i + dp < n) ? src[i + dp] : 0.0f;
    const float jm = (i - dm >= 0) ? src[i - dm] : 0.0f;
    float t = 0.5f * src[i];
    t += 0.25f * jp;
    t += 0.25f * jm;
    dst[i] = t;
  }
}

// update_e_1dgap (field_solver_1dgap.cu:14-24).
__global__ void k_gap_update_e(float *__restrict__ e1, const float *__restrict__ j1, int n, int g,
                               float j0, float dt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x + g + 1; i < n - g - 1;
       i += gridDim.x * blockDim.x)
    e1[i] += (j0 - j1[i]) * dt;
}

int grid_1d(const Ctx &c, size_t n, int block) {
  size_t g = (n + block - 1) / block;
  const size_t cap = (size_t)c.num_sms * 8;
  if (g > cap) g = cap;
  return g < 1 ? 1 : (int)g;
}

}  // namespace

cudaError_t launch_gap_push_deposit(Ctx &c, const PushDepositParams &P) {
  const size_t nchunks = (P.number + kGapChunk - 1) / kGapChunk;
  if (nchunks == 0) return cudaSuccess;
  const int grid = (int)(nchunks < (size_t)c.num_sms * 8 ? nchunks : (size_t)c.num_sms * 8);
  k_gap_push_deposit<<<grid, kGapThreads, 0, c.stream>>>(P);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_gap_filter(Ctx &c, const float *src, float *dst, int bnd_lower,
                              int bnd_upper) {
  const int n = c.mesh.dims[0];
  k_gap_filter<<<grid_1d(c, n, 256), 256, 0, c.stream>>>(src, dst, n, c.mesh.guard[0],
                                                         bnd_lower, bnd_upper);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_gap_update_e(Ctx &c, float j0, float dt) {
  const int n = c.mesh.dims[0];
  k_gap_update_e<<<grid_1d(c, n, 256), 256, 0, c.stream>>>(
      static_cast<float *>(c.fields.E[0].ptr), static_cast<const float *>(c.fields.J[0].ptr), n,
      c.mesh.guard[0], j0, dt);
  c.launches++;
  return cudaGetLastError();
}

}  // namespace apb

// FP64 diagnostics of the particle update, reduced on the device.
// The reference has only per-particle gamma (cuda/core/particles.cu:10-22)
// and EdotB averages; these reductions are new. Values are accumulated in
// double in registers, per block in shared memory, and across blocks with
// double atomics; maxima of non-negative doubles use the integer order of
// their bit patterns.
#include <cuda_runtime.h>

#include "ap_device.cuh"
#include "ap_internal.h"

namespace apb {

namespace {

constexpr int kDiagThreads = 256;

__device__ __forceinline__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += sh[w];
  return r;
}

__device__ __forceinline__ double block_max(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, sh[w]);
  return r;
}

__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long *>(addr),
            (unsigned long long)__double_as_longlong(v));
}

struct DiagParams {
  PtcK p;
  size_t number;
  double mass[AP_MAX_SPECIES];
  double charge[AP_MAX_SPECIES];
  int n0, n1, g0, g1, dim, num_species;
  double cell_volume;
  FieldArr E[3], B[3], J[3], Rho[AP_MAX_SPECIES], divE;
  double *out;  // kinetic, charge, field energy, max|rho|, max|divE - rho|, max|J|
};

__global__ void __launch_bounds__(kDiagThreads) k_diag_particles(const DiagParams P) {
  __shared__ double sh[kDiagThreads / 32];
  double kin = 0.0, q = 0.0;
  auto add = [&](uint32_t cell, uint32_t flag, double p1, double p2, double p3, double w) {
    if (cell == AP_MAX_CELL) return;
    const int sp = ptc_type(flag);
    const double pp = p1 * p1 + p2 * p2 + p3 * p3;
    const double gm1 = pp / (sqrt(1.0 + pp) + 1.0);  // gamma - 1 without cancellation
    kin += w * P.mass[sp] * gm1;
    q += w * P.charge[sp];
  };
  // four particles' loads in flight per thread (a streaming read)
  constexpr int U = 4;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  for (; i + (U - 1) * stride < P.number; i += U * stride) {
    uint32_t c[U], f[U];
    float p1[U], p2[U], p3[U], w[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const size_t k = i + u * stride;
      c[u] = P.p.cell[k];
      f[u] = P.p.flag[k];
      p1[u] = P.p.p1[k];
      p2[u] = P.p.p2[k];
      p3[u] = P.p.p3[k];
      w[u] = P.p.w[k];
    }
#pragma unroll
    for (int u = 0; u < U; ++u) add(c[u], f[u], p1[u], p2[u], p3[u], w[u]);
  }
  for (; i < P.number; i += stride)
    add(P.p.cell[i], P.p.flag[i], P.p.p1[i], P.p.p2[i], P.p.p3[i], P.p.w[i]);
  const double sk = block_sum(kin, sh);
  const double sq = block_sum(q, sh);
  if (threadIdx.x == 0) {
    atomicAdd(P.out + 0, sk);
    atomicAdd(P.out + 1, sq);
  }
}

__global__ void __launch_bounds__(kDiagThreads) k_diag_fields(const DiagParams P) {
  __shared__ double sh[kDiagThreads / 32];
  const int r0 = P.n0 - 2 * P.g0;
  const int r1 = P.dim > 1 ? P.n1 - 2 * P.g1 : 1;
  const int g1 = P.dim > 1 ? P.g1 : 0;
  const size_t total = (size_t)r0 * r1;
  double en = 0.0, mrho = 0.0, mres = 0.0, mj = 0.0;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    int i, j;
    split_index(t, r0, i, j);
    i += P.g0;
    j += g1;
    double s = 0.0;
    for (int k = 0; k < 3; ++k) {
      const double e = P.E[k].ptr[(size_t)j * P.E[k].pitch + i];
      const double b = P.B[k].ptr[(size_t)j * P.B[k].pitch + i];
      s += e * e + b * b;
      mj = fmax(mj, fabs((double)P.J[k].ptr[(size_t)j * P.J[k].pitch + i]));
    }
    en += 0.5 * s * P.cell_volume;
    double rho = 0.0;
    for (int sp = 0; sp < P.num_species; ++sp)
      rho += P.Rho[sp].ptr[(size_t)j * P.Rho[sp].pitch + i];
    mrho = fmax(mrho, fabs(rho));
    if (P.divE.ptr) mres = fmax(mres, fabs((double)P.divE.ptr[(size_t)j * P.divE.pitch + i] - rho));
  }
  const double se = block_sum(en, sh);
  const double a = block_max(mrho, sh);
  const double b = block_max(mres, sh);
  const double cj = block_max(mj, sh);
  if (threadIdx.x == 0) {
    atomicAdd(P.out + 2, se);
    atomic_max_nonneg(P.out + 3, a);
    atomic_max_nonneg(P.out + 4, b);
    atomic_max_nonneg(P.out + 5, cj);
  }
}

struct ContParams {
  FieldArr Rho[AP_MAX_SPECIES], J1, J2;
  double *prev;
  int n0, n1, g0, g1, dim, num_species, per0, per1;
  double *out;
};

__global__ void __launch_bounds__(kDiagThreads) k_rho_snapshot(const ContParams P) {
  const size_t total = (size_t)P.n0 * P.n1;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    int i, j;
    split_index(t, P.n0, i, j);
    double rho = 0.0;
    for (int sp = 0; sp < P.num_species; ++sp)
      rho += P.Rho[sp].ptr[(size_t)j * P.Rho[sp].pitch + i];
    P.prev[t] = rho;
  }
}

// Discrete continuity of the Esirkepov deposit: J1 at index i + 1 is the
// flux through the upper x face of cell i (ptc_updater.cu:364-371), J2 at
// j + 1 through the upper y face; the face past the last bulk cell of a
// periodic side is the first bulk face (the guard cells keep the raw
// deposit).
__global__ void __launch_bounds__(kDiagThreads) k_continuity(const ContParams P) {
  __shared__ double sh[kDiagThreads / 32];
  const int r0 = P.n0 - 2 * P.g0;
  const int r1 = P.dim > 1 ? P.n1 - 2 * P.g1 : 1;
  const int g1 = P.dim > 1 ? P.g1 : 0;
  const size_t total = (size_t)r0 * r1;
  double mres = 0.0;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    int i, j;
    split_index(t, r0, i, j);
    i += P.g0;
    j += g1;
    double rho = 0.0;
    for (int sp = 0; sp < P.num_species; ++sp)
      rho += P.Rho[sp].ptr[(size_t)j * P.Rho[sp].pitch + i];
    const int ip = (i + 1 == P.n0 - P.g0 && P.per0) ? P.g0 : i + 1;
    double div = (double)P.J1.ptr[(size_t)j * P.J1.pitch + ip] -
                 (double)P.J1.ptr[(size_t)j * P.J1.pitch + i];
    if (P.dim > 1) {
      const int jp = (j + 1 == P.n1 - P.g1 && P.per1) ? P.g1 : j + 1;
      div += (double)P.J2.ptr[(size_t)jp * P.J2.pitch + i] -
             (double)P.J2.ptr[(size_t)j * P.J2.pitch + i];
    }
    mres = fmax(mres, fabs(rho - P.prev[(size_t)j * P.n0 + i] + div));
  }
  const double m = block_max(mres, sh);
  if (threadIdx.x == 0) atomic_max_nonneg(P.out, m);
}

ContParams cont_params(const Ctx &c) {
  ContParams P;
  auto fa = [](const ap_array &a) { return FieldArr{a.ptr, (int)(a.pitch / 4)}; };
  for (int s = 0; s < c.params.num_species; ++s) P.Rho[s] = fa(c.fields.Rho[s]);
  P.J1 = fa(c.fields.J[0]);
  P.J2 = fa(c.fields.J[1]);
  P.prev = c.rho_prev;
  P.n0 = c.mesh.dims[0];
  P.n1 = c.mk.dim > 1 ? c.mesh.dims[1] : 1;
  P.g0 = c.mesh.guard[0];
  P.g1 = c.mesh.guard[1];
  P.dim = c.mk.dim;
  P.num_species = c.params.num_species;
  P.per0 = c.params.periodic[0];
  P.per1 = c.params.periodic[1];
  P.out = nullptr;
  return P;
}

}  // namespace

cudaError_t launch_rho_snapshot(Ctx &c) {
  const ContParams P = cont_params(c);
  k_rho_snapshot<<<c.num_sms * 4, kDiagThreads, 0, c.stream>>>(P);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_continuity(Ctx &c, double *out) {
  ContParams P = cont_params(c);
  P.out = out;
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), c.stream);
  if (e != cudaSuccess) return e;
  k_continuity<<<c.num_sms * 4, kDiagThreads, 0, c.stream>>>(P);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_diagnostics(Ctx &c, double *out) {
  DiagParams P;
  // the occupied slots [store_base, number)
  const size_t b = c.store_base;
  P.p = PtcK{c.ptc.x1 + b, c.ptc.x2 + b, c.ptc.x3 + b, c.ptc.p1 + b,     c.ptc.p2 + b,
             c.ptc.p3 + b, c.ptc.E + b,  c.ptc.weight + b, c.ptc.cell + b, c.ptc.flag + b};
  P.number = c.number - b;
  for (int s = 0; s < AP_MAX_SPECIES; ++s) {
    P.mass[s] = c.params.masses[s];
    P.charge[s] = c.params.charges[s];
  }
  P.n0 = c.mesh.dims[0];
  P.n1 = c.mesh.dims[1];
  P.g0 = c.mesh.guard[0];
  P.g1 = c.mesh.guard[1];
  P.dim = c.mk.dim;
  P.num_species = c.params.num_species;
  P.cell_volume = (double)c.mesh.delta[0] * (c.mk.dim > 1 ? (double)c.mesh.delta[1] : 1.0);
  auto fa = [](const ap_array &a) { return FieldArr{a.ptr, (int)(a.pitch / 4)}; };
  for (int k = 0; k < 3; ++k) {
    P.E[k] = fa(c.fields.E[k]);
    P.B[k] = fa(c.fields.B[k]);
    P.J[k] = fa(c.fields.J[k]);
  }
  for (int s = 0; s < c.params.num_species; ++s) P.Rho[s] = fa(c.fields.Rho[s]);
  P.divE = c.fields.divE.ptr ? fa(c.fields.divE) : FieldArr{nullptr, 0};
  P.out = out;
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double) * 6, c.stream);
  if (e != cudaSuccess) return e;
  int grid = c.num_sms * 8;
  if (c.number > 0) {
    k_diag_particles<<<grid, kDiagThreads, 0, c.stream>>>(P);
    c.launches++;
  }
  k_diag_fields<<<grid, kDiagThreads, 0, c.stream>>>(P);
  c.launches++;
  return cudaGetLastError();
}

}  // namespace apb

// Yee FDTD update, divergences, current filter and guard-cell exchange on
// one rank (src/cuda/algorithms/field_solver.cu, ptc_updater.cu:501-560,
// cuda/sim_environment.cpp:9-127).
//
// The reference updates the bulk and then copies interior strips into the
// guard cells with one MPI self-exchange per direction. Here each thread
// that updates a bulk cell near a periodic side also writes that cell's
// periodic images in the guard layers, which leaves every guard cell of a
// periodic dim holding its bulk image -- the state send_guard_cells
// produces -- without a separate pass.
#include <cuda_runtime.h>

#include "ap_device.cuh"
#include "ap_internal.h"

namespace apb {

namespace {

struct Arr {
  float *p;
  int pitch;  // floats
  __device__ __forceinline__ float &operator()(int i, int j) const {
    return p[(size_t)j * pitch + i];
  }
};

__host__ Arr arr(const ap_array &a) { return Arr{a.ptr, (int)(a.pitch / sizeof(float))}; }

struct Geo {
  int n0, n1, g0, g1, r0, r1, per0, per1, dim;
  float id0, id1;
};

// Writes v at (i, j) and at its periodic guard images.
__device__ __forceinline__ void store_with_images(const Arr &a, const Geo &G, int i, int j,
                                                  float v) {
  a(i, j) = v;
  int ix[2] = {i, i}, jx[2] = {j, j};
  int ni = 1, nj = 1;
  if (G.per0) {
    if (i < 2 * G.g0) ix[ni++] = i + G.r0;
    else if (i >= G.n0 - 2 * G.g0) ix[ni++] = i - G.r0;
  }
  if (G.dim > 1 && G.per1) {
    if (j < 2 * G.g1) jx[nj++] = j + G.r1;
    else if (j >= G.n1 - 2 * G.g1) jx[nj++] = j - G.r1;
  }
  for (int b = 0; b < nj; ++b)
    for (int a2 = 0; a2 < ni; ++a2)
      if (a2 || b) a(ix[a2], jx[b]) = v;
}

// compute_e_update2d (field_solver.cu:45-84) / compute_e_update1d (:14-43)
// for bulk cell (n1, n2).
__device__ __forceinline__ void e_update_cell(const Geo &G, const Arr &e1, const Arr &e2,
                                              const Arr &e3, const Arr &b1, const Arr &b2,
                                              const Arr &b3, const Arr &b01, const Arr &b02,
                                              const Arr &b03, const Arr &j1, const Arr &j2,
                                              const Arr &j3, float dt, int n1, int n2) {
  if (G.dim > 1) {
    const float v1 = e1(n1, n2) + dt * ((b3(n1, n2 + 1) - b3(n1, n2) - b03(n1, n2 + 1) +
                                         b03(n1, n2)) * G.id1 - j1(n1, n2));
    const float v2 = e2(n1, n2) + dt * ((b3(n1, n2) - b3(n1 + 1, n2) - b03(n1, n2) +
                                         b03(n1 + 1, n2)) * G.id0 - j2(n1, n2));
    const float v3 =
        e3(n1, n2) + dt * ((b2(n1 + 1, n2) - b2(n1, n2) - b02(n1 + 1, n2) + b02(n1, n2)) *
                               G.id0 +
                           (b1(n1, n2) - b1(n1, n2 + 1) - b01(n1, n2) + b01(n1, n2 + 1)) *
                               G.id1 - j3(n1, n2));
    store_with_images(e1, G, n1, n2, v1);
    store_with_images(e2, G, n1, n2, v2);
    store_with_images(e3, G, n1, n2, v3);
  } else {
    const float v1 = e1(n1, 0) - dt * j1(n1, 0);
    const float v2 = e2(n1, 0) + dt * ((b3(n1, 0) - b3(n1 + 1, 0) - b03(n1, 0) +
                                        b03(n1 + 1, 0)) * G.id0 - j2(n1, 0));
    const float v3 = e3(n1, 0) + dt * ((b2(n1 + 1, 0) - b2(n1, 0) - b02(n1 + 1, 0) +
                                        b02(n1, 0)) * G.id0 - j3(n1, 0));
    store_with_images(e1, G, n1, 0, v1);
    store_with_images(e2, G, n1, 0, v2);
    store_with_images(e3, G, n1, 0, v3);
  }
}

__global__ void k_update_e(Geo G, Arr e1, Arr e2, Arr e3, Arr b1, Arr b2, Arr b3, Arr b01,
                           Arr b02, Arr b03, Arr j1, Arr j2, Arr j3, float dt) {
  const int n1 = G.g0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int n2 = (G.dim > 1 ? G.g1 : 0) + blockIdx.y * blockDim.y + threadIdx.y;
  if (n1 >= G.n0 - G.g0) return;
  if (G.dim > 1 && n2 >= G.n1 - G.g1) return;
  e_update_cell(G, e1, e2, e3, b1, b2, b3, b01, b02, b03, j1, j2, j3, dt, n1, n2);
}

// compute_b_update2d (field_solver.cu:160-193) / compute_b_update1d (:133-158)
// for bulk cell (n1, n2).
__device__ __forceinline__ void b_update_cell(const Geo &G, const Arr &e1, const Arr &e2,
                                              const Arr &e3, const Arr &e01, const Arr &e02,
                                              const Arr &e03, const Arr &b1, const Arr &b2,
                                              const Arr &b3, float dt, int n1, int n2) {
  if (G.dim > 1) {
    const float v1 = b1(n1, n2) - dt * (e3(n1, n2) - e3(n1, n2 - 1) - e03(n1, n2) +
                                        e03(n1, n2 - 1)) * G.id1;
    const float v2 = b2(n1, n2) - dt * (e3(n1 - 1, n2) - e3(n1, n2) - e03(n1 - 1, n2) +
                                        e03(n1, n2)) * G.id0;
    const float v3 =
        b3(n1, n2) - dt * ((e2(n1, n2) - e2(n1 - 1, n2) - e02(n1, n2) + e02(n1 - 1, n2)) *
                               G.id0 +
                           (e1(n1, n2 - 1) - e1(n1, n2) - e01(n1, n2 - 1) + e01(n1, n2)) *
                               G.id1);
    store_with_images(b1, G, n1, n2, v1);
    store_with_images(b2, G, n1, n2, v2);
    store_with_images(b3, G, n1, n2, v3);
  } else {
    // b1 is not updated in 1D; its guards are still refreshed by the
    // reference's exchange, which is a no-op when they already hold images.
    const float v2 = b2(n1, 0) - dt * (e3(n1 - 1, 0) - e3(n1, 0) - e03(n1 - 1, 0) +
                                       e03(n1, 0)) * G.id0;
    const float v3 = b3(n1, 0) - dt * (e2(n1, 0) - e2(n1 - 1, 0) - e02(n1, 0) +
                                       e02(n1 - 1, 0)) * G.id0;
    store_with_images(b1, G, n1, 0, b1(n1, 0));
    store_with_images(b2, G, n1, 0, v2);
    store_with_images(b3, G, n1, 0, v3);
  }
}

__global__ void k_update_b(Geo G, Arr e1, Arr e2, Arr e3, Arr e01, Arr e02, Arr e03, Arr b1,
                           Arr b2, Arr b3, float dt) {
  const int n1 = G.g0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int n2 = (G.dim > 1 ? G.g1 : 0) + blockIdx.y * blockDim.y + threadIdx.y;
  if (n1 >= G.n0 - G.g0) return;
  if (G.dim > 1 && n2 >= G.n1 - G.g1) return;
  b_update_cell(G, e1, e2, e3, e01, e02, e03, b1, b2, b3, dt, n1, n2);
}

// compute_divs_2d (field_solver.cu:261-288) / compute_divs_1d (:237-259) for
// bulk cell (n1, n2).
__device__ __forceinline__ void divs_cell(const Geo &G, const Arr &e1, const Arr &e2,
                                          const Arr &b1, const Arr &b2, const Arr &e01,
                                          const Arr &e02, const Arr &b01, const Arr &b02,
                                          const Arr &divE, const Arr &divB, int n1, int n2) {
  if (G.dim > 1) {
    divE(n1, n2) = (e1(n1 + 1, n2) - e01(n1 + 1, n2) - e1(n1, n2) + e01(n1, n2)) * G.id0 +
                   (e2(n1, n2 + 1) - e02(n1, n2 + 1) - e2(n1, n2) + e02(n1, n2)) * G.id1;
    divB(n1, n2) = (b1(n1, n2) - b01(n1, n2) - b1(n1 - 1, n2) + b01(n1 - 1, n2)) * G.id0 +
                   (b2(n1, n2) - b02(n1, n2) - b2(n1, n2 - 1) + b02(n1, n2 - 1)) * G.id1;
  } else {
    divE(n1, 0) = (e1(n1 + 1, 0) - e01(n1 + 1, 0) - e1(n1, 0) + e01(n1, 0)) * G.id0;
    divB(n1, 0) = (b1(n1, 0) - b01(n1, 0) - b1(n1 - 1, 0) + b01(n1 - 1, 0)) * G.id0;
  }
}

__global__ void k_divs(Geo G, Arr e1, Arr e2, Arr b1, Arr b2, Arr e01, Arr e02, Arr b01,
                       Arr b02, Arr divE, Arr divB) {
  const int n1 = G.g0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int n2 = (G.dim > 1 ? G.g1 : 0) + blockIdx.y * blockDim.y + threadIdx.y;
  if (n1 >= G.n0 - G.g0) return;
  if (G.dim > 1 && n2 >= G.n1 - G.g1) return;
  divs_cell(G, e1, e2, b1, b2, e01, e02, b01, b02, divE, divB, n1, n2);
}

// Guard strips of one dim: mode 0 copies interior strips into the opposite
// guards (send_array_guard_cells_single_dir), mode 1 adds guard strips into
// the opposite interior (send_add_array_guard_cells_single_dir). Both
// directions are handled in one launch; their strips are disjoint.
__global__ void k_guard_strips(Arr a, int n0, int n1, int g, int dim, int mode) {
  const int len = dim == 0 ? n1 : n0;  // extent along the other dim
  const int total = 2 * g * len;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int dir = t / (g * len);  // 0: dir -1, 1: dir +1
    const int rem = t % (g * len);
    const int layer = rem / len, o = rem % len;
    const int n = dim == 0 ? n0 : n1;
    int src, dst;
    if (mode == 0) {
      src = dir == 0 ? g + layer : n - 2 * g + layer;
      dst = dir == 0 ? n - g + layer : layer;
    } else {
      src = dir == 0 ? layer : n - g + layer;
      dst = dir == 0 ? n - 2 * g + layer : g + layer;
    }
    if (dim == 0) {
      if (mode == 0) a(dst, o) = a(src, o);
      else a(dst, o) += a(src, o);
    } else {
      if (mode == 0) a(o, dst) = a(o, src);
      else a(o, dst) += a(o, src);
    }
  }
}

// filter_current_cart_2d / _1d (ptc_updater.cu:501-560): bulk only.
__global__ void k_filter(Geo G, Arr j, Arr t, int bl0, int bu0, int bl1, int bu1) {
  const int a = G.g0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int b = (G.dim > 1 ? G.g1 : 0) + blockIdx.y * blockDim.y + threadIdx.y;
  if (a >= G.n0 - G.g0) return;
  const int xp = (bu0 && a == G.n0 - G.g0 - 1) ? 0 : 1;
  const int xm = (bl0 && a == G.g0) ? 0 : 1;
  if (G.dim > 1) {
    if (b >= G.n1 - G.g1) return;
    const int yp = (bu1 && b == G.n1 - G.g1 - 1) ? 0 : 1;
    const int ym = (bl1 && b == G.g1) ? 0 : 1;
    float v = 0.25f * j(a, b);
    v += 0.125f * j(a + xp, b);
    v += 0.125f * j(a - xm, b);
    v += 0.125f * j(a, b + yp);
    v += 0.125f * j(a, b - ym);
    v += 0.0625f * j(a + xp, b + yp);
    v += 0.0625f * j(a - xm, b + yp);
    v += 0.0625f * j(a + xp, b - ym);
    v += 0.0625f * j(a - xm, b - ym);
    t(a, b) = v;
  } else {
    float v = 0.5f * j(a, 0);
    v += 0.25f * j(a + xp, 0);
    v += 0.25f * j(a - xm, 0);
    t(a, 0) = v;
  }
}

__global__ void k_copy_bulk(Geo G, Arr src, Arr dst) {
  const int a = G.g0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int b = (G.dim > 1 ? G.g1 : 0) + blockIdx.y * blockDim.y + threadIdx.y;
  if (a >= G.n0 - G.g0) return;
  if (G.dim > 1 && b >= G.n1 - G.g1) return;
  dst(a, b) = src(a, b);
}

// Folds the periodic guard layers of the fixed-point accumulators into the
// bulk and rounds once to FP32. For one rank, send_add_guard_cells
// (cuda/sim_environment.cpp:71-127) adds the lower guard strip of a dim into
// the upper interior strip and the upper guard strip into the lower interior
// strip, dim 0 (all rows) before dim 1 (all columns), leaving the guard
// values in place; per cell that is the gather below. The integer sums are
// exact, so the order of the adds does not matter; the only rounding is the
// final conversion (int64 -> double is exact below 2^53, then one rounding
// to FP32).
__device__ __forceinline__ void finalize_cell(const Geo &G, const unsigned long long *a,
                                              int acc_pitch, double inv, const Arr &out, int x,
                                              int y) {
  int xi = -1, yi = -1;
  if (G.per0) {
    if (x >= G.g0 && x < 2 * G.g0) xi = x + G.r0;
    else if (x >= G.n0 - 2 * G.g0 && x < G.n0 - G.g0) xi = x - G.r0;
  }
  if (G.dim > 1 && G.per1) {
    if (y >= G.g1 && y < 2 * G.g1) yi = y + G.r1;
    else if (y >= G.n1 - 2 * G.g1 && y < G.n1 - G.g1) yi = y - G.r1;
  }
  unsigned long long v = a[(size_t)y * acc_pitch + x];
  if (xi >= 0) v += a[(size_t)y * acc_pitch + xi];
  if (yi >= 0) {
    v += a[(size_t)yi * acc_pitch + x];
    if (xi >= 0) v += a[(size_t)yi * acc_pitch + xi];
  }
  out(x, y) = (float)((double)(long long)v * inv);
}

__global__ void k_finalize(Geo G, const unsigned long long *__restrict__ acc, int acc_pitch,
                           size_t acc_comp, const FixedFmt *fmt, int ncomp, Arr o0, Arr o1,
                           Arr o2, Arr o3, Arr o4, Arr o5, Arr o6, Arr o7, Arr o8, Arr o9,
                           Arr o10) {
  const int rows = G.dim > 1 ? G.n1 : 1;
  const size_t total = (size_t)G.n0 * rows;
  const int comp = blockIdx.y;
  if (comp >= ncomp) return;
  Arr outs[11] = {o0, o1, o2, o3, o4, o5, o6, o7, o8, o9, o10};
  const Arr out = outs[comp];
  const unsigned long long *a = acc + comp * acc_comp;
  const double inv = ldexp(1.0, -fmt->S);
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    int x, y;
    split_index(t, G.n0, x, y);
    finalize_cell(G, a, acc_pitch, inv, out, x, y);
  }
}

Geo make_geo(const Ctx &c) {
  const ap_mesh &m = c.mesh;
  Geo G;
  G.n0 = m.dims[0];
  G.n1 = m.dims[1];
  G.g0 = m.guard[0];
  G.g1 = m.guard[1];
  G.r0 = m.dims[0] - 2 * m.guard[0];
  G.r1 = m.dims[1] - 2 * m.guard[1];
  G.per0 = c.params.periodic[0];
  G.per1 = c.params.periodic[1];
  G.dim = c.mk.dim;
  G.id0 = m.inv_delta[0];
  G.id1 = m.inv_delta[1];
  return G;
}

void bulk_launch_shape(const Geo &G, dim3 &grid, dim3 &block) {
  if (G.dim > 1) {
    block = dim3(32, 8);
    grid = dim3((G.r0 + 31) / 32, (G.r1 + 7) / 8);
  } else {
    block = dim3(256, 1);
    grid = dim3((G.r0 + 255) / 256, 1);
  }
}

}  // namespace

namespace {

// ---------------------------------------------------------------------------
// Batched 1D launches: work item g belongs to run r with base[r] <= g <
// base[r + 1]; the per-cell arithmetic is the single-run kernels'.

__device__ __forceinline__ int run_of(const uint32_t *base, int nruns, uint32_t g) {
  int lo = 0, hi = nruns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (base[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ Arr farr(const FieldArr &a) { return Arr{a.ptr, a.pitch}; }

__device__ __forceinline__ Geo geo1(const Run1D &R) {
  Geo G;
  G.n0 = R.n0;
  G.n1 = 1;
  G.g0 = R.g0;
  G.g1 = 0;
  G.r0 = R.r0;
  G.r1 = 0;
  G.per0 = R.per0;
  G.per1 = 0;
  G.dim = 1;
  G.id0 = R.id0;
  G.id1 = 0.0f;
  return G;
}

__global__ void k_b1_zero(const Run1D *__restrict__ runs, const uint32_t *__restrict__ base,
                          int nruns) {
  const uint32_t total = base[nruns];
  for (uint32_t g = blockIdx.x; g < total; g += gridDim.x) {
    const int r = run_of(base, nruns, g);
    const Run1D &R = runs[r];
    const size_t w = (size_t)(g - base[r]) * 256 + threadIdx.x;
    if (w < (size_t)R.zero_comps * R.acc_comp) R.acc[w] = 0ull;
  }
}

__global__ void k_b1_finalize(const Run1D *__restrict__ runs, const uint32_t *__restrict__ base,
                              int nruns) {
  const uint32_t total = base[nruns];
  for (uint32_t g = blockIdx.x; g < total; g += gridDim.x) {
    const int r = run_of(base, nruns, g);
    const Run1D &R = runs[r];
    const int x = (int)(g - base[r]) * 256 + threadIdx.x;
    if (x >= R.n0) continue;
    const Geo G = geo1(R);
    const double inv = ldexp(1.0, -R.fx->S);
    for (int comp = 0; comp < R.ncomp; ++comp) {
      const Arr out = farr(comp < 3 ? R.J[comp] : R.Rho[comp - 3]);
      finalize_cell(G, R.acc + comp * R.acc_comp, R.n0, inv, out, x, 0);
    }
  }
}

__global__ void k_b1_fields(const Run1D *__restrict__ runs, const uint32_t *__restrict__ base,
                            int nruns, int which) {
  const uint32_t total = base[nruns];
  for (uint32_t g = blockIdx.x; g < total; g += gridDim.x) {
    const int r = run_of(base, nruns, g);
    const Run1D &R = runs[r];
    const int n1 = R.g0 + (int)(g - base[r]) * 256 + threadIdx.x;
    if (n1 >= R.n0 - R.g0) continue;
    const Geo G = geo1(R);
    if (which == 0 || which == 2) {
      const float dt = which == 0 ? R.dt_half : R.dt;
      if (which == 0 && !(dt > 0.0f)) continue;
      e_update_cell(G, farr(R.E[0]), farr(R.E[1]), farr(R.E[2]), farr(R.B[0]), farr(R.B[1]),
                    farr(R.B[2]), farr(R.Bb[0]), farr(R.Bb[1]), farr(R.Bb[2]), farr(R.J[0]),
                    farr(R.J[1]), farr(R.J[2]), dt, n1, 0);
    } else if (which == 1) {
      b_update_cell(G, farr(R.E[0]), farr(R.E[1]), farr(R.E[2]), farr(R.Eb[0]), farr(R.Eb[1]),
                    farr(R.Eb[2]), farr(R.B[0]), farr(R.B[1]), farr(R.B[2]), R.dt, n1, 0);
    } else if (R.has_divs) {
      divs_cell(G, farr(R.E[0]), farr(R.E[1]), farr(R.B[0]), farr(R.B[1]), farr(R.Eb[0]),
                farr(R.Eb[1]), farr(R.Bb[0]), farr(R.Bb[1]), farr(R.divE), farr(R.divB), n1, 0);
    }
  }
}

uint32_t grid_of(uint32_t total, int num_sms) {
  const uint32_t cap = (uint32_t)num_sms * 16;
  return total < cap ? total : cap;
}

}  // namespace

cudaError_t launch_b1_zero(cudaStream_t s, int num_sms, const Run1D *runs, const uint32_t *base,
                           int nruns, uint32_t total) {
  if (total == 0) return cudaSuccess;
  k_b1_zero<<<grid_of(total, num_sms), 256, 0, s>>>(runs, base, nruns);
  return cudaGetLastError();
}

cudaError_t launch_b1_finalize(cudaStream_t s, int num_sms, const Run1D *runs,
                               const uint32_t *base, int nruns, uint32_t total) {
  if (total == 0) return cudaSuccess;
  k_b1_finalize<<<grid_of(total, num_sms), 256, 0, s>>>(runs, base, nruns);
  return cudaGetLastError();
}

cudaError_t launch_b1_fields(cudaStream_t s, int num_sms, const Run1D *runs, const uint32_t *base,
                             int nruns, uint32_t total, int which) {
  if (total == 0) return cudaSuccess;
  k_b1_fields<<<grid_of(total, num_sms), 256, 0, s>>>(runs, base, nruns, which);
  return cudaGetLastError();
}

cudaError_t launch_update_e(Ctx &c, float dt) {
  const ap_fields &f = c.fields;
  Geo G = make_geo(c);
  dim3 grid, block;
  bulk_launch_shape(G, grid, block);
  k_update_e<<<grid, block, 0, c.stream>>>(G, arr(f.E[0]), arr(f.E[1]), arr(f.E[2]),
                                           arr(f.B[0]), arr(f.B[1]), arr(f.B[2]),
                                           arr(f.Bbg[0]), arr(f.Bbg[1]), arr(f.Bbg[2]),
                                           arr(f.J[0]), arr(f.J[1]), arr(f.J[2]), dt);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_update_b(Ctx &c, float dt) {
  const ap_fields &f = c.fields;
  Geo G = make_geo(c);
  dim3 grid, block;
  bulk_launch_shape(G, grid, block);
  k_update_b<<<grid, block, 0, c.stream>>>(G, arr(f.E[0]), arr(f.E[1]), arr(f.E[2]),
                                           arr(f.Ebg[0]), arr(f.Ebg[1]), arr(f.Ebg[2]),
                                           arr(f.B[0]), arr(f.B[1]), arr(f.B[2]), dt);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_divs(Ctx &c) {
  const ap_fields &f = c.fields;
  if (!f.divE.ptr || !f.divB.ptr) return cudaSuccess;
  Geo G = make_geo(c);
  dim3 grid, block;
  bulk_launch_shape(G, grid, block);
  k_divs<<<grid, block, 0, c.stream>>>(G, arr(f.E[0]), arr(f.E[1]), arr(f.B[0]), arr(f.B[1]),
                                       arr(f.Ebg[0]), arr(f.Ebg[1]), arr(f.Bbg[0]),
                                       arr(f.Bbg[1]), arr(f.divE), arr(f.divB));
  c.launches++;
  return cudaGetLastError();
}

static cudaError_t guard_pass(Ctx &c, ap_array a, int mode) {
  const ap_mesh &m = c.mesh;
  const int nd = c.mk.dim;
  for (int d = 0; d < nd && d < 2; ++d) {
    if (!c.params.periodic[d]) continue;
    const int len = d == 0 ? m.dims[1] : m.dims[0];
    const int total = 2 * m.guard[d] * len;
    int grid = (total + 255) / 256;
    if (grid > 1024) grid = 1024;
    k_guard_strips<<<grid, 256, 0, c.stream>>>(arr(a), m.dims[0], m.dims[1], m.guard[d], d, mode);
    c.launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_copy_guards(Ctx &c, ap_array a) { return guard_pass(c, a, 0); }
cudaError_t launch_fold_guards(Ctx &c, ap_array a) { return guard_pass(c, a, 1); }

cudaError_t launch_filter(Ctx &c, ap_array a, int bnd[4]) {
  Geo G = make_geo(c);
  dim3 grid, block;
  bulk_launch_shape(G, grid, block);
  Arr t{c.tmp_j, c.tmp_pitch};
  k_filter<<<grid, block, 0, c.stream>>>(G, arr(a), t, bnd[0], bnd[1], bnd[2], bnd[3]);
  c.launches++;
  k_copy_bulk<<<grid, block, 0, c.stream>>>(G, t, arr(a));
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_finalize_current(Ctx &c, int ncomp) {
  Geo G = make_geo(c);
  Arr o[11];
  for (int k = 0; k < 11; ++k) o[k] = Arr{nullptr, 0};
  for (int k = 0; k < 3; ++k) o[k] = arr(c.fields.J[k]);
  for (int s = 0; s < c.params.num_species && 3 + s < 11; ++s) o[3 + s] = arr(c.fields.Rho[s]);
  const size_t total = (size_t)G.n0 * (G.dim > 1 ? G.n1 : 1);
  int gx = (int)((total + 255) / 256);
  if (gx > c.num_sms * 8) gx = c.num_sms * 8;
  dim3 grid(gx, ncomp);
  k_finalize<<<grid, 256, 0, c.stream>>>(G, c.acc, c.mesh.dims[0], c.acc_comp, c.fx_used, ncomp,
                                         o[0], o[1],
                                         o[2], o[3], o[4], o[5], o[6], o[7], o[8], o[9], o[10]);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_zero(Ctx &c, ap_array a) {
  const ap_mesh &m = c.mesh;
  return cudaMemset2DAsync(a.ptr, a.pitch, 0, sizeof(float) * m.dims[0],
                           (size_t)m.dims[1] * m.dims[2], c.stream);
}

}  // namespace apb

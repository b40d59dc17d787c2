// Log-spherical (ln r, theta) grid: coefficients, current post-processing
// and the integral-form Yee solver.
//
// Replaces Grid_LogSph::compute_coef (src/grids/grid_log_sph.cpp:11-126),
// process_j / axis_rho_* / filter_current_logsph
// (src/cuda/algorithms/ptc_updater_logsph.cu:284-299, 414-438, 616-666) and
// field_solver_logsph (src/cuda/algorithms/field_solver_logsph.cu:16-428).
// The particle push and move run in the fused 2D kernel of
// k_push_deposit.cu (its kLS variant).
//
// The coefficients are host code in the reference too; they are evaluated
// here with the same float / double mixture (Scalar arguments and results,
// double intermediates where the reference's literals make them double),
// so they equal the reference's bit for bit, and are uploaded once.
// The field kernels keep the reference's expression order; they are
// bandwidth-bound stencils (one thread per bulk cell, rows coalesced).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "ap_device.cuh"
#include "ap_internal.h"

namespace apb {

namespace {

constexpr double kPi = 3.14159265358979323846;

// Quadmesh::pos on the host (float arithmetic, quadmesh.h:144-150).
float hpos(const ap_mesh &m, int i, int n, float x) {
  return m.lower[i] + m.delta[i] * ((float)(n - m.guard[i]) + x);
}

// Grid_LogSph::alpha / l1 / A2 / V3 (grid_log_sph.h:23-38): Scalar (float)
// arguments and results, double intermediates.
float h_alpha(float r, float rs) { return (float)std::sqrt(1.0 - (double)(rs / r)); }
float h_l1(float r, float rs) {
  const float a = h_alpha(r, rs);
  return (float)((double)(r * a) +
                 0.5 * (double)rs * std::log(2.0 * (double)r * (1.0 + (double)a) - (double)rs));
}
float h_A2(float r, float rs) {
  const float a = h_alpha(r, rs);
  return (float)(0.25 * (double)r * (double)a * (2.0 * (double)r + 3.0 * (double)rs) +
                 0.375 * (double)rs * (double)rs *
                     std::log(2.0 * (double)r * (1.0 + (double)a) - (double)rs));
}
float h_V3(float r, float rs) {
  const float a = h_alpha(r, rs);
  return (float)((double)(r * a) *
                     (8.0 * (double)r * (double)r + 10.0 * (double)r * (double)rs +
                      15.0 * (double)rs * (double)rs) /
                     24.0 +
                 0.3125 * (double)rs * (double)rs * (double)rs *
                     std::log(2.0 * (double)r * (1.0 + (double)a) - (double)rs));
}

// compute_coef with r_g = 0 (grid_log_sph.cpp:14). out[k] is row-major
// dims[0] x dims[1].
void host_coef(const ap_mesh &m, std::vector<float> *out) {
  const float r_g = 0.0f;
  const int n0 = m.dims[0], n1 = m.dims[1];
  const double d0 = (double)m.delta[0], d1 = (double)m.delta[1];
  const double d01 = (double)(m.delta[0] * m.delta[1]);
  for (int k = 0; k < AP_NUM_COEF; ++k) out[k].assign((size_t)n0 * n1, 0.0f);
  for (int j = 0; j < n1; ++j) {
    const double x2 = (double)hpos(m, 1, j, 0.5f);
    const double x2s = (double)hpos(m, 1, j, 1.0f);
    for (int i = 0; i < n0; ++i) {
      const double x1 = (double)hpos(m, 0, i, 0.5f);
      const double x1s = (double)hpos(m, 0, i, 1.0f);
      const double r_plus = std::exp(x1 + d0);
      const double r = std::exp(x1);
      const double rs = std::exp(x1s);
      const double rs_minus = std::exp(x1s - d0);
      const size_t o = (size_t)i + (size_t)j * n0;
      out[AP_COEF_L1E][o] = h_l1((float)rs, r_g) - h_l1((float)rs_minus, r_g);
      out[AP_COEF_L2E][o] = (float)(rs * d1);
      out[AP_COEF_L3E][o] = (float)(rs * std::sin(x2s));
      out[AP_COEF_L1B][o] = h_l1((float)r_plus, r_g) - h_l1((float)r, r_g);
      out[AP_COEF_L2B][o] = (float)(r * d1);
      out[AP_COEF_L3B][o] = (float)(r * std::sin(x2));
      out[AP_COEF_A1E][o] = (float)(r * r * (std::cos(x2) - std::cos(x2 + d1)));
      if (std::fabs(x2s) < 1.0e-5)
        out[AP_COEF_A1E][o] = (float)(r * r * 2.0 * (1.0 - std::cos(0.5 * d1)));
      else if (std::fabs(x2s - kPi) < 1.0e-5)
        out[AP_COEF_A1E][o] = (float)(r * r * 2.0 * (1.0 - std::cos(0.5 * d1)));
      const float a2e = h_A2((float)r_plus, r_g) - h_A2((float)r, r_g);
      out[AP_COEF_A2E][o] = (float)((double)a2e * std::sin(x2));
      out[AP_COEF_A3E][o] = (float)((double)a2e * d1);
      out[AP_COEF_A1B][o] = (float)(rs * rs * (std::cos(x2s - d1) - std::cos(x2s)));
      const float a2b = h_A2((float)rs, r_g) - h_A2((float)rs_minus, r_g);
      out[AP_COEF_A2B][o] = (float)((double)a2b * std::sin(x2s));
      out[AP_COEF_A3B][o] = (float)((double)a2b * d1);
      const float v3 = h_V3((float)r_plus, r_g) - h_V3((float)r, r_g);
      out[AP_COEF_DV][o] = (float)((double)v3 * (std::cos(x2) - std::cos(x2 + d1)) / d01);
      if (std::fabs(x2s) < 1.0e-5 || std::fabs(x2s - kPi) < 1.0e-5)
        out[AP_COEF_DV][o] = (float)((double)v3 * 2.0 * (1.0 - std::cos(0.5 * d1)) / d01);
    }
  }
}

// Grid constants of the log-spherical kernels.
struct LsGeo {
  int n0, n1, g0, g1;
  float lower0, lower1, d0, d1, size1;
  float compactness, omega;
};

struct Arr {
  float *p;
  int pitch;  // floats
  __device__ __forceinline__ float &operator()(int i, int j) const {
    return p[(size_t)j * pitch + i];
  }
};

Arr arr(const ap_array &a) { return Arr{a.ptr, (int)(a.pitch / sizeof(float))}; }

struct LsFields {
  Arr E1, E2, E3, B1, B2, B3, Eb1, Eb2, Eb3, Bb1, Bb2, Bb3, J1, J2, J3, divE, divB;
};

struct LsCoef {
  Arr c[AP_NUM_COEF];
};

__device__ __forceinline__ float pos0(const LsGeo &G, int n, float x) {
  return mesh_pos(G.lower0, G.d0, n, G.g0, x);
}
__device__ __forceinline__ float pos1(const LsGeo &G, int n, float x) {
  return mesh_pos(G.lower1, G.d1, n, G.g1, x);
}
__device__ __forceinline__ float alpha_gr(float) { return 1.0f; }

// compute_b_update_logsph (field_solver_logsph.cu:117-185). Every input is
// loaded into a register before the first division or transcendental: the
// slow paths of those sit behind branches, and global loads written inside
// the expressions are not moved above a branch, so they would go out in
// several dependent rounds. The expressions are the reference's, in its
// order; the new values are stored once all three are computed.
__global__ void k_ls_update_b(LsGeo G, LsFields F, LsCoef K, float dt) {
  const int n1 = G.g0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int n2 = G.g1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (n1 >= G.n0 - G.g0 || n2 >= G.n1 - G.g1) return;
  const Arr &l1e = K.c[AP_COEF_L1E], &l2e = K.c[AP_COEF_L2E], &l3e = K.c[AP_COEF_L3E];
  const Arr &A1b = K.c[AP_COEF_A1B], &A2b = K.c[AP_COEF_A2B], &A3b = K.c[AP_COEF_A3B];
  const float b1 = F.B1(n1, n2), b2 = F.B2(n1, n2), b3 = F.B3(n1, n2);
  const float e1 = F.E1(n1, n2), eb1 = F.Eb1(n1, n2);
  const float e1_jm = F.E1(n1, n2 - 1), eb1_jm = F.Eb1(n1, n2 - 1);
  const float e2 = F.E2(n1, n2), eb2 = F.Eb2(n1, n2);
  const float e2_im = F.E2(n1 - 1, n2), eb2_im = F.Eb2(n1 - 1, n2);
  const float e3 = F.E3(n1, n2), eb3 = F.Eb3(n1, n2);
  const float e3_jm = F.E3(n1, n2 - 1), eb3_jm = F.Eb3(n1, n2 - 1);
  const float e3_im = F.E3(n1 - 1, n2), eb3_im = F.Eb3(n1 - 1, n2);
  const float bb1 = F.Bb1(n1, n2), bb1_im = F.Bb1(n1 - 1, n2);
  const float bb2 = F.Bb2(n1, n2), bb2_jm = F.Bb2(n1, n2 - 1);
  const float l1 = l1e(n1, n2), l1_jm = l1e(n1, n2 - 1);
  const float l2 = l2e(n1, n2), l2_im = l2e(n1 - 1, n2);
  const float l3 = l3e(n1, n2), l3_jm = l3e(n1, n2 - 1), l3_im = l3e(n1 - 1, n2);
  const float a1 = A1b(n1, n2), a2 = A2b(n1, n2), a3 = A3b(n1, n2);
  const float r1 = expf(pos0(G, n1, 1.0f));
  const float r0 = expf(pos0(G, n1 - 1, 1.0f));
  const float r = expf(pos0(G, n1, 0.5f));
  const float v1 = b1 + -dt *
                            ((e3 - eb3) * alpha_gr(r1) * l3 -
                             (e3_jm - eb3_jm) * alpha_gr(r1) * l3_jm) /
                            a1;
  const float v2 = b2 + -dt *
                            ((e3_im - eb3_im) * alpha_gr(r0) * l3_im -
                             (e3 - eb3) * alpha_gr(r1) * l3) /
                            a2;
  const float v3 =
      b3 + -dt * ((((e2 - eb2) * alpha_gr(r1) +
                    bb1 * beta_phi(G.compactness, G.omega, r1, pos1(G, n2, 0.5f))) *
                       l2 -
                   ((e2_im - eb2_im) * alpha_gr(r0) +
                    bb1_im * beta_phi(G.compactness, G.omega, r0, pos1(G, n2, 0.5f))) *
                       l2_im +
                   ((e1_jm - eb1_jm) * alpha_gr(r) -
                    bb2_jm * beta_phi(G.compactness, G.omega, r, pos1(G, n2 - 1, 1.0f))) *
                       l1_jm -
                   ((e1 - eb1) * alpha_gr(r) -
                    bb2 * beta_phi(G.compactness, G.omega, r, pos1(G, n2, 1.0f))) *
                       l1) /
                  a3);
  F.B1(n1, n2) = v1;
  F.B2(n1, n2) = v2;
  F.B3(n1, n2) = v3;
  // axis at theta = 0: written by the threads of the first bulk row; no
  // thread of this kernel reads B
  if (fabsf(pos1(G, n2, 1.0f) - G.d1) < 1.0e-5) {
    const int a = G.g1 - 1;
    F.B2(n1, a) = F.Bb2(n1, a);
  }
}

// compute_e_update_logsph (field_solver_logsph.cu:29-114), with the inputs
// loaded first as in k_ls_update_b (both branches' inputs of E1).
__global__ void k_ls_update_e(LsGeo G, LsFields F, LsCoef K, float dt) {
  const int n1 = G.g0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int n2 = G.g1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (n1 >= G.n0 - G.g0 || n2 >= G.n1 - G.g1) return;
  const Arr &l1b = K.c[AP_COEF_L1B], &l2b = K.c[AP_COEF_L2B], &l3b = K.c[AP_COEF_L3B];
  const Arr &A1e = K.c[AP_COEF_A1E], &A2e = K.c[AP_COEF_A2E], &A3e = K.c[AP_COEF_A3E];
  const float e1 = F.E1(n1, n2), e2 = F.E2(n1, n2), e3 = F.E3(n1, n2);
  const float j1 = F.J1(n1, n2), j2 = F.J2(n1, n2), j3 = F.J3(n1, n2);
  const float b1 = F.B1(n1, n2), bb1 = F.Bb1(n1, n2);
  const float b1_jp = F.B1(n1, n2 + 1), bb1_jp = F.Bb1(n1, n2 + 1);
  const float b2 = F.B2(n1, n2), bb2 = F.Bb2(n1, n2);
  const float b2_ip = F.B2(n1 + 1, n2), bb2_ip = F.Bb2(n1 + 1, n2);
  const float b3 = F.B3(n1, n2), bb3 = F.Bb3(n1, n2);
  const float b3_jp = F.B3(n1, n2 + 1), bb3_jp = F.Bb3(n1, n2 + 1);
  const float b3_ip = F.B3(n1 + 1, n2), bb3_ip = F.Bb3(n1 + 1, n2);
  const float l1 = l1b(n1, n2), l1_jp = l1b(n1, n2 + 1);
  const float l2 = l2b(n1, n2), l2_ip = l2b(n1 + 1, n2);
  const float l3 = l3b(n1, n2), l3_jp = l3b(n1, n2 + 1), l3_ip = l3b(n1 + 1, n2);
  const float a1 = A1e(n1, n2), a2 = A2e(n1, n2), a3 = A3e(n1, n2);
  const float r = expf(pos0(G, n1, 1.0f));
  const float r1 = expf(pos0(G, n1 + 1, 0.5f));
  const float r0 = expf(pos0(G, n1, 0.5f));
  float v1;
  if (fabs((double)pos1(G, n2, 1.0f) - kPi) < 1.0e-5) {
    v1 = e1 + dt * (-4.0f * (b3 - bb3) * alpha_gr(r0) / (G.d1 * r0) - j1);
  } else {
    v1 = e1 + dt * (((b3_jp - bb3_jp) * alpha_gr(r0) * l3_jp - (b3 - bb3) * alpha_gr(r0) * l3) /
                        a1 -
                    j1);
  }
  const float v2 =
      e2 + dt * (((b3 - bb3) * alpha_gr(r0) * l3 - (b3_ip - bb3_ip) * alpha_gr(r1) * l3_ip) /
                     a2 -
                 j2);
  const float v3 = e3 + dt * (((b2_ip - bb2_ip) * alpha_gr(r1) * l2_ip -
                               (b2 - bb2) * alpha_gr(r0) * l2 +
                               (b1 - bb1) * alpha_gr(r) * l1 -
                               (b1_jp - bb1_jp) * alpha_gr(r) * l1_jp) /
                                  a3 -
                              j3);
  F.E1(n1, n2) = v1;
  F.E2(n1, n2) = v2;
  F.E3(n1, n2) = v3;
  // axis at theta = 0; these cells are read by no thread of this kernel
  if (fabsf(pos1(G, n2, 1.0f) - G.d1) < 1.0e-5) {
    const int a = G.g1 - 1;
    F.E3(n1, a) = F.Eb3(n1, a);
    F.E1(n1, a) += dt * (4.0f * (F.B3(n1, a + 1) - F.Bb3(n1, a + 1)) * alpha_gr(r0) /
                             (G.d1 * r0) -
                         F.J1(n1, a));
  }
}

// compute_divs_logsph (field_solver_logsph.cu:188-250), with the inputs
// loaded first as in k_ls_update_b.
__global__ void k_ls_divs(LsGeo G, LsFields F, LsCoef K) {
  const int n1 = G.g0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int n2 = G.g1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (n1 >= G.n0 - G.g0 || n2 >= G.n1 - G.g1) return;
  const Arr &A1e = K.c[AP_COEF_A1E], &A2e = K.c[AP_COEF_A2E];
  const Arr &A1b = K.c[AP_COEF_A1B], &A2b = K.c[AP_COEF_A2B], &dV = K.c[AP_COEF_DV];
  const float e1 = F.E1(n1, n2), eb1 = F.Eb1(n1, n2);
  const float e1_ip = F.E1(n1 + 1, n2), eb1_ip = F.Eb1(n1 + 1, n2);
  const float e2 = F.E2(n1, n2), eb2 = F.Eb2(n1, n2);
  const float e2_jp = F.E2(n1, n2 + 1), eb2_jp = F.Eb2(n1, n2 + 1);
  const float b1 = F.B1(n1, n2), bb1 = F.Bb1(n1, n2);
  const float b1_im = F.B1(n1 - 1, n2), bb1_im = F.Bb1(n1 - 1, n2);
  const float b2 = F.B2(n1, n2), bb2 = F.Bb2(n1, n2);
  const float b2_jm = F.B2(n1, n2 - 1), bb2_jm = F.Bb2(n1, n2 - 1);
  const float a1e = A1e(n1, n2), a1e_ip = A1e(n1 + 1, n2);
  const float a2e = A2e(n1, n2), a2e_jp = A2e(n1, n2 + 1);
  const float a1b = A1b(n1, n2), a1b_im = A1b(n1 - 1, n2);
  const float a2b = A2b(n1, n2), a2b_jm = A2b(n1, n2 - 1);
  const float dv = dV(n1, n2);
  const bool has_e = pos0(G, n1, 1.0f) > G.d0;
  float de = 0.0f;
  if (has_e) {
    if (fabsf(pos1(G, n2, 1.0f) - G.size1 + G.lower1) < 1.0e-5) {
      de = (float)(((double)((e1_ip - eb1_ip) * a1e_ip - (e1 - eb1) * a1e) -
                    2.0 * (double)(e2 - eb2) * (double)a2e) /
                   (double)(dv * G.d0 * G.d1));
    } else {
      de = ((e1_ip - eb1_ip) * a1e_ip - (e1 - eb1) * a1e + (e2_jp - eb2_jp) * a2e_jp -
            (e2 - eb2) * a2e) /
           (dv * G.d0 * G.d1);
    }
  }
  const float db =
      ((b1 - bb1) * a1b - (b1_im - bb1_im) * a1b_im + (b2 - bb2) * a2b - (b2_jm - bb2_jm) * a2b_jm) /
      (dv * G.d0 * G.d1);
  if (has_e) F.divE(n1, n2) = de;
  F.divB(n1, n2) = db;
  // the reference tests |pos| - delta here (not |pos - delta|)
  if (fabsf(pos1(G, n2, 1.0f)) - G.d1 < 1.0e-5) {
    const int a = G.g1 - 1;
    F.divE(n1, a) = ((F.E1(n1 + 1, a) - F.Eb1(n1 + 1, a)) * A1e(n1 + 1, a) -
                     (F.E1(n1, a) - F.Eb1(n1, a)) * A1e(n1, a) +
                     2.0f * (F.E2(n1, a + 1) - F.Eb2(n1, a + 1)) * A2e(n1, a + 1)) /
                    (dV(n1, a) * G.d0 * G.d1);
  }
}

// stellar_boundary then outflow_boundary_sph (field_solver_logsph.cu:
// 252-275, 322-345), one thread per theta row: each touches only its row.
__global__ void k_ls_bnd_radial(LsGeo G, LsFields F, float omega, int damping_length,
                                float damping_coef) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= G.n1) return;
  const float theta_s = pos1(G, j, 1.0f);
  const float theta = pos1(G, j, 0.5f);
  for (int i = 0; i < G.g0; ++i) {
    const float r_s = expf(pos0(G, i, 1.0f));
    const float r = expf(pos0(G, i, 0.5f));
    const float omega_LT = 0.4f * omega * G.compactness;
    F.B1(i, j) = F.Bb1(i, j);
    F.B3(i, j) = F.Bb3(i, j);
    F.E2(i, j) = -(omega - omega_LT) * sinf(theta) * F.Bb1(i, j) / alpha_gr(r_s) / r_s / r_s +
                 F.Eb2(i, j);
    F.E1(i, j) = (omega - omega_LT) * sinf(theta_s) * F.Bb2(i, j) / alpha_gr(r_s) / r / r +
                 F.Eb1(i, j);
    F.B2(i, j) = F.Bb2(i, j);
    F.B3(i, j) = F.Bb3(i, j);
  }
  for (int i = 0; i < damping_length; ++i) {
    const int n1 = G.n0 - damping_length + i;
    const float q = (float)i / (float)damping_length;
    const float lambda = 1.0f - damping_coef * (q * q);
    F.E1(n1, j) = lambda * (F.E1(n1, j) - F.Eb1(n1, j)) + F.Eb1(n1, j);
    F.E2(n1, j) = lambda * (F.E2(n1, j) - F.Eb2(n1, j)) + F.Eb2(n1, j);
    F.E3(n1, j) = lambda * (F.E3(n1, j) - F.Eb3(n1, j)) + F.Eb3(n1, j);
    F.B3(n1, j) = lambda * (F.B3(n1, j) - F.Bb3(n1, j)) + F.Bb3(n1, j);
  }
}

// The same two boundaries with one thread per cell of the two bands of each
// theta row: columns [0, g0) (stellar) and the last damping_length columns
// (outflow). Every assignment of either loop reads and writes only its own
// cell (and the background fields), so the cells are independent as long as
// the bands do not overlap (n0 - damping_length >= g0, checked by the
// launch). Consecutive threads take consecutive columns of a row, so a warp
// reads and writes contiguous memory instead of 32 rows a pitch apart.
__global__ void k_ls_bnd_radial_cells(LsGeo G, LsFields F, float omega, int damping_length,
                                      float damping_coef) {
  const int w = G.g0 + damping_length;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= w * G.n1) return;
  const int j = t / w, k = t - j * w;
  if (k < G.g0) {
    const int i = k;
    const float theta_s = pos1(G, j, 1.0f);
    const float theta = pos1(G, j, 0.5f);
    const float r_s = expf(pos0(G, i, 1.0f));
    const float r = expf(pos0(G, i, 0.5f));
    const float omega_LT = 0.4f * omega * G.compactness;
    F.B1(i, j) = F.Bb1(i, j);
    F.E2(i, j) = -(omega - omega_LT) * sinf(theta) * F.Bb1(i, j) / alpha_gr(r_s) / r_s / r_s +
                 F.Eb2(i, j);
    F.E1(i, j) = (omega - omega_LT) * sinf(theta_s) * F.Bb2(i, j) / alpha_gr(r_s) / r / r +
                 F.Eb1(i, j);
    F.B2(i, j) = F.Bb2(i, j);
    F.B3(i, j) = F.Bb3(i, j);
  } else {
    const int i = k - G.g0;
    const int n1 = G.n0 - damping_length + i;
    const float q = (float)i / (float)damping_length;
    const float lambda = 1.0f - damping_coef * (q * q);
    F.E1(n1, j) = lambda * (F.E1(n1, j) - F.Eb1(n1, j)) + F.Eb1(n1, j);
    F.E2(n1, j) = lambda * (F.E2(n1, j) - F.Eb2(n1, j)) + F.Eb2(n1, j);
    F.E3(n1, j) = lambda * (F.E3(n1, j) - F.Eb3(n1, j)) + F.Eb3(n1, j);
    F.B3(n1, j) = lambda * (F.B3(n1, j) - F.Bb3(n1, j)) + F.Bb3(n1, j);
  }
}

// axis_boundary_lower then axis_boundary_upper (field_solver_logsph.cu:
// 277-320), one thread per r column.
__global__ void k_ls_bnd_axis(LsGeo G, LsFields F) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= G.n0) return;
  const int g = G.g1;
  F.E3(i, g - 1) = F.Eb3(i, g - 1);
  F.E2(i, g - 1) = -(F.E2(i, g) - F.Eb2(i, g)) + F.Eb2(i, g - 1);
  F.B3(i, g - 1) = F.Bb3(i, g - 1);
  F.B3(i, g) = F.Bb3(i, g);
  F.B2(i, g - 1) = F.Bb2(i, g - 1);
  F.B1(i, g - 1) = (F.B1(i, g) - F.Bb1(i, g)) + F.Bb1(i, g - 1);
  const int jl = G.n1 - g;
  F.E3(i, jl - 1) = F.Eb3(i, jl - 1);
  F.E2(i, jl) = -(F.E2(i, jl - 1) - F.Eb2(i, jl - 1)) + F.Eb2(i, jl);
  F.B3(i, jl) = F.Bb3(i, jl);
  F.B3(i, jl - 1) = F.Bb3(i, jl - 1);
  F.B2(i, jl - 1) = F.Bb2(i, jl - 1);
  F.B1(i, jl) = (F.B1(i, jl - 1) - F.Bb1(i, jl - 1)) + F.Bb1(i, jl);
}

// Rounding of the exact current / charge sums to FP32 fused with process_j
// (ptc_updater_logsph.cu:284-299) and, when no smoothing follows,
// axis_rho_lower / upper (:414-438). Component blockIdx.y: J1, J2, J3,
// Rho[0..nsp). Every cell, guards included, as process_j does; Rho of a
// step without charge deposition is 0 / dV.
struct LsOut {
  Arr a[3 + AP_MAX_SPECIES];
};

constexpr int kFinU = 4;  // cells per thread and loop pass, loads issued together

__global__ void k_ls_finalize(LsGeo G, const unsigned long long *__restrict__ acc,
                              size_t acc_comp, const FixedFmt *fmt, int ncomp, int do_rho,
                              int zero_axis, float w, LsOut out, Arr A1e, Arr A2e, Arr dV) {
  const int comp = blockIdx.y;
  if (comp >= ncomp) return;
  const Arr o = out.a[comp];
  const unsigned long long *a = acc + comp * acc_comp;
  const double inv = ldexp(1.0, -fmt->S);
  const bool summed = comp < 3 || do_rho;
  const Arr cA = comp == 0 ? A1e : comp == 1 ? A2e : dV;  // unused for J3
  const bool has_coef = comp != 2;
  const size_t total = (size_t)G.n0 * G.n1;
  const int jl = G.n1 - G.g1;
  const size_t stride = (size_t)gridDim.x * blockDim.x * kFinU;
  for (size_t t0 = (size_t)blockIdx.x * blockDim.x * kFinU + threadIdx.x; t0 < total;
       t0 += stride) {
    long long raw[kFinU];
    float cf[kFinU];
    int xs[kFinU], ys[kFinU];
#pragma unroll
    for (int k = 0; k < kFinU; ++k) {
      const size_t t = t0 + (size_t)k * blockDim.x;
      raw[k] = 0;
      cf[k] = 1.0f;
      xs[k] = ys[k] = 0;
      if (t < total) {
        split_index(t, G.n0, xs[k], ys[k]);
        if (summed) raw[k] = (long long)a[t];
        if (has_coef) cf[k] = cA(xs[k], ys[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < kFinU; ++k) {
      const size_t t = t0 + (size_t)k * blockDim.x;
      if (t >= total) break;
      const int x = xs[k], y = ys[k];
      float v = summed ? (float)((double)raw[k] * inv) : 0.0f;
      if (comp == 0 || comp == 1)
        v *= w / cf[k];
      else if (comp == 2) {
        if (zero_axis && (y == G.g1 - 1 || y == G.g1 || y == jl - 1 || y == jl)) v = 0.0f;
      } else
        v /= cf[k];
      o(x, y) = v;
    }
  }
}

// filter_current_logsph (ptc_updater_logsph.cu:616-666) with all four
// boundaries of a single rank: bulk cells into tmp.
__global__ void k_ls_filter(LsGeo G, Arr j, Arr tmp, Arr A) {
  const int n1 = G.g0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int n2 = G.g1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (n1 >= G.n0 - G.g0 || n2 >= G.n1 - G.g1) return;
  const int xp = (n1 == G.n0 - G.g0 - 1) ? 0 : 1;
  const int xm = (n1 == G.g0) ? 0 : 1;
  const int yp = (n2 == G.n1 - G.g1 - 1) ? 0 : 1;
  const int ym = (n2 == G.g1) ? 0 : 1;
  float t = 0.25f * j(n1, n2) * A(n1, n2);
  t += 0.125f * j(n1 + xp, n2) * A(n1 + xp, n2);
  t += 0.125f * j(n1 - xm, n2) * A(n1 - xm, n2);
  t += 0.125f * j(n1, n2 + yp) * A(n1, n2 + yp);
  t += 0.125f * j(n1, n2 - ym) * A(n1, n2 - ym);
  t += 0.0625f * j(n1 + xp, n2 + yp) * A(n1 + xp, n2 + yp);
  t += 0.0625f * j(n1 - xm, n2 + yp) * A(n1 - xm, n2 + yp);
  t += 0.0625f * j(n1 + xp, n2 - ym) * A(n1 + xp, n2 - ym);
  t += 0.0625f * j(n1 - xm, n2 - ym) * A(n1 - xm, n2 - ym);
  t /= A(n1, n2);
  tmp(n1, n2) = t;
}

__global__ void k_ls_copy_bulk(LsGeo G, Arr dst, Arr src) {
  const int n1 = G.g0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int n2 = G.g1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (n1 >= G.n0 - G.g0 || n2 >= G.n1 - G.g1) return;
  dst(n1, n2) = src(n1, n2);
}

__global__ void k_ls_axis_j3(LsGeo G, Arr J3) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= G.n0) return;
  const int jl = G.n1 - G.g1;
  J3(i, G.g1 - 1) = 0.0f;
  J3(i, G.g1) = 0.0f;
  J3(i, jl) = 0.0f;
  J3(i, jl - 1) = 0.0f;
}

LsGeo make_ls_geo(const Ctx &c) {
  LsGeo G;
  G.n0 = c.mesh.dims[0];
  G.n1 = c.mesh.dims[1];
  G.g0 = c.mesh.guard[0];
  G.g1 = c.mesh.guard[1];
  G.lower0 = c.mesh.lower[0];
  G.lower1 = c.mesh.lower[1];
  G.d0 = c.mesh.delta[0];
  G.d1 = c.mesh.delta[1];
  G.size1 = c.mesh.sizes[1];
  G.compactness = c.lsp.compactness;
  G.omega = c.lsp.omega;
  return G;
}

LsFields make_ls_fields(const Ctx &c) {
  const ap_fields &f = c.fields;
  LsFields F;
  F.E1 = arr(f.E[0]);
  F.E2 = arr(f.E[1]);
  F.E3 = arr(f.E[2]);
  F.B1 = arr(f.B[0]);
  F.B2 = arr(f.B[1]);
  F.B3 = arr(f.B[2]);
  F.Eb1 = arr(f.Ebg[0]);
  F.Eb2 = arr(f.Ebg[1]);
  F.Eb3 = arr(f.Ebg[2]);
  F.Bb1 = arr(f.Bbg[0]);
  F.Bb2 = arr(f.Bbg[1]);
  F.Bb3 = arr(f.Bbg[2]);
  F.J1 = arr(f.J[0]);
  F.J2 = arr(f.J[1]);
  F.J3 = arr(f.J[2]);
  F.divE = arr(f.divE);
  F.divB = arr(f.divB);
  return F;
}

LsCoef make_ls_coef(const Ctx &c) {
  LsCoef K;
  for (int k = 0; k < AP_NUM_COEF; ++k) K.c[k] = arr(coef_array(c, k));
  return K;
}

void bulk_shape(const LsGeo &G, dim3 &grid, dim3 &block) {
  block = dim3(32, 8);
  grid = dim3((G.n0 - 2 * G.g0 + 31) / 32, (G.n1 - 2 * G.g1 + 7) / 8);
}

}  // namespace

ap_array coef_array(const Ctx &c, int which) {
  ap_array a;
  a.ptr = reinterpret_cast<float *>(reinterpret_cast<char *>(c.coef) +
                                    (size_t)which * c.mesh.dims[1] * c.coef_pitch);
  a.pitch = c.coef_pitch;
  return a;
}

int logsph_setup(Ctx &c) {
  const ap_mesh &m = c.mesh;
  std::vector<float> h[AP_NUM_COEF];
  host_coef(m, h);
  size_t pitch = 0;
  if (cudaMallocPitch(reinterpret_cast<void **>(&c.coef), &pitch, sizeof(float) * m.dims[0],
                      (size_t)m.dims[1] * AP_NUM_COEF) != cudaSuccess)
    return AP_ERR_NOMEM;
  c.coef_pitch = pitch;
  float dv_min = INFINITY;
  for (int k = 0; k < AP_NUM_COEF; ++k) {
    ap_array a = coef_array(c, k);
    if (cudaMemcpy2D(a.ptr, a.pitch, h[k].data(), sizeof(float) * m.dims[0],
                     sizeof(float) * m.dims[0], m.dims[1], cudaMemcpyHostToDevice) != cudaSuccess)
      return AP_ERR_CUDA;
  }
  for (float v : h[AP_COEF_DV]) dv_min = fminf(dv_min, fabsf(v));
  // |J3 contribution| <= |q| w |v3_gr| / |dV| with |v3_gr| <= 1 + max|beta_phi|;
  // beta_phi is largest at the smallest radius of the grid.
  const double r_min = std::exp((double)m.lower[0] - (double)m.guard[0] * m.delta[0]);
  const double beta = 0.4 * std::fabs((double)c.lsp.compactness * c.lsp.omega) / (r_min * r_min);
  double k = (1.0 + beta) / (dv_min > 0.0f ? (double)dv_min : 1e-30);
  c.ls_kfac = (float)(k > 1.0 ? k * 1.01 : 1.0);
  return AP_OK;
}

cudaError_t launch_ls_finalize(Ctx &c, float dt, bool do_rho, bool zero_axis) {
  const LsGeo G = make_ls_geo(c);
  const int ncomp = 3 + c.params.num_species;
  LsOut out;
  for (int k = 0; k < 3; ++k) out.a[k] = arr(c.fields.J[k]);
  for (int s = 0; s < c.params.num_species; ++s) out.a[3 + s] = arr(c.fields.Rho[s]);
  // process_j's w = delta[0] * delta[1] / dt, in float
  volatile float d01 = c.mesh.delta[0] * c.mesh.delta[1];
  const float w = d01 / dt;
  const size_t total = (size_t)G.n0 * G.n1;
  int gx = (int)((total + 256 * kFinU - 1) / (256 * kFinU));
  if (gx > c.num_sms * 8) gx = c.num_sms * 8;
  dim3 grid(gx, ncomp);
  k_ls_finalize<<<grid, 256, 0, c.stream>>>(G, c.acc, c.acc_comp, c.fx_used, ncomp,
                                            do_rho ? 1 : 0, zero_axis ? 1 : 0, w, out,
                                            arr(coef_array(c, AP_COEF_A1E)),
                                            arr(coef_array(c, AP_COEF_A2E)),
                                            arr(coef_array(c, AP_COEF_DV)));
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_ls_smooth(Ctx &c, bool do_rho) {
  const LsGeo G = make_ls_geo(c);
  dim3 grid, block;
  bulk_shape(G, grid, block);
  const Arr tmp{c.tmp_j, c.tmp_pitch};
  auto pass = [&](const ap_array &a, int coef) -> cudaError_t {
    k_ls_filter<<<grid, block, 0, c.stream>>>(G, arr(a), tmp, arr(coef_array(c, coef)));
    k_ls_copy_bulk<<<grid, block, 0, c.stream>>>(G, arr(a), tmp);
    c.launches += 2;
    return cudaGetLastError();
  };
  for (int it = 0; it < c.params.current_smoothing; ++it) {
    cudaError_t e;
    if ((e = pass(c.fields.J[0], AP_COEF_A1E)) != cudaSuccess) return e;
    if ((e = pass(c.fields.J[1], AP_COEF_A2E)) != cudaSuccess) return e;
    if ((e = pass(c.fields.J[2], AP_COEF_A3E)) != cudaSuccess) return e;
    if (do_rho)
      for (int s = 0; s < c.params.num_species; ++s)
        if ((e = pass(c.fields.Rho[s], AP_COEF_DV)) != cudaSuccess) return e;
  }
  // apply_boundary's axis_rho_lower / upper run after the smoothing
  k_ls_axis_j3<<<(G.n0 + 255) / 256, 256, 0, c.stream>>>(G, arr(c.fields.J[2]));
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_ls_update_b(Ctx &c, float dt) {
  const LsGeo G = make_ls_geo(c);
  dim3 grid, block;
  bulk_shape(G, grid, block);
  k_ls_update_b<<<grid, block, 0, c.stream>>>(G, make_ls_fields(c), make_ls_coef(c), dt);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_ls_update_e(Ctx &c, float dt) {
  const LsGeo G = make_ls_geo(c);
  dim3 grid, block;
  bulk_shape(G, grid, block);
  k_ls_update_e<<<grid, block, 0, c.stream>>>(G, make_ls_fields(c), make_ls_coef(c), dt);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_ls_divs(Ctx &c) {
  const LsGeo G = make_ls_geo(c);
  dim3 grid, block;
  bulk_shape(G, grid, block);
  k_ls_divs<<<grid, block, 0, c.stream>>>(G, make_ls_fields(c), make_ls_coef(c));
  c.launches++;
  return cudaGetLastError();
}

namespace {

// measure_surface_density (ptc_updater_logsph.cu:441-490): electrons and
// ions in the cells guard0 + 1 .. guard0 + 4, spread 1-4-6-4-1 over theta
// rows with w / 3 / 16 each, summed in double.
__global__ void k_ls_surface(MeshK m, PtcK p, size_t num, double *se, double *sp) {
  const int d0 = m.dims[0], g0 = m.guard[0], g1 = m.guard[1];
  const int red = m.dims[1] - 2 * g1;
  const int ic = g0 + 2;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < num;
       idx += (size_t)gridDim.x * blockDim.x) {
    const uint32_t c = p.cell[idx];
    if (c == AP_MAX_CELL) continue;
    const int c2 = (int)__umul64hi((unsigned long long)c, m.div0);
    const int c1 = (int)c - c2 * d0;
    if (!(c1 >= ic - 1 && c1 <= ic - 1 + 3)) continue;
    const int s = ptc_type(p.flag[idx]);
    double *a = s == 0 ? se : (s == 2 ? sp : nullptr);
    if (!a) continue;
    const float wt = p.w[idx];
    const int r = c2 - g1;
    const int at[5] = {max(r - 2, 0), max(r - 1, 0), r, min(r + 1, red - 1), min(r + 2, red - 1)};
    const float k[5] = {1.0f, 4.0f, 6.0f, 4.0f, 1.0f};
#pragma unroll
    for (int q = 0; q < 5; ++q) atomicAdd(a + at[q], (double)(k[q] * wt / 3.0f / 16.0f));
  }
}

// inject_ptc (ptc_updater_logsph.cu:301-393) with the library's build
// semantics: one thread per (bulk theta row r, pair n); pair n of row r
// takes slots num + 2 (r inj + n) and + 1, empty when the row gets no
// injection (the outermost rows, or a surface denser than
// 1.5 sin(theta_c) / dtheta^2 / q_e). x2 from Philox4x32-10 with counter
// (call, i, n, 0).
__global__ void k_ls_inject(MeshK m, PtcK p, uint64_t *ids, size_t num, int inj, float p1,
                            float w, float q_e, float gamma, uint32_t key0, uint32_t key1,
                            uint32_t call, uint64_t first_id, const double *se,
                            const double *sp) {
  const int d0 = m.dims[0], d1 = m.dims[1], g0 = m.guard[0], g1 = m.guard[1];
  const int red = d1 - 2 * g1;
  const float inv_d = 1.0f / m.delta[1];
  const uint32_t key[2] = {key0, key1};
  const size_t total = (size_t)red * inj;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(t / inj), n = (int)(t % inj);
    const int i = r + g1;
    const float dens = (float)(se[r] > sp[r] ? se[r] : sp[r]);
    const float sin_c = sinf(mesh_pos(m.lower[1], m.delta[1], i, g1, 0.5f));
    const bool on =
        i >= g1 + 1 && i < d1 - g1 - 1 && !(q_e * dens > 1.5f * (inv_d * inv_d) * sin_c);
    const size_t s0 = num + 2 * t;
    float x2 = 0.0f, st = 0.0f, ct = 0.0f;
    if (on) {
      const uint32_t ctr[4] = {call, (uint32_t)i, (uint32_t)n, 0u};
      uint32_t out[4];
      philox4x32_10(ctr, key, out);
      x2 = (float)(((double)(out[0] >> 8) + 0.5) * (1.0 / 16777216.0));
      const float th = mesh_pos(m.lower[1], m.delta[1], i, g1, x2);
      st = sinf(th);
      ct = cosf(th);
    }
    const float sg = (float)((0.0f < ct) - (ct < 0.0f));
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const size_t s = s0 + h;
      ids[s] = first_id + (s - num);
      if (!on) {
        p.cell[s] = AP_MAX_CELL;
        continue;
      }
      p.x1[s] = 0.5f;
      p.x2[s] = x2;
      p.x3[s] = 0.0f;
      p.p1[s] = p1 * 2.0f * fabsf(ct);
      p.p2[s] = p1 * st * sg;
      p.p3[s] = 0.0f;
      p.E[s] = gamma;
      p.cell[s] = (uint32_t)(g0 + 2 + i * d0);
      p.w[s] = w * st;
      p.flag[s] = (1u << 6) | ((uint32_t)h << 29);  // primary; e- then e+
    }
  }
}

}  // namespace

cudaError_t launch_ls_inject(Ctx &c, int inj, float p1, float w, uint64_t seed, uint32_t call,
                             uint64_t first_id, double *surface) {
  const int red = c.mesh.dims[1] - 2 * c.mesh.guard[1];
  cudaError_t e = cudaMemsetAsync(surface, 0, sizeof(double) * 2 * red, c.stream);
  if (e != cudaSuccess) return e;
  const PtcK p{c.ptc.x1, c.ptc.x2, c.ptc.x3, c.ptc.p1, c.ptc.p2,
               c.ptc.p3, c.ptc.E,  c.ptc.weight, c.ptc.cell, c.ptc.flag};
  if (c.number > 0) {
    size_t g = (c.number + 255) / 256;
    if (g > (size_t)c.num_sms * 8) g = (size_t)c.num_sms * 8;
    k_ls_surface<<<(int)g, 256, 0, c.stream>>>(c.mk, p, c.number, surface, surface + red);
    c.launches++;
  }
  const size_t total = (size_t)red * inj;
  if (total == 0) return cudaGetLastError();
  // E = sqrt(1.0 + p1 p1 + vphi vphi) with vphi = 0 (ptc_updater_logsph.cu:350)
  const float gamma = (float)std::sqrt(1.0 + (double)(p1 * p1) + (double)(0.0f * 0.0f));
  k_ls_inject<<<(int)((total + 255) / 256), 256, 0, c.stream>>>(
      c.mk, p, c.ptc.id, c.number, inj, p1, w, c.params.charges[1], gamma, (uint32_t)seed,
      (uint32_t)(seed >> 32), call, first_id, surface, surface + red);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_ls_field_boundary(Ctx &c, float omega) {
  const LsGeo G = make_ls_geo(c);
  const LsFields F = make_ls_fields(c);
  const int dl = c.lsp.damping_length;
  if (dl >= 0 && G.n0 - dl >= G.g0) {
    const int cells = (G.g0 + dl) * G.n1;
    if (cells > 0)
      k_ls_bnd_radial_cells<<<(cells + 255) / 256, 256, 0, c.stream>>>(G, F, omega, dl,
                                                                       c.lsp.damping_coef);
  } else {
    k_ls_bnd_radial<<<(G.n1 + 127) / 128, 128, 0, c.stream>>>(G, F, omega, dl,
                                                              c.lsp.damping_coef);
  }
  k_ls_bnd_axis<<<(G.n0 + 127) / 128, 128, 0, c.stream>>>(G, F);
  c.launches += 2;
  return cudaGetLastError();
}

}  // namespace apb

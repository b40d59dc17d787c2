// Photons and pair production: the photon movers of the particle updaters
// and radiative_transfer's emit_photons / produce_pairs with the default,
// the pulsar lab's or the 1D GR lab's user radiative functions (semantics
// in aperture_b200.h, ap_rad_params). Each pass is three launches in slot order, so its result
// does not depend on scheduling:
//   1. mark:   per slot, the model's check (a Philox draw where the model
//              draws one); per-chunk counts; per-cell produced weights,
//   2. scan:   one CTA turns the chunk counts into offsets and the total,
//   3. append: per chunk, a block scan ranks the marked slots; rank k writes
//              its photon (pair) after the store's count.
// The arithmetic keeps the reference's expressions and order; the library
// is built with -fmad=false and IEEE division and square root, and the
// float transcendentals are CUDA's expf, sinf, cosf, acosf, logf, atan2f
// (the reference's device code calls the same), pow and the square root of
// chi in double as there.
#include <cuda_runtime.h>

#include "ap_device.cuh"
#include "ap_ic.cuh"
#include "ap_internal.h"

namespace apb {

namespace {

constexpr int kRadThreads = 256;
constexpr int kRadPer = 4;
constexpr int kRadChunk = kRadThreads * kRadPer;  // 1024 slots
constexpr uint32_t kTracked = 1u << 1;            // ParticleFlag / PhotonFlag::tracked
constexpr uint32_t kSecondary = 1u << 7;          // ParticleFlag::secondary
constexpr double kPi = 3.14159265358979323846;    // CONST_PI (constant_defs.h:11)

struct PhK {
  float *x1, *x2, *x3, *p1, *p2, *p3, *E, *w, *path;
  uint32_t *cell;
  uint64_t *id;
  uint32_t *flag;
};

struct RadK {
  MeshK m;
  int model;
  float delta_t, gamma_thr, E_secondary, photon_path, r_cutoff, track_percent;
  float e_curv, l_curv, BQ, omega;
  uint32_t key[2];
  uint32_t call;
  FieldArr B[3];
  FieldArr Rho[2];
  FieldArr produced;  // ptr null: not accumulated
  // 1D GR model: Grid_1dGR's per-cell arrays, spin, omega, IC tables
  const float *alpha, *D1, *D2, *D3, *B3B1, *grr, *gff, *beta_phi;
  float a, gr_omega;
  IcK ic;
  float e_min;  // 1D gap model: photons below 0.001 / e_min are not kept
};

// The four uniforms in (0, 1] of one particle (tag 1) or photon (tag 2):
// Philox4x32-10, counter (call, id, tag); k * 2^-24, k in [1, 2^24].
__device__ __forceinline__ void uniforms(const RadK &K, uint32_t tag, uint64_t id, float u[4]) {
  const uint32_t ctr[4] = {K.call, (uint32_t)id, (uint32_t)(id >> 32), tag};
  uint32_t out[4];
  philox4x32_10(ctr, K.key, out);
#pragma unroll
  for (int i = 0; i < 4; ++i) u[i] = (float)((out[i] >> 8) + 1u) * (1.0f / 16777216.0f);
}

// Quadmesh: get_c1 / get_c2 (quadmesh.h:327-332), pos (:144-150),
// is_in_bulk (:232-251).
__device__ __forceinline__ int c1_of(const MeshK &m, uint32_t c) {
  return (int)(c % (uint32_t)m.dims[0]);
}
__device__ __forceinline__ int c2_of(const MeshK &m, uint32_t c) {
  return (int)((c / (uint32_t)m.dims[0]) % (uint32_t)m.dims[1]);
}
__device__ __forceinline__ float mpos(const MeshK &m, int i, int n, float x) {
  if (i < m.dim) return m.lower[i] + m.delta[i] * ((float)(n - m.guard[i]) + x);
  return x * m.delta[i];
}
__device__ __forceinline__ bool in_bulk(const MeshK &m, uint32_t c) {
  const int c1 = c1_of(m, c), c2 = c2_of(m, c);
  const uint32_t c3 = c / ((uint32_t)m.dims[0] * (uint32_t)m.dims[1]);
  return c1 >= m.guard[0] && c1 < m.dims[0] - m.guard[0] && c2 >= m.guard[1] &&
         c2 < m.dims[1] - m.guard[1] && c3 < (uint32_t)m.dims[2];
}

// Interpolator2D with spline_t<1> (interpolation.cuh:146-171) over the
// reference's 3 x 3 nodes, in its summation order; st0 / st1 are the x / y
// stagger bits.
__device__ __forceinline__ float cic(float dx) {
  const float w = 1.0f - fabsf(dx);
  return w > 0.0f ? w : 0.0f;
}
__device__ float interp2d(const FieldArr &f, float x1, float x2, int c1, int c2, int st0,
                          int st1) {
  float r = 0.0f;
#pragma unroll
  for (int j = 0; j <= 2; j++) {
    const int jj = j + c2 - 1;
    const float wy = cic(((float)jj + (st1 == 0 ? 0.5f : 1.0f)) - (x2 + (float)c2));
#pragma unroll
    for (int i = 0; i <= 2; i++) {
      const int ii = i + c1 - 1;
      const float wx = cic(((float)ii + (st0 == 0 ? 0.5f : 1.0f)) - (x1 + (float)c1));
      r += f.ptr[(size_t)jj * f.pitch + ii] * wx * wy;
    }
  }
  return r;
}

// rho_c of the pulsar lab (user_radiative_functions.cu:18-24).
__device__ float rho_c(float r, float theta) {
  const float c = cosf(theta);
  const float c2 = c * c;
  const float s = sinf(theta);
  if ((double)fabsf(s) < 1.0e-5) return 1.0e10f;
  return (float)((double)r * pow((double)(1.0f + 3.0f * c2), 1.5) /
                 (double)(3.0f * s * (1.0f + c2)));
}

// ---- The 1D GR lab's functions (labs/1dgr/src/cuda/radiation/
// user_radiative_functions.cuh:19-189). A metric array at x1 of cell c is
// interpolated between c - 1 and c. Draws: u0 the emission / conversion
// test, u1 the photon energy.
__device__ __forceinline__ float gr_at(const float *a, uint32_t c, float x1) {
  return a[c] * x1 + a[c - 1] * (1.0f - x1);
}
__device__ __forceinline__ float sgnf(float v) { return (float)((0.0f < v) - (v < 0.0f)); }

// Boyer-Lindquist r of the tortoise coordinate xi (the division in double
// as the reference writes it).
__device__ __forceinline__ float gr_r(float xi, float a) {
  const float rp = 1.0f + sqrtf(1.0f - a * a);
  const float rm = 1.0f - sqrtf(1.0f - a * a);
  const float exp_xi = expf(xi * (rp - rm));
  return (float)((rp - rm * exp_xi) / (1.0 - exp_xi));
}

__device__ bool check_emit_gr(const RadK &K, const PtcK &p, size_t tid, uint32_t cell,
                              const float u[4]) {
  const float alpha = gr_at(K.alpha, cell, p.x1[tid]);
  const float gamma = alpha * p.E[tid];
  return u[0] < ic_rate(K.ic, gamma) * alpha * K.delta_t;
}

__device__ void emit_photon_gr(const RadK &K, const PtcK &p, size_t tid, const PhK &ph,
                               size_t off, const float u[4]) {
  const float x1 = p.x1[tid], p1 = p.p1[tid], u0_ptc = p.E[tid];
  const uint32_t c = p.cell[tid];
  const float xi = mpos(K.m, 0, c1_of(K.m, c), x1);
  const float a = K.a;
  const float r = gr_r(xi, a);
  const float Delta = (float)(r * r - 2.0 * r + a * a);
  const float alpha = gr_at(K.alpha, c, x1), D1 = gr_at(K.D1, c, x1);
  const float D2 = gr_at(K.D2, c, x1), D3 = gr_at(K.D3, c, x1);
  const float B3B1 = gr_at(K.B3B1, c, x1), g11 = gr_at(K.grr, c, x1);
  const float g33 = gr_at(K.gff, c, x1), beta = gr_at(K.beta_phi, c, x1);
  const float ur_ptc = u0_ptc * Delta * (p1 / u0_ptc - D1) / D2;
  const float gamma = alpha * u0_ptc;
  const float Eph = ic_photon_e(K.ic, gamma, u[1]);
  const float En = (gamma - Eph) / alpha;
  p.E[tid] = En;
  float np1 = sgnf(p1) * sqrtf(En * En * (D2 * (alpha * alpha - D3) + D1 * D1) - D2);
  if (np1 != np1) np1 = 0.0f;
  p.p1[tid] = np1;
  if (fabsf(Eph) < 50.0f) return;  // the energy is taken, no photon kept
  ph.x1[off] = x1;
  ph.x2[off] = ph.x3[off] = 0.0f;
  ph.p1[off] = Delta * (Eph / gamma) * ur_ptc / g11;
  ph.p2[off] = 0.0f;
  ph.p3[off] = (Eph / gamma) * (u0_ptc * (K.gr_omega + beta) + B3B1 * ur_ptc) / g33;
  ph.E[off] = Eph / alpha;
  ph.w[off] = p.w[tid];
  ph.path[off] = 0.0f;
  ph.cell[off] = c;
}

__device__ bool check_pair_gr(const RadK &K, const PhK &ph, size_t tid, uint32_t cell,
                              const float u[4]) {
  const float alpha = gr_at(K.alpha, cell, ph.x1[tid]);
  const float u0_hat = alpha * fabsf(ph.E[tid]);
  const float prob = gg_rate(K.ic, u0_hat) * alpha * K.delta_t;
  return u[1] < prob;
}

__device__ void produce_pair_gr(const RadK &K, const PhK &ph, size_t tid, const PtcK &p,
                                size_t off) {
  const float u0 = 0.5f * fabsf(ph.E[tid]);
  const uint32_t c = ph.cell[tid];
  const float x1 = ph.x1[tid];
  ph.cell[tid] = AP_MAX_CELL;
  const float alpha = gr_at(K.alpha, c, x1), D1 = gr_at(K.D1, c, x1);
  const float D2 = gr_at(K.D2, c, x1), D3 = gr_at(K.D3, c, x1);
  float p1 = sgnf(ph.p1[tid]) * sqrtf(u0 * u0 * (D2 * (alpha * alpha - D3) + D1 * D1) - D2);
  if (p1 != p1) p1 = 0.0f;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const size_t o = off + (size_t)k;
    p.x1[o] = x1;
    p.x2[o] = p.x3[o] = 0.0f;
    p.p1[o] = p1;
    p.p2[o] = p.p3[o] = 0.0f;
    p.E[o] = u0;
    p.w[o] = ph.w[tid];
    p.cell[o] = c;
    p.flag[o] = kSecondary | ((uint32_t)k << 29);
  }
}

// ---- The 1D gap lab's functions (labs/1dgap/src/cuda/radiation/
// user_radiative_functions.cuh:17-131): the same tables on a flat line.
// Draws: u0 the emission / conversion test, u1 the photon energy.
__device__ __forceinline__ bool check_emit_gap(const RadK &K, const PtcK &p, size_t tid,
                                               const float u[4]) {
  return u[0] < ic_rate(K.ic, p.E[tid]) * K.delta_t;
}

__device__ void emit_photon_gap(const RadK &K, const PtcK &p, size_t tid, const PhK &ph,
                                size_t off, const float u[4]) {
  const float x1 = p.x1[tid], p1 = p.p1[tid];
  const uint32_t c = p.cell[tid];
  const float gamma = p.E[tid];
  float Eph = ic_photon_e(K.ic, gamma, u[1]);
  if (Eph >= gamma - 1.01f) Eph = gamma - 1.01f;
  const float En = gamma - Eph;
  p.E[tid] = En;
  float np1 = En * p1 / gamma;
  if (np1 != np1) np1 = 0.0f;
  p.p1[tid] = np1;
  if (fabsf(Eph) < 0.001f / K.e_min) return;  // the energy is taken, no photon kept
  ph.x1[off] = x1;
  ph.x2[off] = ph.x3[off] = 0.0f;
  ph.p1[off] = sgnf(p1) * Eph;
  ph.p2[off] = ph.p3[off] = 0.0f;
  ph.E[off] = Eph;
  ph.w[off] = p.w[tid];
  ph.path[off] = 0.0f;
  ph.cell[off] = c;
}

__device__ __forceinline__ bool check_pair_gap(const RadK &K, const PhK &ph, size_t tid,
                                               const float u[4]) {
  return u[1] < gg_rate(K.ic, ph.E[tid]) * K.delta_t;
}

__device__ void produce_pair_gap(const RadK &K, const PhK &ph, size_t tid, const PtcK &p,
                                 size_t off) {
  const float Eph = fabsf(ph.p1[tid]);
  const uint32_t c = ph.cell[tid];
  const float x1 = ph.x1[tid];
  ph.cell[tid] = AP_MAX_CELL;
  float p1 = sgnf(ph.p1[tid]) * sqrtf(0.25f * Eph * Eph - 1.0f);
  if (p1 != p1) p1 = 0.0f;
  const float beta = mpos(K.m, 0, c1_of(K.m, c), x1);
  const float E = sqrtf(1.0f + p1 * p1 + beta * beta);
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const size_t o = off + (size_t)k;
    p.x1[o] = x1;
    p.x2[o] = p.x3[o] = 0.0f;
    p.p1[o] = p1;
    p.p2[o] = p.p3[o] = 0.0f;
    p.E[o] = E;
    p.w[o] = ph.w[tid];
    p.cell[o] = c;
    p.flag[o] = kSecondary | ((uint32_t)k << 29);
  }
}

// check_emit_photon (default :13-17; pulsar :26-53).
__device__ bool check_emit(const RadK &K, const PtcK &p, size_t tid, uint32_t cell,
                           const float u[4]) {
  const float gamma = p.E[tid];
  if (K.model == AP_RAD_DEFAULT) return gamma > K.gamma_thr;
  if (K.model == AP_RAD_GR1D) return check_emit_gr(K, p, tid, cell, u);
  if (K.model == AP_RAD_GAP1D) return check_emit_gap(K, p, tid, u);
  const int c1 = c1_of(K.m, cell), c2 = c2_of(K.m, cell);
  const float r = expf(mpos(K.m, 0, c1, p.x1[tid]));
  if (r > 0.6f / K.omega) return false;
  if ((double)r < 1.05) return false;
  const float theta = mpos(K.m, 1, c2, p.x2[tid]);
  const float rc = rho_c(r, theta);
  if (rc < 1.0f) return false;
  const float rate = K.delta_t * gamma / (K.l_curv * rc);
  const float Eph = K.e_curv * gamma * gamma * gamma / rc;
  return u[0] < rate && Eph > 2.1f;
}

// emit_photon (default :19-63; pulsar :55-131): the parent loses the photon
// energy and the photon goes to slot off, or the slot stays empty.
__device__ void emit_photon(const RadK &K, const PtcK &p, size_t tid, const PhK &ph, size_t off,
                            const float u[4]) {
  if (K.model == AP_RAD_GR1D) {
    emit_photon_gr(K, p, tid, ph, off, u);
    return;
  }
  if (K.model == AP_RAD_GAP1D) {
    emit_photon_gap(K, p, tid, ph, off, u);
    return;
  }
  const uint32_t c = p.cell[tid];
  const int c1 = c1_of(K.m, c), c2 = c2_of(K.m, c);
  const float p1 = p.p1[tid], p2 = p.p2[tid], p3 = p.p3[tid];
  const float gamma = p.E[tid];
  if (K.model == AP_RAD_DEFAULT) {
    const float pi = sqrtf(gamma * gamma - 1.0f);
    const float Eph = 2.5f + u[0] * (K.E_secondary - 1.0f) * 2.0f;
    const float gr = gamma - Eph;
    const float pf = sqrtf(gr * gr - 1.0f);
    p.p1[tid] = p1 * pf / pi;
    p.p2[tid] = p2 * pf / pi;
    p.p3[tid] = p3 * pf / pi;
    p.E[tid] = gamma - Eph;
    const float theta = mpos(K.m, 1, c2, p.x2[tid]);
    const float l = (1.0f / sinf(theta) - 1.0f) * K.photon_path;
    const float lph = l < 10.0f ? l : 10.0f;  // min(10.0f, l)
    if (theta < 0.005f || (double)theta > kPi - 0.005f) return;
    const float path = lph * (0.5f + 0.5f * u[1]);
    if (path > K.r_cutoff) return;
    ph.x1[off] = p.x1[tid];
    ph.x2[off] = p.x2[tid];
    ph.x3[off] = p.x3[tid];
    ph.p1[off] = Eph * p1 / pi;
    ph.p2[off] = Eph * p2 / pi;
    ph.p3[off] = Eph * p3 / pi;
    ph.E[off] = 0.0f;  // not set by the default model
    ph.w[off] = p.w[tid];
    ph.path[off] = path;
    ph.cell[off] = c;
    return;
  }
  const float x1 = p.x1[tid], x2 = p.x2[tid];
  const float pi = sqrtf(p1 * p1 + p2 * p2 + p3 * p3);
  const float r = expf(mpos(K.m, 0, c1, x1));
  const float theta = mpos(K.m, 1, c2, x2);
  const float a = gamma - 1.0f;
  const float b = K.e_curv * gamma * gamma * gamma / rho_c(r, theta);
  const float Eph = b < a ? b : a;  // std::min(a, b)
  if (Eph < 2.1f) return;
  const float gr = gamma - Eph;
  const float pf = sqrtf(gr * gr - 1.0f);
  p.p1[tid] = p1 * pf / pi;
  p.p2[tid] = p2 * pf / pi;
  p.p3[tid] = p3 * pf / pi;
  p.E[tid] = gamma - Eph;
  const float B1 = interp2d(K.B[0], x1, x2, c1, c2, 1, 0);
  const float B2 = interp2d(K.B[1], x1, x2, c1, c2, 0, 1);
  const float B3 = interp2d(K.B[2], x1, x2, c1, c2, 0, 0);
  const float B = sqrtf(B1 * B1 + B2 * B2 + B3 * B3);
  if (Eph * B / K.BQ < 2.1f && p1 > 0.0f) return;
  ph.x1[off] = p.x1[tid];
  ph.x2[off] = p.x2[tid];
  ph.x3[off] = p.x3[tid];
  ph.p1[off] = Eph * p1 / pi;
  ph.p2[off] = Eph * p2 / pi;
  ph.p3[off] = Eph * p3 / pi;
  ph.E[off] = Eph;
  ph.w[off] = p.w[tid];
  ph.path[off] = 0.0f;
  ph.cell[off] = c;
}

// check_produce_pair (default :65-68; pulsar :134-171); the pulsar checks
// remove photons by the axis and in dense plasma.
__device__ bool check_pair(const RadK &K, const PhK &ph, size_t tid, uint32_t cell) {
  if (K.model == AP_RAD_DEFAULT) return ph.path[tid] <= 0.0f;
  const int c1 = c1_of(K.m, cell), c2 = c2_of(K.m, cell);
  const float x1 = ph.x1[tid], x2 = ph.x2[tid];
  const float p1 = ph.p1[tid], p2 = ph.p2[tid], p3 = ph.p3[tid];
  const float Eph = ph.E[tid];
  const float theta = mpos(K.m, 1, c2, x2);
  if (theta < K.m.delta[1] || (double)theta > kPi - (double)K.m.delta[1]) {
    ph.cell[tid] = AP_MAX_CELL;
    return false;
  }
  const float r0 = K.Rho[0].ptr[(size_t)c2 * K.Rho[0].pitch + c1];
  const float r1 = K.Rho[1].ptr[(size_t)c2 * K.Rho[1].pitch + c1];
  const float s = fabsf(r0 + r1);
  const float rho = s < 0.0001f ? 0.0001f : s;  // max(s, 0.0001f)
  const float N = fabsf(r0) + fabsf(r1);
  const float multiplicity = N / rho;
  if (multiplicity > 50.0f) {
    ph.cell[tid] = AP_MAX_CELL;
    return false;
  }
  const float B1 = interp2d(K.B[0], x1, x2, c1, c2, 1, 0);
  const float B2 = interp2d(K.B[1], x1, x2, c1, c2, 0, 1);
  const float B3 = interp2d(K.B[2], x1, x2, c1, c2, 0, 0);
  const float B = sqrtf(B1 * B1 + B2 * B2 + B3 * B3);
  const float cth = (B1 * p1 + B2 * p2 + B3 * p3) / (B * Eph);
  const float chi = (float)((double)(Eph * B) * sqrt(1.0 - (double)(cth * cth)) / (double)K.BQ);
  return (double)chi > 0.12;
}

// produce_pair (default :70-121, the pulsar lab's is the same).
__device__ void produce_pair(const PhK &ph, size_t tid, const PtcK &p, size_t off) {
  const float p1 = ph.p1[tid], p2 = ph.p2[tid], p3 = ph.p3[tid];
  float E_ph2 = p1 * p1 + p2 * p2 + p3 * p3;
  if (E_ph2 <= 4.01f) E_ph2 = 4.01f;
  const float ratio = sqrtf(0.25f - 1.0f / E_ph2);
  const float gamma = sqrtf(1.0f + ratio * ratio * E_ph2);
  if (gamma != gamma) {
    ph.cell[tid] = AP_MAX_CELL;
    return;
  }
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const size_t o = off + (size_t)k;
    p.x1[o] = ph.x1[tid];
    p.x2[o] = ph.x2[tid];
    p.x3[o] = ph.x3[tid];
    p.p1[o] = ratio * p1;
    p.p2[o] = ratio * p2;
    p.p3[o] = ratio * p3;
    p.E[o] = gamma;
    p.w[o] = ph.w[tid];
    p.cell[o] = ph.cell[tid];
    p.flag[o] = kSecondary | ((uint32_t)k << 29);  // electron, then positron
  }
  ph.cell[tid] = AP_MAX_CELL;
}

// photon_produced / pair_produced (cell) += w for the lanes with `on`.
// Lanes hold consecutive slots, mostly sorted by cell, so many of them add
// to one cell: each group of lanes with the same cell sums its weights in
// lane order and its lowest lane adds once (the reference adds per particle
// with float atomics, radiative_transfer.cu:57-58, 126-130).
__device__ __forceinline__ void add_produced(const RadK &K, uint32_t cell, float w, bool on) {
  const unsigned any = __ballot_sync(0xffffffffu, on);
  if (!any) return;
  const uint32_t key = on ? cell : AP_MAX_CELL;
  const unsigned peers = __match_any_sync(0xffffffffu, key);
  float sum = 0.0f;
  for (int o = 0; o < 32; ++o) {
    const float v = __shfl_sync(0xffffffffu, w, o);
    if ((peers >> o) & 1u) sum += v;
  }
  const int lane = threadIdx.x & 31;
  if (on && lane == __ffs(peers) - 1)
    atomicAdd(K.produced.ptr + (size_t)c2_of(K.m, cell) * K.produced.pitch + c1_of(K.m, cell),
              sum);
}

// Exclusive scan of the chunk counts (one CTA of 1024 threads); the total
// goes to offs[nchunks].
__global__ void __launch_bounds__(1024) k_rad_scan(const uint32_t *counts, uint32_t nchunks,
                                                   uint32_t *offs) {
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t b0 = 0; b0 < nchunks; b0 += blockDim.x) {
    const uint32_t i = b0 + threadIdx.x;
    const uint32_t v = i < nchunks ? counts[i] : 0u;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0u;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      s_warp[lane] = w;
    }
    __syncthreads();
    const uint32_t before = (warp ? s_warp[warp - 1] : 0u) + s_carry;
    if (i < nchunks) offs[i] = before + x - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) s_carry = before + x;
    __syncthreads();
  }
  if (threadIdx.x == 0) offs[nchunks] = s_carry;
}

// Rank of each of this thread's four slots (ch * 1024 + 4 t + [0, 4)) among
// the marked slots, in slot order: returns the first rank and the marks.
__device__ __forceinline__ uint32_t chunk_ranks(const uint8_t *mark, size_t number, uint32_t ch,
                                                uint32_t off_ch, uint32_t *e4_out) {
  __shared__ uint32_t s_warp[kRadThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const size_t first = (size_t)ch * kRadChunk + (size_t)threadIdx.x * kRadPer;
  uint32_t e4 = 0;
  if (first + kRadPer <= number) {
    e4 = *reinterpret_cast<const uint32_t *>(mark + first);
  } else {
#pragma unroll
    for (int k = 0; k < kRadPer; ++k)
      if (first + k < number) e4 |= (uint32_t)mark[first + k] << (8 * k);
  }
  const uint32_t mine = (e4 * 0x01010101u) >> 24;  // sum of the four 0/1 bytes
  uint32_t x = mine;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  uint32_t before = 0;
  for (int w = 0; w < warp; ++w) before += s_warp[w];
  __syncthreads();
  *e4_out = e4;
  return off_ch + before + x - mine;
}

__global__ void __launch_bounds__(kRadThreads)
    k_rad_emit_mark(RadK K, PtcK p, const uint64_t *ids, size_t number, uint8_t *mark,
                    uint32_t *counts, uint32_t nchunks) {
  for (uint32_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    int cnt = 0;
#pragma unroll 1
    for (int k = 0; k < kRadPer; ++k) {
      const size_t idx = (size_t)ch * kRadChunk + (size_t)k * kRadThreads + threadIdx.x;
      bool e = false;
      uint32_t cell = AP_MAX_CELL;
      if (idx < number) {
        cell = p.cell[idx];
        if (cell != AP_MAX_CELL && in_bulk(K.m, cell) && (p.flag[idx] >> 29) != 2u) {
          float u[4];
          uniforms(K, 1u, ids[idx], u);
          e = check_emit(K, p, idx, cell, u);
        }
        mark[idx] = e ? 1 : 0;
      }
      if (K.produced.ptr) add_produced(K, cell, e ? p.w[idx] : 0.0f, e);
      cnt += __syncthreads_count(e);
    }
    if (threadIdx.x == 0) counts[ch] = (uint32_t)cnt;
  }
}

__global__ void __launch_bounds__(kRadThreads)
    k_rad_emit_append(RadK K, PtcK p, const uint64_t *ids, PhK ph, const uint8_t *mark,
                      const uint32_t *offs, size_t number, size_t ph_base, size_t ph_cap,
                      uint64_t id0, uint32_t nchunks) {
  for (uint32_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    uint32_t e4;
    uint32_t rank = chunk_ranks(mark, number, ch, offs[ch], &e4);
    const size_t first = (size_t)ch * kRadChunk + (size_t)threadIdx.x * kRadPer;
#pragma unroll 1
    for (int k = 0; k < kRadPer; ++k) {
      if (!((e4 >> (8 * k)) & 0xffu)) continue;
      const size_t idx = first + k;
      const uint32_t r = rank++;
      const size_t off = ph_base + r;
      if (off >= ph_cap) continue;  // over capacity: the parent keeps its energy
      float u[4];
      uniforms(K, 1u, ids[idx], u);
      ph.cell[off] = AP_MAX_CELL;
      emit_photon(K, p, idx, ph, off, u);
      ph.flag[off] = u[2] < K.track_percent ? kTracked : 0u;
      ph.id[off] = id0 + r;
    }
  }
}

__global__ void __launch_bounds__(kRadThreads)
    k_rad_pair_mark(RadK K, PhK ph, size_t number, uint8_t *mark, uint32_t *counts,
                    uint32_t nchunks) {
  for (uint32_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    int cnt = 0;
#pragma unroll 1
    for (int k = 0; k < kRadPer; ++k) {
      const size_t idx = (size_t)ch * kRadChunk + (size_t)k * kRadThreads + threadIdx.x;
      bool e = false;
      uint32_t cell = AP_MAX_CELL;
      if (idx < number) {
        cell = ph.cell[idx];
        if (cell != AP_MAX_CELL && in_bulk(K.m, cell)) {
          if (K.model == AP_RAD_GR1D || K.model == AP_RAD_GAP1D) {
            float u[4];
            uniforms(K, 2u, ph.id[idx], u);
            e = K.model == AP_RAD_GR1D ? check_pair_gr(K, ph, idx, cell, u)
                                       : check_pair_gap(K, ph, idx, u);
          } else {
            e = check_pair(K, ph, idx, cell);
          }
        }
        mark[idx] = e ? 1 : 0;
      }
      if (K.produced.ptr) add_produced(K, cell, e ? ph.w[idx] : 0.0f, e);
      cnt += __syncthreads_count(e);
    }
    if (threadIdx.x == 0) counts[ch] = (uint32_t)cnt;
  }
}

__global__ void __launch_bounds__(kRadThreads)
    k_rad_pair_append(RadK K, PhK ph, PtcK p, uint64_t *ids, const uint8_t *mark,
                      const uint32_t *offs, size_t number, size_t ptc_base, size_t ptc_cap,
                      uint64_t id0, uint32_t nchunks) {
  for (uint32_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    uint32_t e4;
    uint32_t rank = chunk_ranks(mark, number, ch, offs[ch], &e4);
    const size_t first = (size_t)ch * kRadChunk + (size_t)threadIdx.x * kRadPer;
#pragma unroll 1
    for (int k = 0; k < kRadPer; ++k) {
      if (!((e4 >> (8 * k)) & 0xffu)) continue;
      const size_t idx = first + k;
      const uint32_t r = rank++;
      const size_t off = ptc_base + 2 * (size_t)r;
      if (off + 1 >= ptc_cap) {  // over capacity: the photon is removed
        ph.cell[idx] = AP_MAX_CELL;
        continue;
      }
      float u[4];
      uniforms(K, 2u, ph.id[idx], u);
      p.cell[off] = p.cell[off + 1] = AP_MAX_CELL;
      p.flag[off] = p.flag[off + 1] = 0u;
      if (K.model == AP_RAD_GR1D)
        produce_pair_gr(K, ph, idx, p, off);
      else if (K.model == AP_RAD_GAP1D)
        produce_pair_gap(K, ph, idx, p, off);
      else
        produce_pair(ph, idx, p, off);
      const bool tracked = u[0] < K.track_percent;
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        if (tracked) p.flag[off + m] |= kTracked;
        ids[off + m] = id0 + 2 * (uint64_t)r + (uint64_t)m;
      }
    }
  }
}

// move_photons_cart_1d / _2d (ptc_updater.cu:627-690), then the exchange:
// wrap through periodic sides, removal through the others.
__global__ void k_rad_move_cart(MeshK m, PhK ph, size_t num, float dt, int per0, int per1) {
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < num;
       idx += (size_t)blockDim.x * gridDim.x) {
    const uint32_t c = ph.cell[idx];
    if (c == AP_MAX_CELL) continue;
    if (m.dim == 1) {
      const float p1 = ph.p1[idx], p2 = ph.p2[idx], p3 = ph.p3[idx];
      const float E = sqrtf(p1 * p1 + p2 * p2 + p3 * p3);
      const float old_x1 = ph.x1[idx], old_x2 = ph.x2[idx], old_x3 = ph.x3[idx];
      float new_x1 = old_x1 + p1 / E * dt * m.inv_delta[0];
      const int dc1 = (int)floorf(new_x1);
      int cn = (int)c + dc1;
      new_x1 -= (float)dc1;
      ph.x1[idx] = new_x1;
      ph.x2[idx] = old_x2 + p2 * dt / E;
      ph.x3[idx] = old_x3 + p3 * dt / E;
      ph.path[idx] -= dt;
      ph.cell[idx] = wrap_coord(cn, m.guard[0], m.dims[0], m.red[0], per0) ? (uint32_t)cn
                                                                            : AP_MAX_CELL;
    } else {
      const int c1 = c1_of(m, c), c2 = c2_of(m, c);
      float v1 = ph.p1[idx], v2 = ph.p2[idx], v3 = ph.p3[idx];
      const float E = sqrtf(v1 * v1 + v2 * v2 + v3 * v3);
      v1 /= E;
      v2 /= E;
      v3 /= E;
      const float old_x1 = ph.x1[idx], old_x2 = ph.x2[idx], old_x3 = ph.x3[idx];
      float new_x1 = old_x1 + v1 * dt * m.inv_delta[0];
      float new_x2 = old_x2 + v2 * dt * m.inv_delta[1];
      const int dc1 = (int)floorf(new_x1);
      const int dc2 = (int)floorf(new_x2);
      int n1 = c1 + dc1, n2 = c2 + dc2;
      new_x1 -= (float)dc1;
      new_x2 -= (float)dc2;
      ph.x1[idx] = new_x1;
      ph.x2[idx] = new_x2;
      ph.x3[idx] = old_x3 + v3 * dt;
      ph.path[idx] -= dt;
      const bool keep = wrap_coord(n1, m.guard[0], m.dims[0], m.red[0], per0) &&
                        wrap_coord(n2, m.guard[1], m.dims[1], m.red[1], per1);
      ph.cell[idx] = keep ? (uint32_t)(n1 + n2 * m.dims[0]) : AP_MAX_CELL;
    }
  }
}

// update_photon_1dgr (ptc_updater_1dgr.cu:301-400): photons outside the
// bulk are removed; the others get the GR force on p1 and move in x1, and
// tracked ones keep the lower u_0 in p2 when step % data_interval == 0.
// The reference fixes the spin to 0.99 here (:322).
struct GrPhK {
  const float *alpha, *grr, *gff, *beta_phi, *theta;
  float inv_delta, dt;
  uint32_t step, data_interval;
};
__global__ void k_rad_move_gr(MeshK m, PhK ph, size_t num, GrPhK G) {
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < num;
       idx += (size_t)blockDim.x * gridDim.x) {
    const uint32_t c = ph.cell[idx];
    if (c == AP_MAX_CELL) continue;
    if (!in_bulk(m, c)) {
      ph.cell[idx] = AP_MAX_CELL;
      continue;
    }
    float p1 = ph.p1[idx];
    const float p3 = ph.p3[idx], x1 = ph.x1[idx];
    float u0 = fabsf(ph.E[idx]);
    const float nx1 = 1.0f - x1;
    const float xi = mpos(m, 0, (int)c, x1);
    const float a = 0.99f;
    const float r = gr_r(xi, a);
    const float alpha = G.alpha[c] * x1 + G.alpha[c - 1] * nx1;
    const float gamma11 = G.grr[c] * x1 + G.grr[c - 1] * nx1;
    const float gamma33 = G.gff[c] * x1 + G.gff[c - 1] * nx1;
    const float dDelta_dr = 2.0f * r - 2.0f;
    const float dl = r * r - 2.0f * r + a * a;
    const float Delta_sqr = dl * dl;
    u0 = sqrtf(gamma11 * p1 * p1 / Delta_sqr + gamma33 * p3 * p3) / alpha;
    const float da2dr = (G.alpha[c] * G.alpha[c] - G.alpha[c - 1] * G.alpha[c - 1]) * G.inv_delta;
    const float dgamma11dxi = (G.grr[c] - G.grr[c - 1]) * G.inv_delta;
    const float dgamma33dxi = (G.gff[c] - G.gff[c - 1]) * G.inv_delta;
    const float dbetadxi = (G.beta_phi[c] - G.beta_phi[c - 1]) * G.inv_delta;
    const float gr_term =
        (-0.5f * u0 * da2dr -
         (p1 * p1 * dgamma11dxi / Delta_sqr + p3 * p3 * dgamma33dxi) * 0.5f / u0 +
         p3 * dbetadxi + gamma11 * p1 * p1 * dDelta_dr / (Delta_sqr * u0)) *
        G.dt;
    p1 += gr_term;
    u0 = sqrtf(gamma11 * p1 * p1 / Delta_sqr + gamma33 * p3 * p3) / alpha;
    ph.p1[idx] = p1;
    ph.E[idx] = u0;
    const float vr = gamma11 * p1 / (Delta_sqr * u0);
    if (G.step % G.data_interval == 0 && (ph.flag[idx] & kTracked)) {
      const float theta = G.theta[c] * x1 + G.theta[c - 1] * nx1;
      const float ct = cosf(theta);
      const float Sigma = (r * r + a * a * (ct * ct));
      const float Delta = (r * r - 2.0f * r + a * a);
      const float g_00 = -(1.0f + 2.0f * r * (r * r + a * a) / Sigma / Delta);
      const float g_03 = -2.0f * r * a / Sigma / Delta;
      ph.p2[idx] = (u0 - g_03 * p3) / g_00;
    }
    float new_x1 = x1 + vr * G.dt * G.inv_delta;
    const int dc1 = (int)floorf(new_x1);
    new_x1 -= (float)dc1;
    ph.cell[idx] = c + (uint32_t)dc1;
    ph.x1[idx] = new_x1;
  }
}

// update_photon_1dgap (ptc_updater_1dgap.cu:163-192): photons outside the
// bulk are removed, the others move one light step along the sign of p1.
__global__ void k_rad_move_gap(MeshK m, PhK ph, size_t num, float dt) {
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < num;
       idx += (size_t)blockDim.x * gridDim.x) {
    const uint32_t c = ph.cell[idx];
    if (c == AP_MAX_CELL) continue;
    if (!in_bulk(m, c)) {
      ph.cell[idx] = AP_MAX_CELL;
      continue;
    }
    const float p1 = ph.p1[idx], x1 = ph.x1[idx];
    float new_x1 = x1 + sgnf(p1) * dt * m.inv_delta[0];
    const int dc1 = (int)floorf(new_x1);
    new_x1 -= (float)dc1;
    ph.cell[idx] = c + (uint32_t)dc1;
    ph.x1[idx] = new_x1;
  }
}

// move_photons (ptc_updater_logsph.cu:58-131), then send_particles and
// clear_guard_cells: photons outside the bulk are removed. The cell is
// taken before the axis reflection, as the reference does.
__global__ void k_rad_move_logsph(MeshK m, PhK ph, size_t num, float dt, float r_cutoff) {
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < num;
       idx += (size_t)blockDim.x * gridDim.x) {
    const uint32_t c = ph.cell[idx];
    if (c == AP_MAX_CELL) continue;
    const int c1 = c1_of(m, c), c2 = c2_of(m, c);
    float v1 = ph.p1[idx], v2 = ph.p2[idx], v3 = ph.p3[idx];
    const float E = sqrtf(v1 * v1 + v2 * v2 + v3 * v3);
    v1 = v1 / E;
    v2 = v2 / E;
    v3 = v3 / E;
    const float old_x1 = ph.x1[idx], old_x2 = ph.x2[idx], old_x3 = ph.x3[idx];
    const float r1 = mpos(m, 0, c1, old_x1);
    const float exp_r1 = expf(r1);
    if (exp_r1 > r_cutoff || (double)exp_r1 < 1.02) {
      ph.cell[idx] = AP_MAX_CELL;
      continue;
    }
    const float r2 = mpos(m, 1, c2, old_x2);
    // sines and cosines from one out-of-line copy, as in the particle move
    const float2 sc2 = sin_cos_ool(r2), sc3 = sin_cos_ool(old_x3);
    float x = exp_r1 * sc2.x * sc3.y;
    float y = exp_r1 * sc2.x * sc3.x;
    float z = exp_r1 * sc2.y;
    logsph2cart_sc(v1, v2, v3, sc2.y, sc2.x, sc3.y, sc3.x);
    x += v1 * dt;
    y += v2 * dt;
    z += v3 * dt;
    float r1p = sqrtf(x * x + y * y + z * z);
    const float r2p = acosf(z / r1p);
    r1p = logf(r1p);
    const float r3p = atan2f(y, x);
    const float2 sp2 = sin_cos_ool(r2p), sp3 = sin_cos_ool(r3p);
    cart2logsph_sc(v1, v2, v3, sp2.y, sp2.x, sp3.y, sp3.x);
    ph.p1[idx] = v1 * E;
    ph.p2[idx] = v2 * E;
    ph.p3[idx] = v3 * E;
    float new_x1 = old_x1 + (r1p - r1) / m.delta[0];
    float new_x2 = old_x2 + (r2p - r2) / m.delta[1];
    int dc1 = (int)floorf(new_x1);
    int dc2 = (int)floorf(new_x2);
    const int n1 = c1 + dc1, n2 = c2 + dc2;
    new_x1 -= (float)dc1;
    new_x2 -= (float)dc2;
    if (mpos(m, 1, c2 + dc2, new_x2) < 0.0f) {
      dc2 += 1;
      new_x2 = 1.0f - new_x2;
    } else if ((double)mpos(m, 1, c2 + dc2, new_x2) >= kPi) {
      dc2 -= 1;
      new_x2 = 1.0f - new_x2;
    }
    ph.x1[idx] = new_x1;
    ph.x2[idx] = new_x2;
    ph.x3[idx] = r3p;
    ph.path[idx] -= dt;
    const bool keep = n1 >= m.guard[0] && n1 < m.dims[0] - m.guard[0] && n2 >= m.guard[1] &&
                      n2 < m.dims[1] - m.guard[1];
    ph.cell[idx] = keep ? (uint32_t)(n1 + n2 * m.dims[0]) : AP_MAX_CELL;
  }
}

PhK phk_of(const Ctx &c) {
  const ap_photons &s = c.ph;
  return PhK{s.x1, s.x2, s.x3, s.p1, s.p2, s.p3, s.E, s.weight, s.path_left, s.cell, s.id, s.flag};
}

PtcK ptck_of(const Ctx &c) {
  const ap_particles &s = c.ptc;
  return PtcK{s.x1, s.x2, s.x3, s.p1, s.p2, s.p3, s.E, s.weight, s.cell, s.flag};
}

FieldArr field_of(ap_array a) { return FieldArr{a.ptr, (int)(a.pitch / sizeof(float))}; }

RadK radk_of(const Ctx &c, ap_array produced, uint32_t call) {
  RadK K;
  K.m = c.mk;
  K.model = c.rad.model;
  K.delta_t = c.rad.delta_t;
  K.gamma_thr = c.rad.gamma_thr;
  K.E_secondary = c.rad.E_secondary;
  K.photon_path = c.rad.photon_path;
  K.r_cutoff = c.rad.r_cutoff;
  K.track_percent = c.rad.track_percent;
  K.e_curv = c.rad.e_curv;
  K.l_curv = c.rad.l_curv;
  K.BQ = c.rad.BQ;
  K.omega = c.rad.omega;
  K.key[0] = (uint32_t)c.rad.seed;
  K.key[1] = (uint32_t)(c.rad.seed >> 32);
  K.call = call;
  for (int k = 0; k < 3; ++k) K.B[k] = field_of(c.fields.B[k]);
  for (int s = 0; s < 2; ++s)
    K.Rho[s] = s < c.params.num_species ? field_of(c.fields.Rho[s]) : FieldArr{nullptr, 0};
  K.produced = field_of(produced);
  K.alpha = K.D1 = K.D2 = K.D3 = K.B3B1 = K.grr = K.gff = K.beta_phi = nullptr;
  K.a = K.gr_omega = 0.0f;
  K.ic = IcK{};
  K.e_min = c.rad.e_min;
  if (c.coord == 3) {
    K.alpha = coef_array(c, AP_GR_ALPHA).ptr;
    K.D1 = coef_array(c, AP_GR_D1).ptr;
    K.D2 = coef_array(c, AP_GR_D2).ptr;
    K.D3 = coef_array(c, AP_GR_D3).ptr;
    K.B3B1 = coef_array(c, AP_GR_B3B1).ptr;
    K.grr = coef_array(c, AP_GR_GAMMA_RR).ptr;
    K.gff = coef_array(c, AP_GR_GAMMA_FF).ptr;
    K.beta_phi = coef_array(c, AP_GR_BETA_PHI).ptr;
    K.a = (float)c.gr.a;
    K.gr_omega = (float)c.gr.omega;
  }
  if (c.ic_ready) {
    const int ng = c.ic_n_gamma, ne = c.ic_n_ep;
    K.ic.ic_rate = c.ic_buf;
    K.ic.gg_rate = c.ic_buf + ng;
    K.ic.gammas = c.ic_buf + 2 * ng;
    K.ic.dNde = c.ic_buf + 3 * ng;
    K.ic.dNde_th = c.ic_buf + 3 * ng + (size_t)ng * ne;
    K.ic.n_gamma = ng;
    K.ic.n_ep = ne;
    K.ic.dep = c.ic_dep;
    K.ic.dg = c.ic_dg;
    K.ic.dlep = c.ic_dlep;
  }
  return K;
}

// Mark bytes for n slots (rounded up to whole chunks) and chunk counts,
// offsets and the total.
int ensure_rad_scratch(Ctx &c, size_t n) {
  const size_t nchunks = (n + kRadChunk - 1) / kRadChunk;
  const size_t bytes = nchunks * kRadChunk + 16;
  if (bytes > c.rad_mark_cap) {
    cudaFree(c.rad_mark);
    c.rad_mark = nullptr;
    if (cudaMalloc(&c.rad_mark, bytes) != cudaSuccess) return AP_ERR_NOMEM;
    c.rad_mark_cap = bytes;
  }
  if (2 * nchunks + 8 > c.rad_chunks_cap) {
    cudaFree(c.rad_chunks);
    c.rad_chunks = nullptr;
    const size_t cap = 2 * nchunks + 64;
    if (cudaMalloc(&c.rad_chunks, sizeof(uint32_t) * cap) != cudaSuccess) return AP_ERR_NOMEM;
    c.rad_chunks_cap = cap;
  }
  if (!c.rad_total_host &&
      cudaMallocHost(reinterpret_cast<void **>(&c.rad_total_host), sizeof(uint32_t)) !=
          cudaSuccess)
    return AP_ERR_NOMEM;
  return AP_OK;
}

uint32_t grid_of(const Ctx &c, uint32_t nchunks) {
  const uint32_t cap = (uint32_t)c.num_sms * 8;
  return nchunks < cap ? nchunks : cap;
}

}  // namespace

int rad_move_photons(Ctx &c, float dt, uint32_t step) {
  if (!c.ph_bound || c.ph_number == 0) return AP_OK;
  const uint32_t grid = (uint32_t)c.num_sms * 4;
  if (c.coord == 3) {
    GrPhK G;
    G.alpha = coef_array(c, AP_GR_ALPHA).ptr;
    G.grr = coef_array(c, AP_GR_GAMMA_RR).ptr;
    G.gff = coef_array(c, AP_GR_GAMMA_FF).ptr;
    G.beta_phi = coef_array(c, AP_GR_BETA_PHI).ptr;
    G.theta = coef_array(c, AP_GR_THETA).ptr;
    G.inv_delta = c.mesh.inv_delta[0];
    G.dt = dt;
    G.step = step;
    G.data_interval = (uint32_t)c.params.data_interval;
    k_rad_move_gr<<<grid, 256, 0, c.stream>>>(c.mk, phk_of(c), c.ph_number, G);
  } else if (c.coord == 2) {
    k_rad_move_gap<<<grid, 256, 0, c.stream>>>(c.mk, phk_of(c), c.ph_number, dt);
  } else if (c.coord == 1)
    k_rad_move_logsph<<<grid, 256, 0, c.stream>>>(c.mk, phk_of(c), c.ph_number, dt,
                                                    c.rad.r_cutoff);
  else
    k_rad_move_cart<<<grid, 256, 0, c.stream>>>(c.mk, phk_of(c), c.ph_number, dt,
                                                  c.params.periodic[0], c.params.periodic[1]);
  c.launches++;
  return cudaGetLastError() == cudaSuccess ? AP_OK : AP_ERR_CUDA;
}

// Scratch for either store at its capacity, allocated once: an allocation
// inside a pass would stall the device between its launches.
static size_t rad_scratch_slots(const Ctx &c) {
  return c.capacity > c.ph_capacity ? c.capacity : c.ph_capacity;
}

int rad_emit_photons(Ctx &c, ap_array produced, ap_rad_counts *out) {
  const size_t number = c.number;
  if (ensure_rad_scratch(c, rad_scratch_slots(c)) != AP_OK) return AP_ERR_NOMEM;
  const uint32_t nchunks = (uint32_t)((number + kRadChunk - 1) / kRadChunk);
  uint32_t marked = 0;
  if (nchunks > 0) {
    const RadK K = radk_of(c, produced, c.rad_emit_calls);
    uint32_t *counts = c.rad_chunks, *offs = c.rad_chunks + nchunks;
    const uint32_t grid = grid_of(c, nchunks);
    k_rad_emit_mark<<<grid, kRadThreads, 0, c.stream>>>(K, ptck_of(c), c.ptc.id, number,
                                                         c.rad_mark, counts, nchunks);
    k_rad_scan<<<1, 1024, 0, c.stream>>>(counts, nchunks, offs);
    k_rad_emit_append<<<grid, kRadThreads, 0, c.stream>>>(
        K, ptck_of(c), c.ptc.id, phk_of(c), c.rad_mark, offs, number, c.ph_number, c.ph_capacity,
        c.rad_next_photon_id, nchunks);
    c.launches += 3;
    if (cudaGetLastError() != cudaSuccess) return AP_ERR_CUDA;
    if (cudaMemcpyAsync(c.rad_total_host, offs + nchunks, sizeof(uint32_t),
                        cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess)
      return AP_ERR_CUDA;
    marked = *c.rad_total_host;
  }
  const size_t room = c.ph_capacity > c.ph_number ? c.ph_capacity - c.ph_number : 0;
  const size_t written = marked < room ? marked : room;
  out->marked = marked;
  out->written = written;
  out->dropped = marked - written;
  const size_t n = c.ph_number + marked + 1;  // the reference's padding of one slot
  c.ph_number = n < c.ph_capacity ? n : c.ph_capacity;
  c.rad_next_photon_id += marked;
  c.rad_emit_calls++;
  return AP_OK;
}

int rad_produce_pairs(Ctx &c, ap_array produced, ap_rad_counts *out) {
  const size_t number = c.ph_number;
  if (ensure_rad_scratch(c, rad_scratch_slots(c)) != AP_OK) return AP_ERR_NOMEM;
  const uint32_t nchunks = (uint32_t)((number + kRadChunk - 1) / kRadChunk);
  uint32_t marked = 0;
  const size_t base = c.number + 20;  // produce_pairs starts at number + 20 (:281)
  if (nchunks > 0) {
    const RadK K = radk_of(c, produced, c.rad_pair_calls);
    uint32_t *counts = c.rad_chunks, *offs = c.rad_chunks + nchunks;
    const uint32_t grid = grid_of(c, nchunks);
    k_rad_pair_mark<<<grid, kRadThreads, 0, c.stream>>>(K, phk_of(c), number, c.rad_mark,
                                                         counts, nchunks);
    k_rad_scan<<<1, 1024, 0, c.stream>>>(counts, nchunks, offs);
    k_rad_pair_append<<<grid, kRadThreads, 0, c.stream>>>(
        K, phk_of(c), ptck_of(c), c.ptc.id, c.rad_mark, offs, number, base, c.capacity,
        c.rad_next_ptc_id, nchunks);
    c.launches += 3;
    if (cudaGetLastError() != cudaSuccess) return AP_ERR_CUDA;
    if (cudaMemcpyAsync(c.rad_total_host, offs + nchunks, sizeof(uint32_t),
                        cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess)
      return AP_ERR_CUDA;
    marked = *c.rad_total_host;
  }
  // pair k fits when base + 2k + 1 < capacity
  const size_t room = c.capacity > base + 1 ? (c.capacity - base) / 2 : 0;
  const size_t written = marked < room ? marked : room;
  out->marked = marked;
  out->written = written;
  out->dropped = marked - written;
  const size_t n = c.number + 2 * (size_t)marked + 50;  // the reference's padding
  c.number = n < c.capacity ? n : c.capacity;
  c.rad_next_ptc_id += 2 * (uint64_t)marked;
  c.rad_pair_calls++;
  return AP_OK;
}

void rad_free(Ctx &c) {
  cudaFree(c.rad_mark);
  cudaFree(c.rad_chunks);
  cudaFreeHost(c.rad_total_host);
  c.rad_mark = nullptr;
  c.rad_chunks = nullptr;
  c.rad_total_host = nullptr;
  c.rad_mark_cap = c.rad_chunks_cap = 0;
}

}  // namespace apb

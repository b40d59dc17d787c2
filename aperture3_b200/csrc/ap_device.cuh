// Device-side arithmetic of the particle update.
//
// Every expression keeps the operation order of the reference kernels and
// the library is compiled with -fmad=false and IEEE division / square root,
// so each FP32 result is the correctly rounded value of the same sequence
// of operations the reference writes down: momenta, positions and cell
// indices match an FP32 CPU evaluation of the reference bit for bit.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace apb {

// ParticleFlag bits (src/core/enum_types.h:76-87); species in the top three
// bits of the flag (src/utils/util_functions.h:66-69).
constexpr uint32_t kFlagIgnoreCurrent = 1u << 3;
constexpr uint32_t kFlagIgnoreEM = 1u << 4;
__device__ __forceinline__ int ptc_type(uint32_t flag) { return (int)(flag >> 29); }

// spline_t<1> (src/cuda/utils/interpolation.cuh:28-37): max(1 - |dx|, 0).
__device__ __forceinline__ float cic(float dx) {
  float w = 1.0f - fabsf(dx);
  return w > 0.0f ? w : 0.0f;
}

// Interpolation weights of one dimension for a particle at cell c with
// offset rel (interp_cell, interpolation.cuh:79-87). The reference visits
// the three nodes c-1, c, c+1; for an offset in [0, 1] at most two of them
// carry a nonzero weight, and which two is decided exactly:
//  - stagger 1 (node at t + 1): nodes c-1 and c; node c+1 sits at distance
//    (c + 2) - (c + rel) >= 1.
//  - stagger 0 (node at t + 0.5): nodes c-1, c when c + rel < c + 0.5,
//    otherwise c, c+1; the skipped node is at distance >= 1.
// Skipping a node whose weight is exactly zero leaves the accumulated sum
// bit-identical (the running sum starts at +0 and x + (+-0) == x).
struct Weights1D {
  int base0;       // first node for stagger 0 (c-1 or c)
  float w0[2];     // stagger-0 weights of nodes base0, base0 + 1
  float w1[2];     // stagger-1 weights of nodes c-1, c
};

__device__ __forceinline__ Weights1D weights_1d(float rel, int c) {
  Weights1D W;
  float xc = rel + (float)c;
  float fc = (float)c;
  float fcm = (float)(c - 1);
  W.w1[0] = cic((fcm + 1.0f) - xc);
  W.w1[1] = cic((fc + 1.0f) - xc);
  if (xc < fc + 0.5f) {
    W.base0 = c - 1;
    W.w0[0] = cic((fcm + 0.5f) - xc);
    W.w0[1] = cic((fc + 0.5f) - xc);
  } else {
    W.base0 = c;
    W.w0[0] = cic((fc + 0.5f) - xc);
    W.w0[1] = cic(((float)(c + 1) + 0.5f) - xc);
  }
  return W;
}

// vay_push (src/cuda/algorithms/vay_push.cuh:8-30). E and B are already
// scaled by q dt / (2 m).
__device__ __forceinline__ void vay_push(float &p1, float &p2, float &p3, float &gamma,
                                         float E1, float E2, float E3, float B1,
                                         float B2, float B3) {
  float up1 = p1 + 2.0f * E1 + (p2 * B3 - p3 * B2) / gamma;
  float up2 = p2 + 2.0f * E2 + (p3 * B1 - p1 * B3) / gamma;
  float up3 = p3 + 2.0f * E3 + (p1 * B2 - p2 * B1) / gamma;
  float tt = B1 * B1 + B2 * B2 + B3 * B3;
  float ut = up1 * B1 + up2 * B2 + up3 * B3;
  float sigma = 1.0f + up1 * up1 + up2 * up2 + up3 * up3 - tt;
  float inv_gamma2 = 2.0f / (sigma + sqrtf(sigma * sigma + 4.0f * (tt + ut * ut)));
  float s = 1.0f / (1.0f + inv_gamma2 * tt);
  gamma = 1.0f / sqrtf(inv_gamma2);
  p1 = (up1 + B1 * ut * inv_gamma2 + (up2 * B3 - up3 * B2) / gamma) * s;
  p2 = (up2 + B2 * ut * inv_gamma2 + (up3 * B1 - up1 * B3) / gamma) * s;
  p3 = (up3 + B3 * ut * inv_gamma2 + (up1 * B2 - up2 * B1) / gamma) * s;
}

// movement2d / center2d (src/cuda/algorithms/ptc_updater_helper.cuh:26-41).
__device__ __forceinline__ float movement2d(float sx0, float sx1, float sy0, float sy1) {
  return (sy1 - sy0) * 0.5f * (sx0 + sx1);
}
__device__ __forceinline__ float center2d(float sx0, float sx1, float sy0, float sy1) {
  return (2.0f * sx1 * sy1 + sx0 * sy1 + sx1 * sy0 + 2.0f * sx0 * sy0) * 0.1666667f;
}

// Staggers of E1..B3 (ptc_updater.cu:55-60): bit 0 = x stagger, bit 1 = y.
// E1 0b110, E2 0b101, E3 0b011, B1 0b001, B2 0b010, B3 0b100.
__host__ __device__ constexpr int stag_x(int k) {
  return (k == 0) ? 0 : (k == 1) ? 1 : (k == 2) ? 1 : (k == 3) ? 1 : (k == 4) ? 0 : 0;
}
__host__ __device__ constexpr int stag_y(int k) {
  return (k == 0) ? 1 : (k == 1) ? 0 : (k == 2) ? 1 : (k == 3) ? 0 : (k == 4) ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Log-spherical helpers. The reference's device code calls the float
// functions expf, sinf, cosf, acosf, logf, atan2f (unqualified calls on
// float arguments); these are the same functions, with their CUDA
// accuracy, so only the transcendentals differ from an FP32 CPU run.

// (t % n, t / n) of a flat cell index: one 32-bit division when t fits in
// 32 bits (every grid of realistic size), else the 64-bit forms, which are
// long instruction sequences that cost more than a cell's memory traffic.
__device__ __forceinline__ void split_index(size_t t, int n, int &x, int &y) {
  if (t <= 0xffffffffull) {
    const unsigned tu = (unsigned)t, q = tu / (unsigned)n;
    x = (int)(tu - q * (unsigned)n);
    y = (int)q;
  } else {
    x = (int)(t % (size_t)n);
    y = (int)(t / (size_t)n);
  }
}

// Quadmesh::pos(i, n, pos_in_cell) (quadmesh.h:144-150).
__device__ __forceinline__ float mesh_pos(float lower, float delta, int n, int guard, float x) {
  return lower + delta * ((float)(n - guard) + x);
}

// beta_phi (field_solver_logsph.cu:16-20); beta_phi_s takes sin(theta).
__device__ __forceinline__ float beta_phi_s(float compactness, float omega, float r,
                                            float sin_theta) {
  return -0.4f * compactness * omega * sin_theta / (r * r);
}
__device__ __forceinline__ float beta_phi(float compactness, float omega, float r, float theta) {
  return beta_phi_s(compactness, omega, r, sinf(theta));
}

// sinf(x) and cosf(x) (.x, .y) from one out-of-line copy. The fused
// log-spherical kernel takes the sine and cosine of four angles per
// particle; inlined, every copy carries the functions' full argument
// reduction and the kernel's code grows past what the instruction cache
// holds. The values are those of inline sinf / cosf.
static __device__ __noinline__ float2 sin_cos_ool(float x) {
  return make_float2(sinf(x), cosf(x));
}

// logsph2cart / cart2logsph (ptc_updater_logsph.cu:26-44); the _sc forms
// take cos x2, sin x2, cos x3, sin x3.
__device__ __forceinline__ void logsph2cart_sc(float &v1, float &v2, float &v3, float c2,
                                               float s2, float c3, float s3) {
  const float v1n = v1, v2n = v2, v3n = v3;
  v1 = v1n * s2 * c3 + v2n * c2 * c3 - v3n * s3;
  v2 = v1n * s2 * s3 + v2n * c2 * s3 + v3n * c3;
  v3 = v1n * c2 - v2n * s2;
}
__device__ __forceinline__ void cart2logsph_sc(float &v1, float &v2, float &v3, float c2,
                                               float s2, float c3, float s3) {
  const float v1n = v1, v2n = v2, v3n = v3;
  v1 = v1n * s2 * c3 + v2n * s2 * s3 + v3n * c2;
  v2 = v1n * c2 * c3 + v2n * c2 * s3 - v3n * s2;
  v3 = -v1n * s3 + v2n * c3;
}
__device__ __forceinline__ void logsph2cart(float &v1, float &v2, float &v3, float x2, float x3) {
  logsph2cart_sc(v1, v2, v3, cosf(x2), sinf(x2), cosf(x3), sinf(x3));
}
__device__ __forceinline__ void cart2logsph(float &v1, float &v2, float &v3, float x2, float x3) {
  cart2logsph_sc(v1, v2, v3, cosf(x2), sinf(x2), cosf(x3), sinf(x3));
}

// sync_kill_perp (sync_cooling.cuh:59-86); B1..B3 are the pusher's scaled
// fields, divided back by q_over_m here as the reference does.
__device__ __forceinline__ void sync_kill_perp(float &p1, float &p2, float &p3, float &gamma,
                                               float B1, float B2, float B3, float q_over_m,
                                               float coef, float B0) {
  B1 /= q_over_m;
  B2 /= q_over_m;
  B3 /= q_over_m;
  float p = sqrtf(p1 * p1 + p2 * p2 + p3 * p3);
  const float B_sqr = B1 * B1 + B2 * B2 + B3 * B3;
  const float pdotB = (p1 * B1 + p2 * B2 + p3 * B3);
  const float delta_p1 = -coef * (p1 - B1 * pdotB / B_sqr);
  const float delta_p2 = -coef * (p2 - B2 * pdotB / B_sqr);
  const float delta_p3 = -coef * (p3 - B3 * pdotB / B_sqr);
  const float f = sqrtf(B_sqr) / B0;
  p1 += delta_p1 * f;
  p2 += delta_p2 * f;
  p3 += delta_p3 * f;
  p = sqrtf(p1 * p1 + p2 * p2 + p3 * p3);
  gamma = sqrtf(1.0f + p * p);
}

// ---------------------------------------------------------------------------
// Philox4x32-10 counter-based generator (J. K. Salmon, M. A. Moraes,
// R. O. Dror, D. E. Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC 2011): ten rounds of two 32x32 -> 64-bit products with the published
// multipliers and Weyl key increments. Host and device give the same bits.
__host__ __device__ __forceinline__ uint32_t mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
#endif
}

__host__ __device__ __forceinline__ void philox4x32_10(const uint32_t ctr_in[4],
                                                      const uint32_t key_in[2],
                                                      uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int round = 0; round < 10; ++round) {
    const uint32_t hi0 = mulhi32(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    const uint32_t hi1 = mulhi32(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0;
    c1 = n1;
    c2 = n2;
    c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

// Zone-based wrap of one coordinate after a move of at most one cell
// (find_zone, quadmesh.h:264-273; cell shift of copy_component_to_buffer,
// kernels.cu:134-142). Returns false when the particle leaves through a
// non-periodic side.
__device__ __forceinline__ bool wrap_coord(int &c, int g, int n, int red, int periodic) {
  if (c < g) {
    if (!periodic) return false;
    c += red;
  } else if (c >= n - g) {
    if (!periodic) return false;
    c -= red;
  }
  return true;
}

}  // namespace apb

// Fused Vay push + Esirkepov deposition + move for Cartesian 1D and 2D.
//
// Replaces Kernels::ptc_push_cart_{1,2}d and deposit_current_cart_{1,2}d
// (src/cuda/algorithms/ptc_updater.cu:21-141, 220-386), which the
// reference runs as two grid-stride launches with global float atomics.
//
// 2D design: the particles are kept in a stable tile order (one list of
// slot indices per tile of TX x TY cells, maintained by a counting sort each
// step). A persistent CTA takes tiles from a queue; for each tile it
//   1. stages the E/B tile plus a one-cell halo into shared memory with six
//      TMA 2D tiled loads (no multicast) completing on an mbarrier,
//   2. zeroes a shared-memory J (and Rho) tile with a two-cell halo,
//   3. walks the tile's list in chunks of CH particles: a coalesced load
//      stages the chunk's records in shared memory, each warp then pushes
//      and deposits 32 particles that sit CH/32 places apart in the list
//      (in a cell-sorted list that puts the lanes of a warp in different
//      cells, so their current updates do not collide), and a coalesced
//      store writes the chunk back,
//   4. flushes the J tile once into 64-bit accumulators in global memory; a
//      finalize pass folds the periodic guards and rounds each cell once to
//      FP32, and
//   5. records, per particle, the direction of its new tile (0..8, 9 = gone)
//      plus per-direction counts, which the order update consumes.
//
// Current and charge are accumulated exactly in fixed point: each FP32
// contribution (the reference's value) becomes X = rint(v * 2^S), added as a
// high word X >> L (int32) and a low word X mod 2^L (uint32) with native
// 32-bit shared atomics. S and L are chosen from the largest tile population
// n so that neither word can overflow over n contributions; the sums are
// exact, so the result does not depend on the order of the atomics.
#include <cuda.h>
#include <cuda_runtime.h>

#include "ap_device.cuh"
#include "ap_internal.h"

namespace apb {

namespace {

constexpr int kThreads2D = 256;
constexpr uint32_t kDirGone = 9;
constexpr uint32_t kMbarSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

// Bounded wait on an mbarrier phase; returns false when the limit is hit.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity,
                                          uint32_t limit = kMbarSpinLimit) {
  uint32_t addr = smem_u32(bar);
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load_2d(float *dst, const CUtensorMap *map, int x, int y,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 4-byte asynchronous global -> shared copy (no register round trip).
__device__ __forceinline__ void cp_async4(void *smem_dst, const void *gmem_src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(smem_dst)),
               "l"(gmem_src)
               : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}

// Waits until at most N of this thread's committed groups are in flight.
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Bits needed to represent n (ceil(log2(n + 1))).
__device__ __forceinline__ int bits_of(uint32_t n) { return 32 - __clz(n); }

// Fixed-point format for sums of at most 2^lg contributions of magnitude at
// most qw: |X| < 2^(B-1), hi = X >> L with L = 32 - lg. With B = 63 - 2 lg,
// |sum hi| < 2^30 and sum lo < 2^32 over 2^lg contributions.
__device__ __forceinline__ FixedFmt fixed_format(int lg, int B, float qw) {
  FixedFmt f;
  f.L = 32 - lg;
  int S = B - 2;
  if (qw > 0.0f) S -= ilogbf(qw);
  f.S = max(-100, min(100, S));
  return f;
}

struct Acc32 {
  int *hi;
  unsigned *lo;
};

__device__ __forceinline__ void add_fixed(const Acc32 &a, int o, float v, float scale, int L) {
  const long long X = __float2ll_rn(v * scale);  // exact scaling by a power of two
  atomicAdd(a.hi + o, (int)(X >> L));
  atomicAdd(a.lo + o, (unsigned)X & ((1u << L) - 1u));
}

// The same for a contribution already scaled by 2^S. Scaling by a power of
// two commutes with rounding, so for a product a * b the value
// (a * 2^S) * b equals (a * b) * 2^S bit for bit whenever the result is a
// normal float; a result below the normal range rounds to X = 0 either way.
__device__ __forceinline__ void add_fixed_scaled(const Acc32 &a, int o, float vs, int L) {
  const long long X = __float2ll_rn(vs);
  atomicAdd(a.hi + o, (int)(X >> L));
  atomicAdd(a.lo + o, (unsigned)X & ((1u << L) - 1u));
}

// Chunks of at most 256 particles are double-buffered: the loads of the
// next chunk run while the current one is pushed and deposited.
template <int CH>
constexpr bool pipelined() {
  return CH <= 256;
}

template <int TX, int TY, int CH>
struct TileGeom {
  static constexpr int BX = TX + 8;   // field box width: x start rounded down to 4 floats
  static constexpr int BY = TY + 2;   // one halo row on each side
  static constexpr int FSZ = ((BX * BY + 31) / 32) * 32;  // 128-byte aligned stride
  static constexpr int JX = TX + 4;   // J tile: two halo cells on each side
  static constexpr int JY = TY + 4;
  static constexpr int JSZ = JX * JY;
  static constexpr int SP = CH + CH / 64;  // staged chunk, one pad word per 64
  static constexpr int HDR = 128;     // mbarrier, tile id, abort flag, counters
  static constexpr size_t stage_bytes() { return 10 * 4 * SP + 2 * SP; }
  static constexpr int NBUF = pipelined<CH>() ? 2 : 1;
  // double-buffered chunks: the order indices of the next two chunks
  static constexpr size_t order_bytes() { return NBUF == 2 ? 2 * 4 * CH : 0; }
  static size_t smem_bytes(int nrho, bool ls = false) {
    return HDR + 4 * 6 * FSZ + 8 * (3 + nrho) * JSZ + NBUF * stage_bytes() + (ls ? 4 * JSZ : 0) +
           order_bytes();
  }
};

__device__ __forceinline__ int spos(int e) { return e + (e >> 6); }

// Write-back modes of a staged particle.
constexpr uint8_t kWritePos = 1;  // x1, x2, x3, cell
constexpr uint8_t kWriteMom = 2;  // p1, p2, p3, E
constexpr uint8_t kWriteFlag = 4; // flag (log-spherical outflow)

// Shared-memory copy of one run's parameters (batched launches only).
template <bool kMulti>
__device__ __forceinline__ uint32_t *param_smem() {
  if constexpr (kMulti) {
    __shared__ __align__(16) uint32_t buf[sizeof(PushDepositParams) / 4];
    return buf;
  } else {
    return nullptr;
  }
}

// The fused push + deposit over the tiles of one run (kMulti false: the
// parameters P0 and tensor maps maps0 live in the kernel's parameter
// space) or of a batch of runs (kMulti true: runs[r] in global memory,
// run r owning tiles [base[r], base[r + 1]) of one queue; each CTA copies
// the parameters of the run whose tile it takes into shared memory, so
// the per-particle code reads them from there and not through global
// loads that the particle stores could alias).
template <int TX, int TY, int CH, bool kTMA, bool kRho, bool kLS, bool kMulti>
__device__ __forceinline__ void push_deposit_tiles(const PushDepositParams &P0,
                                                   const CUtensorMap *maps0,
                                                   const RunDesc *__restrict__ runs,
                                                   const uint32_t *__restrict__ base, int nruns,
                                                   uint32_t *queue) {
  using G = TileGeom<TX, TY, CH>;
  constexpr int SP = G::SP;
  constexpr int PER_THREAD = CH / kThreads2D;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *mbar = reinterpret_cast<uint64_t *>(smem);
  int *s_tile = reinterpret_cast<int *>(smem + 8);
  int *s_abort = reinterpret_cast<int *>(smem + 12);
  uint32_t *s_cnt = reinterpret_cast<uint32_t *>(smem + 16);
  float *sF = reinterpret_cast<float *>(smem + G::HDR);
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;

  if (tid == 0) {
    if (kTMA) mbar_init(mbar, 1);
    *s_abort = 0;
  }
  __syncthreads();

  uint32_t *s_pbuf = param_smem<kMulti>();
  uint32_t phase = 0;
  for (;;) {
    if (tid == 0) *s_tile = (int)atomicAdd(queue, 1u);
    if (tid < 10) s_cnt[tid] = 0;
    __syncthreads();
    const int g = *s_tile;
    const CUtensorMap *mp = maps0;
    int t = g;
    if constexpr (kMulti) {
      if ((uint32_t)g >= base[nruns]) break;
      int lo = 0, hi = nruns - 1;  // largest r with base[r] <= g
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (base[mid] <= (uint32_t)g) lo = mid;
        else hi = mid - 1;
      }
      const uint32_t *src = reinterpret_cast<const uint32_t *>(&runs[lo].P);
      for (int i = tid; i < (int)(sizeof(PushDepositParams) / 4); i += kThreads2D)
        s_pbuf[i] = src[i];
      __syncthreads();
      mp = runs[lo].maps.m;
      t = g - (int)base[lo];
    } else {
      if (g >= P0.t.ntiles) break;
    }
    const PushDepositParams &P =
        kMulti ? *reinterpret_cast<const PushDepositParams *>(s_pbuf) : P0;

    // shared-memory layout of this run (the charge tile depends on its
    // number of species)
    const int ncomp = 3 + (kRho ? P.num_species : 0);
    int *sJhi = reinterpret_cast<int *>(sF + 6 * G::FSZ);
    unsigned *sJlo = reinterpret_cast<unsigned *>(sJhi + ncomp * G::JSZ);
    float *st = reinterpret_cast<float *>(sJlo + ncomp * G::JSZ);
    // log-spherical: cell volumes over the J tile window
    float *s_dv = reinterpret_cast<float *>(reinterpret_cast<unsigned char *>(st) +
                                            G::NBUF * G::stage_bytes());
    uint32_t *s_ord = reinterpret_cast<uint32_t *>(s_dv + (kLS ? G::JSZ : 0));
    const int dims0 = P.m.dims[0], dims1 = P.m.dims[1];
    const int g0 = P.m.guard[0], g1 = P.m.guard[1];
    const int nacc = ncomp * G::JSZ;

    // fixed-point format of this update, from the largest tile population
    const int lg = max(4, bits_of(*P.n_max));
    const FixedFmt fx = fixed_format(lg, 63 - 2 * lg, P.qmax * *P.wmax);
    const float fscale = ldexpf(1.0f, fx.S);
    if (t == 0 && tid == 0) *P.fx_used = fx;

    const int tix = t % P.t.ntx, tiy = t / P.t.ntx;
    const int x0 = g0 + tix * TX, y0 = g1 + tiy * TY;
    const int xs = (x0 - 1) & ~3, ys = y0 - 1;
    const int jx0 = x0 - 2, jy0 = y0 - 2;

    // the tile's particle list; with double-buffered chunks the order
    // indices run two chunks ahead (slot (chunk index) & 1 of s_ord), so
    // the gathers of the next chunk never wait for them
    const uint32_t base = P.tile_start[t];
    const int n_t = (int)(P.tile_start[t + 1] - base);
    auto prefetch_order = [&](int c0) {
      uint32_t *dst = s_ord + ((c0 / CH) & 1) * CH;
      const int nch = min(CH, n_t - c0);
      for (int e = tid; e < nch; e += kThreads2D) cp_async4(dst + e, P.order + base + c0 + e);
      cp_async_commit();
    };
    if (G::NBUF == 2) {
      if (n_t > 0) prefetch_order(0);
      if (CH < n_t) prefetch_order(CH);
    }

    // 1. field tile
    if (kTMA) {
      if (tid == 0) {
        fence_proxy_async_smem();
        mbar_expect_tx(mbar, 6u * G::BX * G::BY * 4u);
#pragma unroll
        for (int k = 0; k < 6; ++k) tma_load_2d(sF + k * G::FSZ, mp + k, xs, ys, mbar);
      }
    } else {
      for (int i = tid; i < 6 * G::BX * G::BY; i += kThreads2D) {
        int k = i / (G::BX * G::BY), rem = i % (G::BX * G::BY);
        int yy = ys + rem / G::BX, xx = xs + rem % G::BX;
        float v = 0.0f;
        if (xx < dims0 && yy < dims1) v = P.F[k].ptr[(size_t)yy * P.F[k].pitch + xx];
        sF[k * G::FSZ + rem] = v;
      }
    }
    // 2. zero the current (and charge) tile
    for (int i = tid; i < nacc; i += kThreads2D) {
      sJhi[i] = 0;
      sJlo[i] = 0u;
    }
    if constexpr (kLS) {
      for (int i = tid; i < G::JSZ; i += kThreads2D) {
        const int gx = jx0 + i % G::JX, gy = jy0 + i / G::JX;
        s_dv[i] = (gx < dims0 && gy < dims1) ? P.dV.ptr[(size_t)gy * P.dV.pitch + gx] : 1.0f;
      }
    }
    if (kTMA) {
      if (!mbar_wait(mbar, phase)) atomicExch(s_abort, 1);
    }
    cp_async_wait_group<0>();
    __syncthreads();
    if (*s_abort) {
      if (tid == 0) {
        atomicAdd(&P.status->timeouts, 1ull);
        mbar_wait(mbar, phase);  // give copies in flight one more bounded wait
      }
      break;
    }

    // 3. particles of this tile, CH at a time
    constexpr int kStageFloats = (int)(G::stage_bytes() / 4);
    // 3a. coalesced asynchronous load of the chunk at c0 into buffer b
    auto issue = [&](int c0, int b) {
      float *sb = st + b * kStageFloats;
      const int nch = min(CH, n_t - c0);
#pragma unroll
      for (int k = 0; k < PER_THREAD; ++k) {
        const int e = tid + k * kThreads2D;
        if (e < nch) {
          const int s = spos(e);
          const uint32_t idx =
              G::NBUF == 2 ? s_ord[((c0 / CH) & 1) * CH + e] : P.order[base + c0 + e];
          reinterpret_cast<uint32_t *>(sb + 9 * SP)[s] = idx;
          cp_async4(sb + 7 * SP + s, P.p.cell + idx);
          cp_async4(sb + 8 * SP + s, P.p.flag + idx);
          cp_async4(sb + s, P.p.x1 + idx);
          cp_async4(sb + SP + s, P.p.x2 + idx);
          cp_async4(sb + 2 * SP + s, P.p.x3 + idx);
          cp_async4(sb + 3 * SP + s, P.p.p1 + idx);
          cp_async4(sb + 4 * SP + s, P.p.p2 + idx);
          cp_async4(sb + 5 * SP + s, P.p.p3 + idx);
          cp_async4(sb + 6 * SP + s, P.p.w + idx);
        }
      }
      cp_async_commit();
    };
    int buf = 0;
    uint32_t cnt_prev = 0;  // threads < 10: the tile's direction count so far
    if (G::NBUF == 2 && n_t > 0) {
      issue(0, 0);
      cp_async_wait_group<0>();
      __syncthreads();
    }
    for (int c0 = 0; c0 < n_t; c0 += CH) {
      const int nch = min(CH, n_t - c0);
      if (G::NBUF == 2) {
        // this chunk landed at the end of the previous one; start the next
        // chunk's gathers and the order indices of the one after
        if (c0 + CH < n_t) issue(c0 + CH, buf ^ 1);
        if (c0 + 2 * CH < n_t) prefetch_order(c0 + 2 * CH);
      } else {
        issue(c0, 0);
        cp_async_wait_group<0>();
        __syncthreads();
      }
      float *stc = st + buf * kStageFloats;
      float *s_x1 = stc, *s_x2 = stc + SP, *s_x3 = stc + 2 * SP;
      float *s_p1 = stc + 3 * SP, *s_p2 = stc + 4 * SP, *s_p3 = stc + 5 * SP;
      float *s_w = stc + 6 * SP;  // weight in, gamma out
      uint32_t *s_cell = reinterpret_cast<uint32_t *>(stc + 7 * SP);
      uint32_t *s_flag = reinterpret_cast<uint32_t *>(stc + 8 * SP);
      uint32_t *s_idx = reinterpret_cast<uint32_t *>(stc + 9 * SP);
      uint8_t *s_dir = reinterpret_cast<uint8_t *>(stc + 10 * SP);
      uint8_t *s_mode = s_dir + SP;
      // 3b. push + deposit: lane l of warp w takes element l*CH/32 + w*PER_THREAD + k
      for (int k = 0; k < PER_THREAD; ++k) {
        const int e = lane * (CH / 32) + warp * PER_THREAD + k;
        if (e >= nch) continue;
        const int s = spos(e);
        const uint32_t c = s_cell[s];
        const uint32_t flag = s_flag[s];
        const float x1 = s_x1[s], x2 = s_x2[s], x3 = s_x3[s];
        float p1 = s_p1[s], p2 = s_p2[s], p3 = s_p3[s];
        const float w = s_w[s];
        const int c2 = (int)__umul64hi((unsigned long long)c, P.m.div0);
        const int c1 = (int)c - c2 * dims0;
        uint32_t dir = 4;
        uint8_t mode = 0;
        const bool in_tile = (c != AP_MAX_CELL) && c1 >= x0 && c1 < x0 + TX && c2 >= y0 &&
                             c2 < y0 + TY;
        if (!in_tile) {
          atomicAdd(&P.status->tile_faults, 1ull);
          dir = kDirGone;
        } else if (p1 != p1 || p2 != p2 || p3 != p3) {
          // The reference traps here (ptc_updater.cu:102-109); the particle is
          // left untouched and reported instead.
          atomicAdd(&P.status->nan_momenta, 1ull);
        } else {
          const int sp = ptc_type(flag);
          float gamma = sqrtf(1.0f + p1 * p1 + p2 * p2 + p3 * p3);
          const bool em = !(flag & kFlagIgnoreEM);
          // log-spherical: r at the particle (user_push_2d_logsph.cuh:36)
          float r_push = 0.0f;
          if constexpr (kLS) r_push = expf(mesh_pos(P.m.lower[0], P.m.delta[0], c1, g0, x1));
          if (em) {
            const float qm = P.qm[sp];
            const Weights1D Wx = weights_1d(x1, c1);
            const Weights1D Wy = weights_1d(x2, c2);
            float fe[6];
#pragma unroll
            for (int q = 0; q < 6; ++q) {
              const float *f = sF + q * G::FSZ;
              const int ib = (stag_x(q) ? c1 - 1 : Wx.base0) - xs;
              const int jb = (stag_y(q) ? c2 - 1 : Wy.base0) - ys;
              const float wx0 = stag_x(q) ? Wx.w1[0] : Wx.w0[0];
              const float wx1 = stag_x(q) ? Wx.w1[1] : Wx.w0[1];
              const float wy0 = stag_y(q) ? Wy.w1[0] : Wy.w0[0];
              const float wy1 = stag_y(q) ? Wy.w1[1] : Wy.w0[1];
              const float *row0 = f + jb * G::BX + ib;
              const float *row1 = row0 + G::BX;
              float acc = 0.0f;
              acc += row0[0] * wx0 * wy0;
              acc += row0[1] * wx1 * wy0;
              acc += row1[0] * wx0 * wy1;
              acc += row1[1] * wx1 * wy1;
              fe[q] = acc * qm;
            }
            vay_push(p1, p2, p3, gamma, fe[0], fe[1], fe[2], fe[3], fe[4], fe[5]);
            if constexpr (kLS) {
              // gravity (gravity.cuh:12-26), applied with strength
              // dev_params.gravity on every push, then sync_kill_perp
              // when radiative cooling is on and the particle is no ion.
              p1 -= P.dt * P.ls_gravity * P.mass[sp] / (r_push * r_push * fabsf(P.charge[sp]));
              gamma = sqrtf(1.0f + p1 * p1 + p2 * p2 + p3 * p3);
              if (gamma != gamma) atomicAdd(&P.status->nan_momenta, 1ull);
              if (P.ls_rad_on && sp != 2)
                sync_kill_perp(p1, p2, p3, gamma, fe[3], fe[4], fe[5], qm, P.ls_rad_coef,
                               P.ls_B0);
            }
          } else {
            gamma = P.p.E[s_idx[s]];  // the deposit reads the stored gamma
          }
          float v1 = p1 / gamma, v2 = p2 / gamma, v3 = p3 / gamma;
          float nx1, nx2, nx3;
          int dc1, dc2;
          if constexpr (!kLS) {
            // deposit_current_cart_2d (ptc_updater.cu:295-386)
            nx1 = x1 + (v1 * P.dt) * P.m.inv_delta[0];
            nx2 = x2 + (v2 * P.dt) * P.m.inv_delta[1];
            dc1 = (int)floorf(nx1);
            dc2 = (int)floorf(nx2);
            nx1 -= (float)dc1;
            nx2 -= (float)dc2;
            nx3 = x3 + v3 * P.dt;
          } else {
            // deposit_and_move_2d_log_sph (ptc_updater_logsph.cu:163-233):
            // move in Cartesian space, return to (ln r, theta, phi), rotate
            // the velocity into the new local basis, reflect at the axis.
            const float r1 = mesh_pos(P.m.lower[0], P.m.delta[0], c1, g0, x1);
            const float exp_r1 = expf(r1);
            const float r2 = mesh_pos(P.m.lower[1], P.m.delta[1], c2, g1, x2);
            const float2 sc2 = sin_cos_ool(r2), sc3 = sin_cos_ool(x3);
            v3 = v3 - beta_phi_s(P.ls_compactness, P.ls_omega, exp_r1, sc2.x);
            float x = exp_r1 * sc2.x * sc3.y;
            float y = exp_r1 * sc2.x * sc3.x;
            float z = exp_r1 * sc2.y;
            logsph2cart_sc(v1, v2, v3, sc2.y, sc2.x, sc3.y, sc3.x);
            x += 1.0f * v1 * P.dt;  // alpha_gr(r) = 1
            y += 1.0f * v2 * P.dt;
            z += 1.0f * v3 * P.dt;
            float r1p = sqrtf(x * x + y * y + z * z);
            const float r2p = acosf(z / r1p);
            const float exp_r1p = r1p;
            r1p = logf(r1p);
            const float r3p = atan2f(y, x);
            const float2 sp2 = sin_cos_ool(r2p), sp3 = sin_cos_ool(r3p);
            cart2logsph_sc(v1, v2, v3, sp2.y, sp2.x, sp3.y, sp3.x);
            p1 = v1 * gamma;
            p2 = v2 * gamma;
            p3 = (v3 + beta_phi_s(P.ls_compactness, P.ls_omega, exp_r1p, sp2.x)) * gamma;
            nx1 = x1 + (r1p - r1) / P.m.delta[0];
            nx2 = x2 + (r2p - r2) / P.m.delta[1];
            dc1 = (int)floorf(nx1);
            dc2 = (int)floorf(nx2);
            nx1 -= (float)dc1;
            nx2 -= (float)dc2;
            if (mesh_pos(P.m.lower[1], P.m.delta[1], c2 + dc2, g1, nx2) < 0.0f) {
              dc2 += 1;
              nx2 = 1.0f - nx2;
              p2 = -p2;
              p3 = -p3;
            }
            if ((double)mesh_pos(P.m.lower[1], P.m.delta[1], c2 + dc2, g1, nx2) >=
                3.14159265358979323846) {
              dc2 -= 1;
              nx2 = 1.0f - nx2;
              p2 = -p2;
              p3 = -p3;
            }
            nx3 = r3p;
          }
          const bool far = dc1 > 1 || dc1 < -1 || dc2 > 1 || dc2 < -1;

          if (!far && !(flag & kFlagIgnoreCurrent)) {
            // Esirkepov over the reference's ranges i in [i0, i1], j in [j0, j1]
            // (2 or 3 nodes per dim). Every lane walks the same 3 x 3 window
            // starting at (ib, jb) so the warp does not diverge; the third
            // node of a 2-node range is predicated off. Cumulative sums run
            // in the reference's order, so each contribution keeps its value.
            // The third column of J1 and the third row of J2 are only ever the
            // last node of a 3-node range, where the cumulative sum covers the
            // whole support (sum of new weights minus sum of old weights,
            // zero up to rounding); the reference adds that rounding residue,
            // these sites are skipped.
            const float weight = -P.charge[sp] * w;
            // the deposit's factors pre-scaled by 2^S (exact): weight, and
            // -weight * v3 as the reference forms it before the site loop
            const float wsc = weight * fscale;
            const float w3s = -wsc * v3;
            const int ib = (dc1 == -1 ? -2 : -1), nib = (dc1 == 0 ? 2 : 3);
            const int jb = (dc2 == -1 ? -2 : -1), njb = (dc2 == 0 ? 2 : 3);
            float sx0[3], sx1[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
              const int i = ib + a;
              sx0[a] = cic(-x1 + i + 1);
              sx1[a] = cic(-nx1 + (i + 1 - dc1));
            }
            float djy[3] = {0.0f, 0.0f, 0.0f};
            const Acc32 J1{sJhi, sJlo}, J2{sJhi + G::JSZ, sJlo + G::JSZ},
                J3{sJhi + 2 * G::JSZ, sJlo + 2 * G::JSZ};
            const Acc32 R{sJhi + (3 + sp) * G::JSZ, sJlo + (3 + sp) * G::JSZ};
            const bool rho = kRho && P.do_rho && sp < P.num_species;
            const int obase = (c2 + jb - jy0) * G::JX + (c1 + ib - jx0);
#pragma unroll
            for (int b = 0; b < 3; ++b) {
              const int j = jb + b;
              const bool jv = b < njb;
              const float sy0 = cic(-x2 + j + 1);
              const float sy1 = cic(-nx2 + (j + 1 - dc2));
              float djx = 0.0f;
#pragma unroll
              for (int a = 0; a < 3; ++a) {
                if (jv && a < nib) {
                  const int o = obase + b * G::JX + a;
                  djx += movement2d(sy0, sy1, sx0[a], sx1[a]);
                  if (a < 2) add_fixed_scaled(J1, o + 1, wsc * djx, fx.L);
                  djy[a] += movement2d(sx0[a], sx1[a], sy0, sy1);
                  if (b < 2) add_fixed_scaled(J2, o + G::JX, wsc * djy[a], fx.L);
                  const float val2 = center2d(sx0[a], sx1[a], sy0, sy1);
                  if constexpr (kLS)
                    add_fixed_scaled(J3, o, w3s * val2 / s_dv[o], fx.L);
                  else
                    add_fixed_scaled(J3, o, w3s * val2, fx.L);
                  if (rho) {
                    const float s1 = sx1[a] * sy1;
                    add_fixed_scaled(R, o, -wsc * s1, fx.L);
                  }
                }
              }
            }
          }
          // move + wrap through periodic sides (send_particles semantics)
          int c1n = c1 + dc1, c2n = c2 + dc2;
          bool keep = !far;
          keep = keep && wrap_coord(c1n, g0, dims0, P.m.red[0], P.periodic[0]);
          keep = keep && wrap_coord(c2n, g1, dims1, P.m.red[1], P.periodic[1]);
          uint32_t ncell = AP_MAX_CELL;
          if (keep) {
            ncell = (uint32_t)(c1n + c2n * dims0);
            int dtx = (c1n - g0) / TX - tix;
            int dty = (c2n - g1) / TY - tiy;
            if (dtx > 1) dtx = -1;
            if (dtx < -1) dtx = 1;
            if (dty > 1) dty = -1;
            if (dty < -1) dty = 1;
            dir = (uint32_t)((dty + 1) * 3 + (dtx + 1));
            if constexpr (kLS) {
              // ptc_outflow (ptc_updater_logsph.cu:440-455)
              if (!(flag & kFlagIgnoreEM) && c1n > P.ls_outflow_c1) {
                s_flag[s] = flag | kFlagIgnoreEM;
                mode |= kWriteFlag;
              }
            }
          } else {
            dir = kDirGone;
            if (far)
              atomicAdd(&P.status->moved_far, 1ull);
            else
              atomicAdd(&P.status->lost, 1ull);
          }
          s_x1[s] = nx1;
          s_x2[s] = nx2;
          s_x3[s] = nx3;
          s_cell[s] = ncell;
          mode |= kWritePos;
          if (em || kLS) {
            s_p1[s] = p1;
            s_p2[s] = p2;
            s_p3[s] = p3;
            s_w[s] = gamma;
            mode |= kWriteMom;
          }
        }
        s_dir[s] = (uint8_t)dir;
        s_mode[s] = mode;
        const unsigned peers = __match_any_sync(__activemask(), dir);
        if (lane == __ffs(peers) - 1) atomicAdd(&s_cnt[dir], (uint32_t)__popc(peers));
      }
      __syncthreads();
      // direction counts of this chunk, for the one-pass order update
      if (P.chunk_count && tid < 10) {
        const uint32_t v = s_cnt[tid];
        P.chunk_count[((size_t)(base / CH + t) + c0 / CH) * 10 + tid] = v - cnt_prev;
        cnt_prev = v;
      }
      // 3c. coalesced write-back of the chunk
#pragma unroll
      for (int k = 0; k < PER_THREAD; ++k) {
        const int e = tid + k * kThreads2D;
        if (e < nch) {
          const int s = spos(e);
          const uint8_t mode = s_mode[s];
          const uint32_t idx = s_idx[s];
          if (P.cout.x1) {
            // compaction: every member to its tile-list position
            const size_t q = base + c0 + e;
            P.cout.x1[q] = s_x1[s];
            P.cout.x2[q] = s_x2[s];
            P.cout.x3[q] = s_x3[s];
            P.cout.p1[q] = s_p1[s];
            P.cout.p2[q] = s_p2[s];
            P.cout.p3[q] = s_p3[s];
            P.cout.E[q] = (mode & kWriteMom) ? s_w[s] : P.p.E[idx];
            P.cout.w[q] = P.p.w[idx];
            P.cout.cell[q] = s_cell[s];
            P.cout.flag[q] = s_flag[s];
            P.cout_id[q] = P.id[idx];
            P.dir[base + c0 + e] = s_dir[s];
            continue;
          }
          if (mode & kWritePos) {
            P.p.x1[idx] = s_x1[s];
            P.p.x2[idx] = s_x2[s];
            P.p.x3[idx] = s_x3[s];
            P.p.cell[idx] = s_cell[s];
          }
          if (mode & kWriteMom) {
            P.p.p1[idx] = s_p1[s];
            P.p.p2[idx] = s_p2[s];
            P.p.p3[idx] = s_p3[s];
            P.p.E[idx] = s_w[s];
          }
          if (kLS && (mode & kWriteFlag)) P.p.flag[idx] = s_flag[s];
          P.dir[base + c0 + e] = s_dir[s];
        }
      }
      if (G::NBUF == 2) cp_async_wait_group<0>();  // the next chunk and order indices
      __syncthreads();
      if (G::NBUF == 2) buf ^= 1;
    }

    // 4. flush the current (and charge) tile once
    for (int i = tid; i < nacc; i += kThreads2D) {
      const long long v = (long long)sJhi[i] * (1ll << fx.L) + (long long)sJlo[i];
      if (v == 0) continue;
      const int comp = i / G::JSZ, rem = i % G::JSZ;
      const int gx = jx0 + rem % G::JX, gy = jy0 + rem / G::JX;
      if (gx >= dims0 || gy >= dims1) continue;
      atomicAdd(P.acc + comp * P.acc_comp + (size_t)gy * P.acc_pitch + gx,
                (unsigned long long)v);
    }
    if (tid < 10) P.dir_count[t * 10 + tid] = s_cnt[tid];
    phase ^= 1u;
  }
}

template <int TX, int TY, int CH, int MINB, bool kTMA, bool kRho, bool kLS>
__global__ void __launch_bounds__(kThreads2D, MINB)
    k_push_deposit_2d(const __grid_constant__ PushDepositParams P,
                      const __grid_constant__ FieldMaps maps) {
  push_deposit_tiles<TX, TY, CH, kTMA, kRho, kLS, false>(P, maps.m, nullptr, nullptr, 0, P.queue);
}

// Many independent Cartesian runs in one persistent launch: CTAs take
// (run, tile) work items from one queue over all runs' tiles.
template <int TX, int TY, int CH, int MINB, bool kTMA, bool kRho>
__global__ void __launch_bounds__(kThreads2D, MINB)
    k_push_deposit_2d_batch(const RunDesc *__restrict__ runs, const uint32_t *__restrict__ base,
                            int nruns, uint32_t *queue) {
  push_deposit_tiles<TX, TY, CH, kTMA, kRho, false, true>(runs[0].P, nullptr, runs, base, nruns,
                                                           queue);
}

// ---------------------------------------------------------------------------
// Self-test of the bounded wait: an mbarrier that announces bytes no copy
// will bring is waited on with the field-tile wait above; the give-up is
// recorded as a timeout in the status word. No asynchronous copy is
// issued, so nothing is left in flight when the kernel returns.
__global__ void k_selftest_wait(DevStatus *status, uint32_t limit) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_expect_tx(&bar, 64u);
    if (!mbar_wait(&bar, 0u, limit)) atomicAdd(&status->timeouts, 1ull);
  }
}

// 1D: the whole line is small, so each CTA takes a contiguous chunk of
// particle slots, finds the cell range it touches, and deposits into a
// shared-memory window over that range (or straight to the global
// accumulators when the window would not fit). Fields are read through the
// read-only cache.

constexpr int kThreads1D = 256;
constexpr int kItems1D = 8;
constexpr int kChunk1D = kThreads1D * kItems1D;  // 2048 particles
constexpr int kWin1D = 6000;                     // cell-components per window

__device__ __forceinline__ float interp_1d_global(const FieldArr &f, const Weights1D &W, int c1,
                                                  int stag) {
  const int b = stag ? c1 - 1 : W.base0;
  const float w0 = stag ? W.w1[0] : W.w0[0];
  const float w1 = stag ? W.w1[1] : W.w0[1];
  float acc = 0.0f;
  acc += __ldg(f.ptr + b) * w0;
  acc += __ldg(f.ptr + b + 1) * w1;
  return acc;
}

// Warp-collective deposit of one node into the 1D window (every lane of the
// warp calls it; `act` lanes contribute a1 to J1 at window offset o + 1 and
// a2, a3 to J2, J3 at o). In a cell-sorted run neighbouring lanes hold
// particles of the same cell, so their atomics would all hit one address:
// when more than kAgg1D lanes are active but they touch at most kAgg1D
// distinct offsets, each offset's fixed-point words are summed across its
// lanes (integer sums, so the result is the same bits) and one lane adds
// them; a few active lanes add directly.
constexpr int kAgg1D = 4;

__device__ __forceinline__ void deposit_1d_node(bool act, int o, float a1, float a2, float a3,
                                                int *hi, unsigned *lo, int win_comp,
                                                float scale, int L) {
  const unsigned am = __ballot_sync(0xffffffffu, act);
  if (am == 0u) return;
  const int lane = threadIdx.x & 31;
  const unsigned mask = (1u << L) - 1u;
  unsigned h[3], l[3];
  const float a[3] = {a1, a2, a3};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const long long X = act ? __float2ll_rn(a[c] * scale) : 0ll;  // exact scaling
    h[c] = (unsigned)(int)(X >> L);
    l[c] = (unsigned)X & mask;
  }
  const int dst[3] = {o + 1, win_comp + o, 2 * win_comp + o};
  if (__popc(am) <= kAgg1D) {  // few lanes (the outer nodes of crossing particles): add directly
    if (act) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        atomicAdd(hi + dst[c], (int)h[c]);
        atomicAdd(lo + dst[c], l[c]);
      }
    }
    return;
  }
  const unsigned key = act ? (unsigned)o : (0x80000000u | (unsigned)lane);
  const unsigned peers = __match_any_sync(0xffffffffu, key);
  const unsigned leaders = __ballot_sync(0xffffffffu, act && lane == __ffs(peers) - 1);
  if (__popc(leaders) <= kAgg1D) {
    for (unsigned m = leaders; m != 0u; m &= m - 1u) {
      const int ld = __ffs(m) - 1;
      const int ko = __shfl_sync(0xffffffffu, o, ld);  // every lane takes part
      const bool in = act && o == ko;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const unsigned sh = __reduce_add_sync(0xffffffffu, in ? h[c] : 0u);
        const unsigned sl = __reduce_add_sync(0xffffffffu, in ? l[c] : 0u);
        if (lane == ld) {
          atomicAdd(hi + dst[c], (int)sh);
          atomicAdd(lo + dst[c], sl);
        }
      }
    }
  } else if (act) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      atomicAdd(hi + dst[c], (int)h[c]);
      atomicAdd(lo + dst[c], l[c]);
    }
  }
}

// One chunk of kChunk1D particle slots of a 1D run: push, deposit into a
// shared-memory window over the cells the chunk touches (or straight into
// the global accumulators when the window would not fit), move.
template <bool kRho>
__device__ __forceinline__ void push_deposit_1d_chunk(const PushDepositParams &P, size_t ch,
                                                      int *sWhi, unsigned *sWlo, int &s_lo,
                                                      int &s_hi) {
  const int tid = threadIdx.x;
  const int n0 = P.m.dims[0], g0 = P.m.guard[0];
  const int ncomp = 3 + (kRho ? P.num_species : 0);
  const int win_comp = kWin1D / ncomp;
  // A window sums at most kChunk1D contributions per cell; the global
  // accumulators at most `number`.
  const int lgw = bits_of(kChunk1D);
  const size_t number = P.d_number ? (size_t)*P.d_number : P.number;
  const int lgn = bits_of((uint32_t)min(number, (size_t)0x7fffffff));
  const FixedFmt fx = fixed_format(lgw, min(63 - 2 * lgw, 62 - lgn), P.qmax * *P.wmax);
  const float fscale = ldexpf(1.0f, fx.S);
  if (ch == 0 && tid == 0) *P.fx_used = fx;
  const size_t first = ch * kChunk1D;
  if (tid == 0) {
    s_lo = INT_MAX;
    s_hi = INT_MIN;
  }
  __syncthreads();
  uint32_t cells[kItems1D];
  int lo = INT_MAX, hi = INT_MIN;
#pragma unroll
  for (int k = 0; k < kItems1D; ++k) {
    const size_t idx = first + (size_t)k * kThreads1D + tid;
    cells[k] = idx < number ? P.p.cell[idx] : AP_MAX_CELL;
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
    for (int i = tid; i < ncomp * wlen; i += kThreads1D) {
      const int si = (i / wlen) * win_comp + i % wlen;
      sWhi[si] = 0;
      sWlo[si] = 0u;
    }
  __syncthreads();

  // The members of item k + 1 are loaded while item k is pushed and
  // deposited (the items of one thread are distinct slots).
  struct Item1D {
    uint32_t flag;
    float x1, x2, x3, p1, p2, p3, w;
  };
  auto load_item = [&](int k, Item1D &it) {
    const uint32_t c = cells[k];
    if (c == AP_MAX_CELL || (int)c < g0 || (int)c >= n0 - g0) return;
    const size_t idx = first + (size_t)k * kThreads1D + tid;
    it.flag = P.p.flag[idx];
    it.x1 = P.p.x1[idx];
    it.x2 = P.p.x2[idx];
    it.x3 = P.p.x3[idx];
    it.p1 = P.p.p1[idx];
    it.p2 = P.p.p2[idx];
    it.p3 = P.p.p3[idx];
    it.w = P.p.w[idx];
  };
  Item1D cur{}, nxt{};
  load_item(0, cur);
#pragma unroll 1
  for (int k = 0; k < kItems1D; ++k) {
    if (k + 1 < kItems1D) load_item(k + 1, nxt);
    // deposit inputs of this item; the deposit runs after the item, with
    // every lane of the warp present
    bool dep = false;
    float d_x1 = 0.0f, d_nx1 = 0.0f, d_w = 0.0f, d_v2 = 0.0f, d_v3 = 0.0f;
    int d_c1 = 0, d_dc1 = 0, d_sp = 0;
    do {  // one item; `break` skips to the next
    const size_t idx = first + (size_t)k * kThreads1D + tid;
    uint32_t c = cells[k];
    if (c == AP_MAX_CELL) break;
    if ((int)c < g0 || (int)c >= n0 - g0) {  // ptc_updater.cu:30-33
      P.p.cell[idx] = AP_MAX_CELL;
      break;
    }
    const uint32_t flag = cur.flag;
    float x1 = cur.x1;
    float p1 = cur.p1, p2 = cur.p2, p3 = cur.p3;
    if (p1 != p1 || p2 != p2 || p3 != p3) {
      atomicAdd(&P.status->nan_momenta, 1ull);
      break;
    }
    const int sp = ptc_type(flag);
    const int c1 = (int)c;
    float gamma = sqrtf(1.0f + p1 * p1 + p2 * p2 + p3 * p3);
    const bool em = !(flag & kFlagIgnoreEM);
    if (em) {
      // ptc_push_cart_1d (ptc_updater.cu:21-76): only the x stagger bit
      // matters in 1D.
      const float qm = P.qm[sp];
      const Weights1D W = weights_1d(x1, c1);
      float fe[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) fe[q] = interp_1d_global(P.F[q], W, c1, stag_x(q)) * qm;
      vay_push(p1, p2, p3, gamma, fe[0], fe[1], fe[2], fe[3], fe[4], fe[5]);
      P.p.p1[idx] = p1;
      P.p.p2[idx] = p2;
      P.p.p3[idx] = p3;
      P.p.E[idx] = gamma;
    } else {
      gamma = P.p.E[idx];
    }
    // deposit_current_cart_1d (ptc_updater.cu:220-293)
    const float w = cur.w;
    const float x2 = cur.x2, x3 = cur.x3;
    const float v1 = p1 / gamma, v2 = p2 / gamma, v3 = p3 / gamma;
    float nx1 = x1 + (v1 * P.dt) / P.m.delta[0];
    const int dc1 = (int)floorf(nx1);
    nx1 -= (float)dc1;
    const bool far = dc1 > 1 || dc1 < -1;
    P.p.x1[idx] = nx1;
    P.p.x2[idx] = x2 + v2 * P.dt;
    P.p.x3[idx] = x3 + v3 * P.dt;
    if (!far && !(flag & kFlagIgnoreCurrent)) {
      dep = true;
      d_x1 = x1;
      d_nx1 = nx1;
      d_w = P.charge[sp] * w;
      d_v2 = v2;
      d_v3 = v3;
      d_c1 = c1;
      d_dc1 = dc1;
      d_sp = sp;
    }
    int cn = c1 + dc1;
    bool keep = !far && wrap_coord(cn, g0, n0, P.m.red[0], P.periodic[0]);
    if (!keep) atomicAdd(far ? &P.status->moved_far : &P.status->lost, 1ull);
    P.p.cell[idx] = keep ? (uint32_t)cn : AP_MAX_CELL;
    } while (false);
    {
      const float weight = d_w;
      // the reference's node range [i0, i1] has 2 or 3 nodes; every lane
      // walks three node slots i0, i0 + 1, i0 + 2 (the third active only for
      // a cell crossing), in the reference's order
      const int i0 = (d_dc1 == -1 ? -2 : -1), i1 = (d_dc1 == 1 ? 1 : 0);
      float djx = 0.0f;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int i = i0 + j;
        const bool act = dep && i <= i1;
        float sx1 = 0.0f, a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;
        const int off = i + d_c1;
        if (act) {
          const float sx0 = cic(-d_x1 + i + 1);
          sx1 = cic(-d_nx1 + (i + 1 - d_dc1));
          djx += sx1 - sx0;
          a1 = -weight * djx;
          const float val1 = 0.5f * (sx0 + sx1);
          a2 = weight * d_v2 * val1;
          a3 = weight * d_v3 * val1;
        }
        if (use_smem) {
          deposit_1d_node(act, off - wlo, a1, a2, a3, sWhi, sWlo, win_comp, fscale, fx.L);
          if (act && kRho && P.do_rho && d_sp < P.num_species) {
            const Acc32 W{sWhi, sWlo};
            add_fixed(W, (3 + d_sp) * win_comp + off - wlo, weight * sx1, fscale, fx.L);
          }
        } else if (act) {
          auto gadd = [&](int k2, int x, float v) {
            atomicAdd(P.acc + k2 * P.acc_comp + x,
                      (unsigned long long)__float2ll_rn(v * fscale));
          };
          gadd(0, off + 1, a1);
          gadd(1, off, a2);
          gadd(2, off, a3);
          if (kRho && P.do_rho && d_sp < P.num_species) gadd(3 + d_sp, off, weight * sx1);
        }
      }
    }
    cur = nxt;
  }
  __syncthreads();
  if (use_smem) {
    for (int i = tid; i < ncomp * wlen; i += kThreads1D) {
      const int comp = i / wlen, o = i % wlen;
      const int si = comp * win_comp + o;
      const long long v = (long long)sWhi[si] * (1ll << fx.L) + (long long)sWlo[si];
      if (v == 0) continue;
      const int gx = wlo + o;
      if (gx < 0 || gx >= n0) continue;
      atomicAdd(P.acc + comp * P.acc_comp + gx, (unsigned long long)v);
    }
  }
  __syncthreads();
}

template <bool kRho>
__global__ void __launch_bounds__(kThreads1D)
    k_push_deposit_1d(const __grid_constant__ PushDepositParams P) {
  __shared__ int sWhi[kWin1D];
  __shared__ unsigned sWlo[kWin1D];
  __shared__ int s_lo, s_hi;
  const size_t nchunks = (P.number + kChunk1D - 1) / kChunk1D;
  for (size_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x)
    push_deposit_1d_chunk<kRho>(P, ch, sWhi, sWlo, s_lo, s_hi);
}

// Many independent 1D runs in one launch: work item g is chunk
// g - base[r] of run r; the CTA copies that run's parameters into shared
// memory before the chunk.
template <bool kRho>
__global__ void __launch_bounds__(kThreads1D)
    k_push_deposit_1d_batch(const RunDesc *__restrict__ runs, const uint32_t *__restrict__ base,
                            int nruns) {
  __shared__ int sWhi[kWin1D];
  __shared__ unsigned sWlo[kWin1D];
  __shared__ int s_lo, s_hi;
  __shared__ __align__(16) uint32_t s_pbuf[sizeof(PushDepositParams) / 4];
  const uint32_t total = base[nruns];
  const PushDepositParams &P = *reinterpret_cast<const PushDepositParams *>(s_pbuf);
  for (uint32_t g = blockIdx.x; g < total; g += gridDim.x) {
    int lo = 0, hi = nruns - 1;  // largest r with base[r] <= g
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (base[mid] <= g) lo = mid;
      else hi = mid - 1;
    }
    __syncthreads();  // the previous chunk is done with s_pbuf
    const uint32_t *src = reinterpret_cast<const uint32_t *>(&runs[lo].P);
    for (int i = threadIdx.x; i < (int)(sizeof(PushDepositParams) / 4); i += kThreads1D)
      s_pbuf[i] = src[i];
    __syncthreads();
    push_deposit_1d_chunk<kRho>(P, g - base[lo], sWhi, sWlo, s_lo, s_hi);
  }
}

template <int TX, int TY, int CH, int MINB, bool kLS = false>
cudaError_t launch_2d_tiles(Ctx &c, const PushDepositParams &P) {
  using G = TileGeom<TX, TY, CH>;
  const int nrho = P.do_rho ? P.num_species : 0;
  const size_t smem = G::smem_bytes(nrho, kLS);
  cudaError_t e = cudaMemsetAsync(P.queue, 0, sizeof(uint32_t), c.stream);
  if (e != cudaSuccess) return e;
  auto run = [&](auto kern) -> cudaError_t {
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem);
    if (err != cudaSuccess) return err;
    int per_sm = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads2D, smem);
    if (err != cudaSuccess) return err;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int grid = c.num_sms * per_sm;
    if (grid > P.t.ntiles) grid = P.t.ntiles;
    if (grid < 1) grid = 1;
    kern<<<grid, kThreads2D, smem, c.stream>>>(P, c.maps);
    c.launches++;
    return cudaGetLastError();
  };
  if (c.use_tma) {
    return P.do_rho ? run(k_push_deposit_2d<TX, TY, CH, MINB, true, true, kLS>)
                    : run(k_push_deposit_2d<TX, TY, CH, MINB, true, false, kLS>);
  }
  return P.do_rho ? run(k_push_deposit_2d<TX, TY, CH, MINB, false, true, kLS>)
                  : run(k_push_deposit_2d<TX, TY, CH, MINB, false, false, kLS>);
}

// Staged chunks of 256 particles, double-buffered, with four CTAs per SM
// (default: 64 registers, no spills; the order indices run two chunks ahead
// and the gathers one chunk ahead, so no global load is waited on inside a
// tile; measured 3 % faster than 512 single-buffered on the 1024^2 box),
// 512 single-buffered with four, 1024 with three, 2048 with two.
template <int TX, int TY>
cudaError_t launch_2d_chunk(Ctx &c, const PushDepositParams &P) {
  // log-spherical: the pipelined 256-particle chunk with three CTAs per SM
  // (64 registers, no spills; the transcendental move makes it the slower
  // kernel, so a third CTA per SM pays: 0.355 ms against 0.476 ms for
  // single-buffered 1024-particle chunks on the pulsar grid)
  if (c.coord == 1) return launch_2d_tiles<TX, TY, 256, 3, true>(c, P);
  switch (chunk_of(c)) {
    case 2048: return launch_2d_tiles<TX, TY, 2048, 2>(c, P);
    case 1024: return launch_2d_tiles<TX, TY, 1024, 3>(c, P);
    case 512: return launch_2d_tiles<TX, TY, 512, 4>(c, P);
    default: return launch_2d_tiles<TX, TY, 256, 4>(c, P);
  }
}

// Largest |weight| over slots [0, n) (non-negative floats order like their
// bit patterns).
__global__ void k_weight_max(const float *w, const uint32_t *cell, size_t n, float *out) {
  float mx = 0.0f;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    if (cell[i] != AP_MAX_CELL) mx = fmaxf(mx, fabsf(w[i]));
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0)
    atomicMax(reinterpret_cast<unsigned int *>(out), __float_as_uint(mx));
}

}  // namespace

// Recomputes the largest particle weight (after the caller changed particles).
cudaError_t launch_fixed_scale(Ctx &c) {
  cudaError_t e = cudaMemsetAsync(c.wmax, 0, sizeof(float), c.stream);
  if (e != cudaSuccess) return e;
  if (c.number > 0) {
    size_t g = (c.number + 255) / 256;
    if (g > (size_t)c.num_sms * 8) g = (size_t)c.num_sms * 8;
    k_weight_max<<<(int)g, 256, 0, c.stream>>>(c.ptc.weight, c.ptc.cell, c.number, c.wmax);
    c.launches++;
  }
  c.scale_valid = true;
  return cudaGetLastError();
}

cudaError_t launch_push_deposit_2d(Ctx &c, const PushDepositParams &P) {
  const int tx = P.t.tx, ty = P.t.ty;
  if (tx == 16 && ty == 16) return launch_2d_chunk<16, 16>(c, P);
  if (tx == 32 && ty == 16) return launch_2d_chunk<32, 16>(c, P);
  if (tx == 8 && ty == 8) return launch_2d_chunk<8, 8>(c, P);
  if (tx == 16 && ty == 8) return launch_2d_chunk<16, 8>(c, P);
  if (tx == 4 && ty == 4) return launch_2d_chunk<4, 4>(c, P);
  return cudaErrorInvalidValue;
}

namespace {

template <int TX, int TY, int CH, int MINB>
cudaError_t launch_batch_tiles(cudaStream_t stream, int num_sms, bool tma, bool do_rho,
                               int max_species, const RunDesc *runs, const uint32_t *base,
                               int nruns, uint32_t total, uint32_t *queue) {
  using G = TileGeom<TX, TY, CH>;
  const size_t smem = G::smem_bytes(do_rho ? max_species : 0);
  cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  auto run = [&](auto kern) -> cudaError_t {
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem);
    if (err != cudaSuccess) return err;
    int per_sm = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads2D, smem);
    if (err != cudaSuccess) return err;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    uint32_t grid = (uint32_t)num_sms * per_sm;
    if (grid > total) grid = total;
    if (grid < 1) grid = 1;
    kern<<<grid, kThreads2D, smem, stream>>>(runs, base, nruns, queue);
    return cudaGetLastError();
  };
  if (tma)
    return do_rho ? run(k_push_deposit_2d_batch<TX, TY, CH, MINB, true, true>)
                  : run(k_push_deposit_2d_batch<TX, TY, CH, MINB, true, false>);
  return do_rho ? run(k_push_deposit_2d_batch<TX, TY, CH, MINB, false, true>)
                : run(k_push_deposit_2d_batch<TX, TY, CH, MINB, false, false>);
}

template <int TX, int TY>
cudaError_t launch_batch_chunk(cudaStream_t stream, int num_sms, int chunk, bool tma,
                               bool do_rho, int max_species, const RunDesc *runs,
                               const uint32_t *base, int nruns, uint32_t total,
                               uint32_t *queue) {
  if (chunk == 2048)
    return launch_batch_tiles<TX, TY, 2048, 2>(stream, num_sms, tma, do_rho, max_species, runs,
                                               base, nruns, total, queue);
  if (chunk == 1024)
    return launch_batch_tiles<TX, TY, 1024, 3>(stream, num_sms, tma, do_rho, max_species, runs,
                                               base, nruns, total, queue);
  if (chunk == 512)
    return launch_batch_tiles<TX, TY, 512, 4>(stream, num_sms, tma, do_rho, max_species, runs,
                                              base, nruns, total, queue);
  return launch_batch_tiles<TX, TY, 256, 4>(stream, num_sms, tma, do_rho, max_species, runs,
                                            base, nruns, total, queue);
}

}  // namespace

cudaError_t launch_push_deposit_2d_batch(cudaStream_t stream, int num_sms, int tx, int ty,
                                         int chunk, bool tma, bool do_rho, int max_species,
                                         const RunDesc *runs, const uint32_t *base, int nruns,
                                         uint32_t total, uint32_t *queue) {
  if (total == 0) return cudaSuccess;
#define AP_BATCH_SHAPE(X, Y)                                                                 \
  if (tx == X && ty == Y)                                                                    \
    return launch_batch_chunk<X, Y>(stream, num_sms, chunk, tma, do_rho, max_species, runs, \
                                    base, nruns, total, queue);
  AP_BATCH_SHAPE(16, 16)
  AP_BATCH_SHAPE(32, 16)
  AP_BATCH_SHAPE(8, 8)
  AP_BATCH_SHAPE(16, 8)
  AP_BATCH_SHAPE(4, 4)
#undef AP_BATCH_SHAPE
  return cudaErrorInvalidValue;
}

cudaError_t launch_push_deposit_1d_batch(cudaStream_t stream, int num_sms, bool do_rho,
                                         const RunDesc *runs, const uint32_t *base, int nruns,
                                         uint32_t total_chunks) {
  if (total_chunks == 0) return cudaSuccess;
  const uint32_t grid = total_chunks < (uint32_t)num_sms * 8 ? total_chunks : (uint32_t)num_sms * 8;
  if (do_rho)
    k_push_deposit_1d_batch<true><<<grid, kThreads1D, 0, stream>>>(runs, base, nruns);
  else
    k_push_deposit_1d_batch<false><<<grid, kThreads1D, 0, stream>>>(runs, base, nruns);
  return cudaGetLastError();
}

cudaError_t launch_selftest_wait(Ctx &c, uint32_t limit) {
  k_selftest_wait<<<1, 32, 0, c.stream>>>(c.status, limit);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_push_deposit_1d(Ctx &c, const PushDepositParams &P) {
  size_t nchunks = (P.number + kChunk1D - 1) / kChunk1D;
  if (nchunks == 0) return cudaSuccess;
  int grid = (int)(nchunks < (size_t)c.num_sms * 8 ? nchunks : (size_t)c.num_sms * 8);
  if (P.do_rho)
    k_push_deposit_1d<true><<<grid, kThreads1D, 0, c.stream>>>(P);
  else
    k_push_deposit_1d<false><<<grid, kThreads1D, 0, c.stream>>>(P);
  c.launches++;
  return cudaGetLastError();
}

}  // namespace apb

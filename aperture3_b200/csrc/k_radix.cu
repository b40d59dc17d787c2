// Stable LSD radix sort of (key, value) pairs of 32-bit words.
//
// Used by sort_by_cell (keys = cell indices, values = slots) and by the
// full tile-order rebuild (keys = tile indices). It replaces the
// thrust::sort_by_key of particle_base::sort_by_cell
// (src/cuda/core/particle_base_impl.cu:435-487); the result is the unique
// stable sort, the same as the reference CPU path's two-pass counting sort
// (src/core/particle_base_impl.hpp:250-332).
//
// Each pass sorts by one 8-bit digit in three launches (reduce, scan,
// scatter):
//   1. k_rx_count: every CTA owns one contiguous range of the input (whole
//      4096-item tiles) and counts its digits into warp-private shared
//      histograms (lanes with the same digit are combined with one match,
//      and a thread's four keys with one digit count once), written
//      bin-major: counts[d * G + cta]. Keys are read 16 bytes at a time,
//      sixteen per thread in flight.
//   2. k_rx_scan_rows: one CTA per digit scans that digit's counts over
//      the CTAs (exclusive, in place) and writes the digit's total; the
//      scatter's prologue adds the exclusive scan of the totals over the
//      digits, which gives each CTA the output position of its first item
//      of every digit.
//   3. k_rx_scatter: every CTA walks its range in tiles of 4096 items; the
//      next tile is copied into shared memory (cp.async, 16 bytes at a time)
//      while the current one is sorted. Each warp ranks its 512 consecutive
//      items in order (a match per 32 items and a per-warp running count
//      per digit), the warps' counts are scanned per digit, the tile is
//      written into shared memory in digit order, and from there to global
//      memory in runs per digit (coalesced stores). Ranks follow the input
//      order inside a warp, across warps and across tiles, which makes each
//      pass stable.
// Traffic per pass and item: 4 bytes read by the count, 8 read and 8
// written by the scatter.
#include <cuda_runtime.h>

#include "ap_internal.h"

namespace apb {

namespace {

constexpr int kRxThreads = 256;
constexpr int kRxWarps = kRxThreads / 32;
constexpr int kRxBits = 8;
constexpr int kRxBins = 1 << kRxBits;
constexpr int kRxPerWarp = 512;                 // consecutive items ranked by one warp
constexpr int kRxRounds = kRxPerWarp / 32;      // 16
constexpr int kRxTile = kRxWarps * kRxPerWarp;  // 4096 items per tile
constexpr int kRxCountThreads = 512;
constexpr int kRxCountWarps = kRxCountThreads / 32;
constexpr int kRxScanThreads = 512;

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// 16-byte global -> shared copy of src_bytes (0..16) bytes, zero-filling
// the rest; with src_bytes 0 nothing is read.
__device__ __forceinline__ void cp_async16(void *dst, const void *src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(dst)), "l"(src),
               "r"(src_bytes)
               : "memory");
}

__global__ void __launch_bounds__(kRxCountThreads)
    k_rx_count(const uint32_t *__restrict__ keys, size_t n, size_t per_cta, int shift,
               uint32_t *__restrict__ counts, int G) {
  __shared__ uint32_t h[kRxCountWarps][kRxBins];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < kRxCountWarps * kRxBins; i += kRxCountThreads) (&h[0][0])[i] = 0;
  __syncthreads();
  const size_t r0 = (size_t)blockIdx.x * per_cta;  // a multiple of 4 items
  const size_t r1 = r0 + per_cta < n ? r0 + per_cta : n;
  // four 16-byte loads per thread in flight; bounds are uniform per block,
  // so every lane takes part in each match
  constexpr int kU = 4;
  for (size_t b = r0; b < r1; b += (size_t)kU * 4 * kRxCountThreads) {
    uint4 v[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const size_t i = b + ((size_t)u * kRxCountThreads + tid) * 4;
      if (i + 3 < r1) {
        v[u] = *reinterpret_cast<const uint4 *>(keys + i);
      } else {
        v[u].x = i < r1 ? keys[i] : 0u;
        v[u].y = i + 1 < r1 ? keys[i + 1] : 0u;
        v[u].z = i + 2 < r1 ? keys[i + 2] : 0u;
        v[u].w = 0u;
      }
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const size_t i = b + ((size_t)u * kRxCountThreads + tid) * 4;
      const uint32_t w4[4] = {v[u].x, v[u].y, v[u].z, v[u].w};
      uint32_t d[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) d[q] = i + q < r1 ? (w4[q] >> shift) & (kRxBins - 1) : kRxBins;
      // a thread's four keys usually share their digit (the store is in
      // cell or tile order): then one match counts all four
      const bool same = i + 3 < r1 && d[0] == d[1] && d[1] == d[2] && d[2] == d[3];
      if (__all_sync(0xffffffffu, same)) {
        const uint32_t peers = __match_any_sync(0xffffffffu, d[0]);
        if (lane == __ffs(peers) - 1) h[warp][d[0]] += 4u * __popc(peers);
        __syncwarp();
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint32_t peers = __match_any_sync(0xffffffffu, d[q]);
          if (d[q] < kRxBins && lane == __ffs(peers) - 1) h[warp][d[q]] += __popc(peers);
          __syncwarp();
        }
      }
    }
  }
  __syncthreads();
  for (int dg = tid; dg < kRxBins; dg += kRxCountThreads) {
    uint32_t s = 0;
#pragma unroll
    for (int w = 0; w < kRxCountWarps; ++w) s += h[w][dg];
    counts[(size_t)dg * G + blockIdx.x] = s;
  }
}

// Per digit (one CTA each): exclusive scan of its row counts[d * G, (d +
// 1) * G) over the CTAs, in place, and the row total into totals[d]. The
// scatter adds the exclusive scan of the totals over the digits.
__global__ void __launch_bounds__(kRxScanThreads)
    k_rx_scan_rows(uint32_t *__restrict__ counts, int G, uint32_t *__restrict__ totals) {
  __shared__ uint32_t s_w[kRxScanThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t *row = counts + (size_t)blockIdx.x * G;
  uint32_t carry = 0;
  for (int c0 = 0; c0 < G; c0 += kRxScanThreads) {
    const int i = c0 + tid;
    const uint32_t own = i < G ? row[i] : 0u;
    uint32_t inc = own;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    if (lane == 31) s_w[warp] = inc;
    __syncthreads();
    uint32_t woff = 0, all = 0;
    for (int w = 0; w < kRxScanThreads / 32; ++w) {
      woff += w < warp ? s_w[w] : 0u;
      all += s_w[w];
    }
    if (i < G) row[i] = carry + woff + inc - own;
    carry += all;
    __syncthreads();
  }
  if (tid == 0) totals[blockIdx.x] = carry;
}

struct RxSmem {
  uint32_t key[2][kRxTile];  // tile input, double-buffered; reused for the sorted tile
  uint32_t val[2][kRxTile];
  uint32_t cnt[kRxWarps][kRxBins];  // per-warp counts, then warp offsets
  uint32_t glob[kRxBins];           // output position of the next item per digit
  uint32_t start[kRxBins];          // tile-local start per digit
  uint32_t tot[kRxBins];            // tile count per digit
  uint32_t wsum[kRxWarps];
};

constexpr size_t kRxSmemBytes = sizeof(RxSmem);

__global__ void __launch_bounds__(kRxThreads, 2)
    k_rx_scatter(const uint32_t *__restrict__ kin, const uint32_t *__restrict__ vin, size_t n,
                 size_t per_cta, int shift, const uint32_t *__restrict__ offs, int G,
                 const uint32_t *__restrict__ totals, uint32_t *__restrict__ kout,
                 uint32_t *__restrict__ vout) {
  extern __shared__ __align__(16) unsigned char rx_smem[];
  RxSmem &S = *reinterpret_cast<RxSmem *>(rx_smem);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const size_t r0 = (size_t)blockIdx.x * per_cta;
  const size_t r1 = r0 + per_cta < n ? r0 + per_cta : n;
  const uint32_t lt = lanemask_lt();
  {
    // output position of this CTA's first item of each digit: the digits
    // before it (exclusive scan of the totals, one digit per thread) plus
    // the CTAs before it (the row scan)
    const uint32_t tot = totals[tid];
    uint32_t inc = tot;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    if (lane == 31) S.wsum[warp] = inc;
    __syncthreads();
    uint32_t woff = 0;
#pragma unroll
    for (int w = 0; w < kRxWarps; ++w) woff += w < warp ? S.wsum[w] : 0u;
    S.glob[tid] = woff + inc - tot + offs[(size_t)tid * G + blockIdx.x];
    __syncthreads();
  }

  // copy of the tile at t0 into buffer bi: each thread 4 x 16 bytes of keys
  // and of values (items past the end are zero-filled, never read)
  auto fetch = [&](size_t t0, int bi) {
#pragma unroll
    for (int u = 0; u < kRxTile / 4 / kRxThreads; ++u) {
      const int e = (u * kRxThreads + tid) * 4;
      const size_t i = t0 + e;
      const uint32_t bytes = i >= r1 ? 0u : (i + 4 <= r1 ? 16u : (uint32_t)(r1 - i) * 4u);
      const size_t src = bytes ? i : 0;
      cp_async16(&S.key[bi][e], kin + src, bytes);
      cp_async16(&S.val[bi][e], vin + src, bytes);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };

  int bi = 0;
  if (r0 < r1) fetch(r0, 0);
  for (size_t t0 = r0; t0 < r1; t0 += kRxTile, bi ^= 1) {
    const int tn = (int)(r1 - t0 < (size_t)kRxTile ? r1 - t0 : (size_t)kRxTile);
    if (t0 + kRxTile < r1) {
      fetch(t0 + kRxTile, bi ^ 1);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    for (int i = tid; i < kRxWarps * kRxBins; i += kRxThreads) (&S.cnt[0][0])[i] = 0;
    __syncthreads();
    // 1. in-order ranks within each warp's 512 items
    uint32_t key[kRxRounds], val[kRxRounds], rk[kRxRounds];
#pragma unroll
    for (int r = 0; r < kRxRounds; ++r) {
      const int e = warp * kRxPerWarp + r * 32 + lane;
      key[r] = S.key[bi][e];
      val[r] = S.val[bi][e];
    }
#pragma unroll
    for (int r = 0; r < kRxRounds; ++r) {
      const int e = warp * kRxPerWarp + r * 32 + lane;
      const uint32_t d = e < tn ? (key[r] >> shift) & (kRxBins - 1) : kRxBins;
      const uint32_t peers = __match_any_sync(0xffffffffu, d);
      const uint32_t base = d < kRxBins ? S.cnt[warp][d] : 0u;
      __syncwarp();
      if (d < kRxBins && lane == __ffs(peers) - 1) S.cnt[warp][d] = base + __popc(peers);
      __syncwarp();
      rk[r] = base + __popc(peers & lt);
    }
    __syncthreads();
    // 2. per digit (one per thread): warp offsets, tile count, then the
    // tile-local starts by a shuffle scan over the digits
    {
      const int dg = tid;
      uint32_t run = 0;
#pragma unroll
      for (int w = 0; w < kRxWarps; ++w) {
        const uint32_t c = S.cnt[w][dg];
        S.cnt[w][dg] = run;
        run += c;
      }
      S.tot[dg] = run;
      uint32_t inc = run;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
      }
      if (lane == 31) S.wsum[warp] = inc;
      __syncthreads();
      uint32_t woff = 0;
#pragma unroll
      for (int w = 0; w < kRxWarps; ++w) woff += w < warp ? S.wsum[w] : 0u;
      S.start[dg] = woff + inc - run;
    }
    __syncthreads();
    // 3. the tile in digit order, into the buffer it was read from
#pragma unroll
    for (int r = 0; r < kRxRounds; ++r) {
      const int e = warp * kRxPerWarp + r * 32 + lane;
      if (e < tn) {
        const uint32_t d = (key[r] >> shift) & (kRxBins - 1);
        const uint32_t lp = S.start[d] + S.cnt[warp][d] + rk[r];
        S.key[bi][lp] = key[r];
        S.val[bi][lp] = val[r];
      }
    }
    __syncthreads();
    // 4. runs per digit to their output positions
    for (int j = tid; j < tn; j += kRxThreads) {
      const uint32_t k = S.key[bi][j];
      const uint32_t d = (k >> shift) & (kRxBins - 1);
      const uint32_t pos = S.glob[d] + ((uint32_t)j - S.start[d]);
      kout[pos] = k;
      vout[pos] = S.val[bi][j];
    }
    __syncthreads();
    S.glob[tid] += S.tot[tid];
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

static_assert(kRxBins == kRxThreads, "the digit scan uses one thread per digit");
static_assert(kRxTile % (4 * kRxThreads) == 0, "whole 16-byte groups per thread");

}  // namespace

size_t radix_count_words(int num_sms) { return (size_t)kRxBins * (size_t)(num_sms * 2 + 1); }

cudaError_t radix_sort_pairs(Ctx &c, size_t n, int end_bit, uint32_t **keys_out,
                             uint32_t **vals_out) {
  uint32_t *kin = c.keys[0], *vin = c.vals[0], *kout = c.keys[1], *vout = c.vals[1];
  if (n == 0) {
    *keys_out = kin;
    *vals_out = vin;
    return cudaSuccess;
  }
  cudaError_t e = cudaFuncSetAttribute(k_rx_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kRxSmemBytes);
  if (e != cudaSuccess) return e;
  // one contiguous range of whole tiles per CTA, at most two CTAs per SM
  const size_t max_g = (size_t)c.num_sms * 2;
  const size_t tiles = (n + kRxTile - 1) / kRxTile;
  const size_t G = tiles < max_g ? tiles : max_g;
  const size_t per_cta = (tiles + G - 1) / G * kRxTile;
  const int g = (int)((n + per_cta - 1) / per_cta);
  for (int shift = 0; shift < end_bit; shift += kRxBits) {
    uint32_t *totals = c.rx_counts + (size_t)kRxBins * g;
    k_rx_count<<<g, kRxCountThreads, 0, c.stream>>>(kin, n, per_cta, shift, c.rx_counts, g);
    k_rx_scan_rows<<<kRxBins, kRxScanThreads, 0, c.stream>>>(c.rx_counts, g, totals);
    k_rx_scatter<<<g, kRxThreads, kRxSmemBytes, c.stream>>>(kin, vin, n, per_cta, shift,
                                                            c.rx_counts, g, totals, kout, vout);
    c.launches += 3;
    uint32_t *tk = kin, *tv = vin;
    kin = kout;
    vin = vout;
    kout = tk;
    vout = tv;
  }
  *keys_out = kin;
  *vals_out = vin;
  return cudaGetLastError();
}

}  // namespace apb

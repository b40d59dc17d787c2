// Pair injection for the served 1D gap runs (semantics in aperture_b200.h,
// ap_pair_params). Three launches, in slot order so that the result does
// not depend on scheduling:
//   1. mark:   per particle, emit or not (Philox draw); per-chunk counts,
//   2. scan:   one CTA turns the chunk counts into offsets and clamps the
//              total to the free capacity,
//   3. append: per chunk, a block scan ranks the emitters; rank k writes
//              its pair to slots number + 2k, number + 2k + 1 and loses
//              the photon energy.
#include <cuda_runtime.h>

#include <cstring>

#include "ap_device.cuh"
#include "ap_internal.h"

namespace apb {

namespace {

constexpr int kPairThreads = 256;
constexpr int kPairPerThread = 4;
constexpr int kPairChunk = kPairThreads * kPairPerThread;  // 1024 slots
constexpr uint32_t kFlagSecondary = 1u << 7;  // ParticleFlag::secondary

struct PairK {
  float gamma_thr, free_path, pair_energy, dt;
  uint32_t key[2];
};

__device__ __forceinline__ double uniform_of(uint32_t step, uint64_t id, const uint32_t key[2]) {
  const uint32_t ctr[4] = {step, (uint32_t)id, (uint32_t)(id >> 32), 0u};
  uint32_t out[4];
  philox4x32_10(ctr, key, out);
  return ((double)(out[0] >> 8) + 0.5) * (1.0 / 16777216.0);
}

// The emission decision of a hot particle (gamma > gamma_thr) from its
// momentum and id.
__device__ __forceinline__ bool emit_decide(const PairK &K, float gamma, float p1, float p2,
                                            float p3, uint64_t id, uint32_t step) {
  const float pm = sqrtf(p1 * p1 + p2 * p2 + p3 * p3);
  const float ds = (pm / gamma) * K.dt;
  const double u = uniform_of(step, id, K.key);
  // The decision is u < 1 - exp(-ds / free_path) evaluated in double. A
  // float estimate decides it first: expm1f is within 1 ulp and the float
  // quotient within half an ulp, so it is within 4e-7 relative of the exact
  // value, and the double expression within 1e-15 absolute of it; only a u
  // inside that band goes on to the double expression.
  const double pf = -(double)expm1f(-(ds / K.free_path));
  const double band = pf * 1e-5 + 1e-15;
  if (u < pf - band) return true;
  if (u > pf + band) return false;
  const double prob = 1.0 - exp(-(double)ds / (double)K.free_path);
  return u < prob;
}

// Marks the emitters of chunk ch and adds the chunk's count to
// chunk_count[ch] (one atomic per warp; the scan resets the counts).
// Thread t takes the four consecutive slots ch * kPairChunk + 4 t + [0, 4):
// their cells and gammas arrive in one 16-byte load each (when the arrays
// are 16-byte aligned), then the momenta and ids of the hot ones, and the
// four emit bytes leave as one word.
__device__ __forceinline__ void mark_chunk(const PairK &K, const PtcK &p, const uint64_t *ids,
                                           size_t number, uint32_t step, uint8_t *emit,
                                           uint32_t *chunk_count, uint32_t ch) {
  static_assert(kPairPerThread == 4, "four consecutive slots per thread");
  const size_t first = (size_t)ch * kPairChunk + (size_t)threadIdx.x * kPairPerThread;
  uint32_t cell[4] = {AP_MAX_CELL, AP_MAX_CELL, AP_MAX_CELL, AP_MAX_CELL};
  float gam[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  const bool vec = ((reinterpret_cast<uintptr_t>(p.cell) | reinterpret_cast<uintptr_t>(p.E)) &
                    15u) == 0;
  if (vec && first + 4 <= number) {
    const uint4 c4 = *reinterpret_cast<const uint4 *>(p.cell + first);
    const float4 g4 = *reinterpret_cast<const float4 *>(p.E + first);
    cell[0] = c4.x; cell[1] = c4.y; cell[2] = c4.z; cell[3] = c4.w;
    gam[0] = g4.x; gam[1] = g4.y; gam[2] = g4.z; gam[3] = g4.w;
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (first + k < number) {
        cell[k] = p.cell[first + k];
        gam[k] = p.E[first + k];
      }
  }
  bool hot[4];
  float q1[4], q2[4], q3[4];
  uint64_t id[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    hot[k] = cell[k] != AP_MAX_CELL && gam[k] > K.gamma_thr;
    q1[k] = hot[k] ? p.p1[first + k] : 0.0f;
    q2[k] = hot[k] ? p.p2[first + k] : 0.0f;
    q3[k] = hot[k] ? p.p3[first + k] : 0.0f;
    id[k] = hot[k] ? ids[first + k] : 0ull;
  }
  uint32_t e4 = 0;
  int cnt = 0;
  if (hot[0] | hot[1] | hot[2] | hot[3]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const bool e = hot[k] && emit_decide(K, gam[k], q1[k], q2[k], q3[k], id[k], step);
      e4 |= (e ? 1u : 0u) << (8 * k);
      cnt += e ? 1 : 0;
    }
  }
  if (first + 4 <= number) {
    *reinterpret_cast<uint32_t *>(emit + first) = e4;
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (first + k < number) emit[first + k] = (uint8_t)((e4 >> (8 * k)) & 1u);
  }
  cnt = (int)__reduce_add_sync(0xffffffffu, (unsigned)cnt);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(chunk_count + ch, (uint32_t)cnt);
}

// One CTA of 1024 threads: exclusive scan of the chunk counts into offs; the
// total is clamped to the free capacity and the device state moves on; the
// old count and next id go to tot[] for the append pass.
__device__ __forceinline__ void scan_chunks(uint32_t *chunk_count, uint32_t nchunks,
                                            uint32_t *offs, size_t capacity, PairState *st,
                                            uint32_t *tot) {
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t b0 = 0; b0 < nchunks; b0 += blockDim.x) {
    const uint32_t i = b0 + threadIdx.x;
    const uint32_t v = i < nchunks ? chunk_count[i] : 0u;
    if (i < nchunks) chunk_count[i] = 0u;  // ready for the next mark pass
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
  if (threadIdx.x == 0) {
    const uint32_t total = s_carry;
    offs[nchunks] = total;  // so that chunk ch holds offs[ch + 1] - offs[ch] emitters
    const uint32_t old = st->number;
    const size_t free_slots = capacity > old ? capacity - old : 0;
    const uint32_t room = (uint32_t)(free_slots / 2 > 0xffffffffu ? 0xffffffffu : free_slots / 2);
    const uint32_t em = total < room ? total : room;
    const unsigned long long id0 = st->next_id;
    tot[0] = em;
    tot[1] = old;
    tot[2] = (uint32_t)id0;
    tot[3] = (uint32_t)(id0 >> 32);
    st->old_number = old;
    st->emitted = em;
    st->dropped = total - em;
    st->number = old + 2 * em;
    st->next_id = id0 + 2ull * em;
    st->particle_steps += old;
    st->emitted_total += em;
    st->dropped_total += total - em;
  }
}

// Appends the pairs of the emitters of chunk ch (ranked in slot order).
// Returns false, having done nothing, for a chunk without emitters (the same
// answer in every thread of the CTA). The warp totals alternate between two
// shared buffers by `parity` (the count of chunks this CTA appended so far),
// so one barrier per chunk suffices: a buffer is rewritten only after the
// barrier of the chunk in between.
__device__ __forceinline__ bool append_chunk(const PairK &K, const PtcK &p, uint64_t *ids,
                                             const uint8_t *emit, const uint32_t *offs,
                                             const uint32_t *tot, uint32_t ch, int parity) {
  __shared__ uint32_t s_warp2[2][kPairThreads / 32];
  if (offs[ch + 1] == offs[ch]) return false;
  uint32_t *s_warp = s_warp2[parity & 1];
  const uint32_t emitted = tot[0];
  const size_t number = tot[1];
  const uint64_t id_base = (uint64_t)tot[2] | ((uint64_t)tot[3] << 32);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float Eph = K.pair_energy;
  float q = sqrtf(0.25f * Eph * Eph - 1.0f);
  if (q != q) q = 0.0f;
  const uint32_t off_ch = offs[ch];
  // thread t ranks slots ch * kPairChunk + t * kPairPerThread + [0, 4); the
  // four emit bytes are read as one word (first is a multiple of 4)
  static_assert(kPairPerThread == 4, "one 32-bit word of emit bytes per thread");
  const size_t first = (size_t)ch * kPairChunk + (size_t)threadIdx.x * kPairPerThread;
  uint32_t e4 = 0;
  if (first + kPairPerThread <= number) {
    e4 = *reinterpret_cast<const uint32_t *>(emit + first);
  } else {
#pragma unroll
    for (int k = 0; k < kPairPerThread; ++k)
      if (first + k < number) e4 |= (uint32_t)emit[first + k] << (8 * k);
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
  uint32_t rank = off_ch + before + x - mine;
#pragma unroll
  for (int k = 0; k < kPairPerThread; ++k) {
    const size_t idx = first + k;
    if (idx >= number || !((e4 >> (8 * k)) & 0xffu)) continue;
    const uint32_t r = rank++;
    if (r >= emitted) continue;  // over capacity: this parent keeps its energy
    const float gamma = p.E[idx];
    const float p1 = p.p1[idx], p2 = p.p2[idx], p3 = p.p3[idx];
    const float pm = sqrtf(p1 * p1 + p2 * p2 + p3 * p3);
    const float gn = gamma - Eph;
    const float scale = sqrtf(gn * gn - 1.0f) / pm;
    p.p1[idx] = p1 * scale;
    p.p2[idx] = p2 * scale;
    p.p3[idx] = p3 * scale;
    p.E[idx] = gn;
    const float pp = p1 > 0.0f ? q : (p1 < 0.0f ? -q : 0.0f);  // sgn(p1) * q
    const float ep = sqrtf(1.0f + pp * pp);
    const size_t d = number + 2 * (size_t)r;
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      p.x1[d + m] = p.x1[idx];
      p.x2[d + m] = p.x2[idx];
      p.x3[d + m] = p.x3[idx];
      p.p1[d + m] = pp;
      p.p2[d + m] = 0.0f;
      p.p3[d + m] = 0.0f;
      p.E[d + m] = ep;
      p.w[d + m] = p.w[idx];
      p.cell[d + m] = p.cell[idx];
      p.flag[d + m] = kFlagSecondary | ((uint32_t)m << 29);  // electron, then positron
      ids[d + m] = id_base + 2 * (uint64_t)r + (uint64_t)m;
    }
  }
}

__global__ void __launch_bounds__(kPairThreads)
    k_pair_mark(PairK K, PtcK p, const uint64_t *ids, const PairState *st, uint32_t step,
                uint8_t *emit, uint32_t *chunk_count, uint32_t nchunks) {
  const size_t number = st->number;
  for (uint32_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x)
    mark_chunk(K, p, ids, number, step, emit, chunk_count, ch);
}

__global__ void __launch_bounds__(1024)
    k_pair_scan(uint32_t *chunk_count, uint32_t nchunks, uint32_t *offs, size_t capacity,
                PairState *st, uint32_t *tot) {
  scan_chunks(chunk_count, nchunks, offs, capacity, st, tot);
}

__global__ void __launch_bounds__(kPairThreads)
    k_pair_append(PairK K, PtcK p, uint64_t *ids, const uint8_t *emit, const uint32_t *offs,
                  const uint32_t *tot, uint32_t nchunks) {
  int parity = 0;
  for (uint32_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x)
    parity += append_chunk(K, p, ids, emit, offs, tot, ch, parity) ? 1 : 0;
}

// Batched over 1D runs: work item g is chunk g - base[r] of run r.
__device__ __forceinline__ int run_of(const uint32_t *base, int nruns, uint32_t g) {
  int lo = 0, hi = nruns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (base[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ PairK pairk_of(const Run1D &R) {
  PairK K;
  K.gamma_thr = R.gamma_thr;
  K.free_path = R.free_path;
  K.pair_energy = R.pair_energy;
  K.dt = R.pair_dt;
  K.key[0] = R.key[0];
  K.key[1] = R.key[1];
  return K;
}

__global__ void __launch_bounds__(kPairThreads)
    k_b1_pair_mark(const Run1D *__restrict__ runs, const uint32_t *__restrict__ base, int nruns) {
  const uint32_t total = base[nruns];
  for (uint32_t g = blockIdx.x; g < total; g += gridDim.x) {
    const int r = run_of(base, nruns, g);
    const Run1D &R = runs[r];
    mark_chunk(pairk_of(R), R.p, R.ids, R.pst->number, R.step, R.emit, R.counts,
               g - base[r]);
  }
}

__global__ void __launch_bounds__(1024)
    k_b1_pair_scan(const Run1D *__restrict__ runs, const uint32_t *__restrict__ base) {
  const int r = blockIdx.x;
  const Run1D &R = runs[r];
  const uint32_t n = base[r + 1] - base[r];
  if (n == 0) return;
  scan_chunks(R.counts, n, R.offs, R.capacity, R.pst, R.tot);
}

__global__ void __launch_bounds__(kPairThreads)
    k_b1_pair_append(const Run1D *__restrict__ runs, const uint32_t *__restrict__ base,
                     int nruns) {
  const uint32_t total = base[nruns];
  int parity = 0;
  for (uint32_t g = blockIdx.x; g < total; g += gridDim.x) {
    const int r = run_of(base, nruns, g);
    const Run1D &R = runs[r];
    parity += append_chunk(pairk_of(R), R.p, R.ids, R.emit, R.offs, R.tot, g - base[r], parity)
                  ? 1
                  : 0;
  }
}

}  // namespace

int enqueue_pairs(Ctx &c, float dt, uint32_t step) {
  if (!c.pstate || c.capacity == 0) return AP_OK;
  // work over the capacity: the live count is only known on the device
  const uint32_t nchunks = pair_chunks_of(c);
  if (ensure_pair_scratch(c) != AP_OK) return AP_ERR_NOMEM;
  uint32_t *counts = c.pair_chunks, *offs = c.pair_chunks + c.pair_cap_chunks;
  uint32_t *tot = offs + c.pair_cap_chunks;
  PairK K;
  K.gamma_thr = c.pair.gamma_thr;
  K.free_path = c.pair.free_path;
  K.pair_energy = c.pair.pair_energy;
  K.dt = dt;
  K.key[0] = (uint32_t)c.pair.seed;
  K.key[1] = (uint32_t)(c.pair.seed >> 32);
  PtcK p{c.ptc.x1, c.ptc.x2, c.ptc.x3, c.ptc.p1, c.ptc.p2,
         c.ptc.p3, c.ptc.E,  c.ptc.weight, c.ptc.cell, c.ptc.flag};
  const uint32_t grid = nchunks < (uint32_t)c.num_sms * 8 ? nchunks : (uint32_t)c.num_sms * 8;
  k_pair_mark<<<grid, kPairThreads, 0, c.stream>>>(K, p, c.ptc.id, c.pstate, step, c.dir,
                                                   counts, nchunks);
  k_pair_scan<<<1, 1024, 0, c.stream>>>(counts, nchunks, offs, c.capacity, c.pstate, tot);
  k_pair_append<<<grid, kPairThreads, 0, c.stream>>>(K, p, c.ptc.id, c.dir, offs, tot, nchunks);
  c.launches += 3;
  c.number_stale = true;
  if (c.mk.dim == 2) c.order_valid = false;  // appended slots are in no tile list
  return cudaGetLastError() == cudaSuccess ? AP_OK : AP_ERR_CUDA;
}

cudaError_t launch_b1_pairs(cudaStream_t s, int num_sms, const Run1D *runs,
                            const uint32_t *base, int nruns, uint32_t total) {
  if (total == 0) return cudaSuccess;
  const uint32_t cap = (uint32_t)num_sms * 8;
  const uint32_t grid = total < cap ? total : cap;
  k_b1_pair_mark<<<grid, kPairThreads, 0, s>>>(runs, base, nruns);
  k_b1_pair_scan<<<nruns, 1024, 0, s>>>(runs, base);
  k_b1_pair_append<<<grid, kPairThreads, 0, s>>>(runs, base, nruns);
  return cudaGetLastError();
}

// Pair scratch of a context (chunk counts, offsets, totals) for its
// capacity; also used by the batched injection.
int ensure_pair_scratch(Ctx &c) {
  const uint32_t nchunks = (uint32_t)((c.capacity + kPairChunk - 1) / kPairChunk);
  if (nchunks + 4 <= c.pair_cap_chunks) return AP_OK;
  cudaFree(c.pair_chunks);
  c.pair_chunks = nullptr;
  const size_t cap = (size_t)nchunks + 64;
  if (cudaMalloc(&c.pair_chunks, sizeof(uint32_t) * (2 * cap + 8)) != cudaSuccess)
    return AP_ERR_NOMEM;
  // the mark pass adds into the counts, the scan resets them
  if (cudaMemset(c.pair_chunks, 0, sizeof(uint32_t) * (2 * cap + 8)) != cudaSuccess)
    return AP_ERR_CUDA;
  c.pair_cap_chunks = cap;
  return AP_OK;
}

uint32_t pair_chunks_of(const Ctx &c) {
  return (uint32_t)((c.capacity + kPairChunk - 1) / kPairChunk);
}

int refresh_number(Ctx *c) {
  if (!c->pstate || !c->number_stale) return AP_OK;
  cudaError_t e = cudaMemcpyAsync(c->pstate_host, c->pstate, sizeof(PairState),
                                  cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return AP_ERR_CUDA;
  c->number = c->pstate_host->number;
  c->number_stale = false;
  return AP_OK;
}

int push_number(Ctx *c) {
  if (!c->pstate) return AP_OK;
  const uint32_t n = (uint32_t)c->number;
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) e = cudaMemcpy(&c->pstate->number, &n, sizeof(n), cudaMemcpyHostToDevice);
  c->number_stale = false;
  return e == cudaSuccess ? AP_OK : AP_ERR_CUDA;
}

}  // namespace apb

// Particle ordering on the device.
//
// Per-step tile counting sort. The push/deposit kernel walks each tile's
// particles in the current (stable) tile order and records, per particle,
// the direction d in 0..8 of the tile it moved to (9 = gone) and per-tile
// direction counts. Because the input is grouped by tile and a particle
// only moves to one of its tile's eight neighbours, the stable counting
// sort by new tile reduces to:
//   k_tile_newcount / k_scan_counts / k_tile_groups: for each destination
//                   tile, sum the counts from its (up
//                   to nine) source tiles, scan to get tile offsets, and
//                   give each (source, direction) group its offset, sources
//                   taken in ascending tile index;
//   k_order_scatter for each source tile, rank particles within their
//                   direction group in order and write them to
//                   group offset + rank.
// The result equals a stable counting sort of the previous order by the new
// tile key (core/particle_base_impl.hpp:250-305 applied to tile keys).
//
// Full rebuild (after binding or external changes) and sort_by_cell
// (cuda/core/particle_base_impl.cu:435-487) use a stable LSD radix sort.
#include <cuda_runtime.h>

#include "ap_device.cuh"
#include "ap_internal.h"

namespace apb {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScatterThreads = 256;

struct TileTopo {
  int ntx, nty, ntiles, per0, per1;
};

// Source tile of destination (ux, uy) for direction (dx, dy) in -1..1, or
// -1 when it falls outside a non-periodic edge.
__device__ __forceinline__ int source_tile(const TileTopo &T, int ux, int uy, int dx, int dy) {
  int sx = ux - dx, sy = uy - dy;
  if (sx < 0) {
    if (!T.per0) return -1;
    sx += T.ntx;
  } else if (sx >= T.ntx) {
    if (!T.per0) return -1;
    sx -= T.ntx;
  }
  if (sy < 0) {
    if (!T.per1) return -1;
    sy += T.nty;
  } else if (sy >= T.nty) {
    if (!T.per1) return -1;
    sy -= T.nty;
  }
  return sx + sy * T.ntx;
}

// Gathers the (source tile, direction, count) triples of destination u,
// sorted by source tile index. Returns how many there are.
__device__ __forceinline__ int gather_sources(const TileTopo &T, const uint32_t *cnt, int u,
                                              int src[9], int dirv[9], uint32_t num[9]) {
  const int ux = u % T.ntx, uy = u / T.ntx;
  int n = 0;
  for (int dy = -1; dy <= 1; ++dy)
    for (int dx = -1; dx <= 1; ++dx) {
      const int s = source_tile(T, ux, uy, dx, dy);
      if (s < 0) continue;
      const int d = (dy + 1) * 3 + (dx + 1);
      // insertion by source index
      int k = n++;
      while (k > 0 && src[k - 1] > s) {
        src[k] = src[k - 1];
        dirv[k] = dirv[k - 1];
        num[k] = num[k - 1];
        --k;
      }
      src[k] = s;
      dirv[k] = d;
      num[k] = cnt[s * 10 + d];
    }
  return n;
}

// New population of every destination tile: the counts its (up to nine)
// source tiles recorded for the direction that leads to it.
__global__ void k_tile_newcount(TileTopo T, const uint32_t *__restrict__ cnt,
                                uint32_t *__restrict__ newcount) {
  for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < T.ntiles; u += gridDim.x * blockDim.x) {
    int src[9], dirv[9];
    uint32_t num[9];
    const int n = gather_sources(T, cnt, u, src, dirv, num);
    uint32_t nu = 0;
    for (int k = 0; k < n; ++k) nu += num[k];
    newcount[u] = nu;
  }
}

// Offsets of the (source, direction) groups inside each destination tile:
// sources in ascending tile index, so the concatenation is the stable order.
__global__ void k_tile_groups(TileTopo T, const uint32_t *__restrict__ cnt,
                              const uint32_t *__restrict__ new_start,
                              uint32_t *__restrict__ grp_off) {
  for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < T.ntiles; u += gridDim.x * blockDim.x) {
    int src[9], dirv[9];
    uint32_t num[9];
    const int n = gather_sources(T, cnt, u, src, dirv, num);
    uint32_t run = new_start[u];
    for (int k = 0; k < n; ++k) {
      grp_off[src[k] * 9 + dirv[k]] = run;
      run += num[k];
    }
  }
}

// One CTA per source tile: stable rank within each direction group. The
// tile's list is cut into one contiguous segment per warp; pass 1 counts the
// directions of each segment (each lane adds its entries into packed
// per-direction counters, summed over the warp at the end), one barrier
// turns the counts into per-warp offsets, and pass 2 walks the segment
// again 32 entries at a time, ranking lanes that share a direction (a
// ballot for the entries that stay in the tile, nearly all of them;
// __match_any_sync for the rest), so every entry lands at group offset +
// entries of that direction before it. Both passes issue the loads of four
// 32-entry steps before using them.
__global__ void __launch_bounds__(kScatterThreads)
    k_order_scatter(int ntiles, const uint32_t *__restrict__ old_start,
                    const uint32_t *__restrict__ old_order, const uint8_t *__restrict__ dir,
                    const uint32_t *__restrict__ grp_off, uint32_t *__restrict__ new_order,
                    uint32_t capacity, uint32_t slot0, const uint32_t *__restrict__ tile_list,
                    DevStatus *status) {
  constexpr int kWarps = kScatterThreads / 32;
  constexpr int kU = 4;  // 32-entry steps per batch of loads
  __shared__ uint32_t s_cnt[kWarps][10];
  __shared__ uint32_t s_base[kWarps][10];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  // all tiles, or the count and indices in tile_list
  const int nlist = tile_list ? (int)tile_list[0] : ntiles;
  for (int li = blockIdx.x; li < nlist; li += gridDim.x) {
    const int s = tile_list ? (int)tile_list[1 + li] : li;
    const uint32_t b = old_start[s], e = old_start[s + 1];
    const uint32_t n = e - b;
    const uint32_t seg = ((n + kWarps * 32 - 1) / (kWarps * 32)) * 32;
    const uint32_t w0 = b + min(n, warp * seg), w1 = b + min(n, (warp + 1) * seg);
    // pass 1: direction counts of this warp's segment; packed counters of
    // 16 bits, directions 0-3 in c0, 4-7 in c1, 8-9 in c2, summed over the
    // warp into lane f's mycnt every 256 batches (at most 32 x 4 x 256 =
    // 32768 entries per counter in between)
    unsigned long long c0 = 0, c1 = 0, c2 = 0;
    uint32_t mycnt = 0;  // lane f < 10: count of direction f
    auto flush = [&]() {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        c0 += __shfl_xor_sync(0xffffffffu, c0, o);
        c1 += __shfl_xor_sync(0xffffffffu, c1, o);
        c2 += __shfl_xor_sync(0xffffffffu, c2, o);
      }
      const unsigned long long w = lane < 4 ? c0 : (lane < 8 ? c1 : c2);
      if (lane < 10) mycnt += (uint32_t)((w >> (16 * (lane & 3))) & 0xffffull);
      c0 = c1 = c2 = 0;
    };
    int batches = 0;
    for (uint32_t q = w0; q < w1; q += 32 * kU) {
      if (++batches == 256) {
        flush();
        batches = 0;
      }
      uint32_t d[kU];
#pragma unroll
      for (int k = 0; k < kU; ++k) {
        const uint32_t p = q + 32 * k + lane;
        d[k] = p < w1 ? dir[p] : 10u;
      }
#pragma unroll
      for (int k = 0; k < kU; ++k) {
        const unsigned long long one = 1ull << (16 * (d[k] & 3u));
        if (d[k] < 4u)
          c0 += one;
        else if (d[k] < 8u)
          c1 += one;
        else if (d[k] < 10u)
          c2 += one;
      }
    }
    flush();
    if (lane < 10) s_cnt[warp][lane] = mycnt;
    __syncthreads();
    if (lane < 9) {
      uint32_t off = grp_off[s * 9 + lane];
      for (int w = 0; w < warp; ++w) off += s_cnt[w][lane];
      s_base[warp][lane] = off;
    }
    __syncwarp();
    // pass 2: stable placement
    uint32_t base4 = s_base[warp][4];
    for (uint32_t q = w0; q < w1; q += 32 * kU) {
      uint32_t d[kU], src[kU];
#pragma unroll
      for (int k = 0; k < kU; ++k) {
        const uint32_t p = q + 32 * k + lane;
        d[k] = p < w1 ? dir[p] : 10u;
        // no old order (after a compacting push): the particle at list
        // position p sits in slot slot0 + p
        src[k] = p < w1 ? (old_order ? old_order[p] : slot0 + p) : 0u;
      }
#pragma unroll
      for (int k = 0; k < kU; ++k) {
        if (q + 32 * k >= w1) break;
        const uint32_t dk = d[k];
        const uint32_t stay = __ballot_sync(0xffffffffu, dk == 4u);
        const uint32_t other = __ballot_sync(0xffffffffu, dk < 9u && dk != 4u);
        uint32_t dst = 0xffffffffu;
        if (dk == 4u) dst = base4 + __popc(stay & lt);
        base4 += __popc(stay);
        if (other) {
          if ((other >> lane) & 1u) {
            const uint32_t peers = __match_any_sync(other, dk);
            const uint32_t bs = s_base[warp][dk];
            dst = bs + __popc(peers & lt);
            __syncwarp(other);
            if ((peers & lt) == 0u) s_base[warp][dk] = bs + __popc(peers);
          }
          __syncwarp();
        }
        if (dst != 0xffffffffu) {
          if (dst < capacity)
            new_order[dst] = src[k];
          else
            atomicAdd(&status->tile_faults, 1ull);
        }
      }
    }
    __syncthreads();
  }
}

// One pass of the same stable placement, using the per-chunk direction
// counts the push / deposit kernel recorded (chunk k of source tile s is
// list entries [k CH, (k + 1) CH) of the tile, its counts at entry
// old_start[s] / CH + s + k of chunk_count). The CTA turns them into the
// group offset of every (chunk, direction); warp w then places chunks w,
// w + 8, ... with the ballot / __match_any_sync ranking of pass 2 above.
// Tiles of more than kMaxChunks chunks take the two-pass kernel.
constexpr int kMaxChunks = 128;

__global__ void __launch_bounds__(kScatterThreads)
    k_order_scatter1(int ntiles, int ch, const uint32_t *__restrict__ old_start,
                     const uint32_t *__restrict__ old_order, const uint8_t *__restrict__ dir,
                     const uint32_t *__restrict__ chunk_count, const uint32_t *__restrict__ grp_off,
                     uint32_t *__restrict__ new_order, uint32_t capacity, uint32_t slot0,
                     uint32_t *__restrict__ big_tiles, DevStatus *status) {
  constexpr int kWarps = kScatterThreads / 32;
  constexpr int kU = 4;
  __shared__ uint32_t s_cb[kMaxChunks][9];  // group offset of each (chunk, direction)
  __shared__ uint32_t s_base[kWarps][9];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  for (int s = blockIdx.x; s < ntiles; s += gridDim.x) {
    const uint32_t b = old_start[s], e = old_start[s + 1];
    const uint32_t n = e - b;
    const int nch = (int)((n + ch - 1) / ch);
    if (nch > kMaxChunks) {  // left to the two-pass kernel
      if (tid == 0) big_tiles[1 + atomicAdd(big_tiles, 1u)] = (uint32_t)s;
      continue;
    }
    const size_t c0 = (size_t)(b / ch) + s;
    // the tile's chunk counts, loaded by all threads, then scanned per
    // direction in shared memory
    for (int i = tid; i < nch * 9; i += kScatterThreads)
      s_cb[i / 9][i % 9] = chunk_count[(c0 + i / 9) * 10 + i % 9];
    const uint32_t off = tid < 9 ? grp_off[s * 9 + tid] : 0u;
    __syncthreads();
    if (tid < 9) {
      uint32_t run = off;
      for (int k = 0; k < nch; ++k) {
        const uint32_t v = s_cb[k][tid];
        s_cb[k][tid] = run;
        run += v;
      }
    }
    __syncthreads();
    for (int k = warp; k < nch; k += kWarps) {
      if (lane < 9) s_base[warp][lane] = s_cb[k][lane];
      __syncwarp();
      uint32_t base4 = s_base[warp][4];
      const uint32_t w0 = b + (uint32_t)k * ch, w1 = min(e, w0 + ch);
      for (uint32_t q = w0; q < w1; q += 32 * kU) {
        uint32_t d[kU], src[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
          const uint32_t p = q + 32 * u + lane;
          d[u] = p < w1 ? dir[p] : 10u;
          src[u] = p < w1 ? (old_order ? old_order[p] : slot0 + p) : 0u;
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
          if (q + 32 * u >= w1) break;
          const uint32_t dk = d[u];
          const uint32_t stay = __ballot_sync(0xffffffffu, dk == 4u);
          const uint32_t other = __ballot_sync(0xffffffffu, dk < 9u && dk != 4u);
          uint32_t dst = 0xffffffffu;
          if (dk == 4u) dst = base4 + __popc(stay & lt);
          base4 += __popc(stay);
          if (other) {
            if ((other >> lane) & 1u) {
              const uint32_t peers = __match_any_sync(other, dk);
              const uint32_t bs = s_base[warp][dk];
              dst = bs + __popc(peers & lt);
              __syncwarp(other);
              if ((peers & lt) == 0u) s_base[warp][dk] = bs + __popc(peers);
            }
            __syncwarp();
          }
          if (dst != 0xffffffffu) {
            if (dst < capacity)
              new_order[dst] = src[u];
            else
              atomicAdd(&status->tile_faults, 1ull);
          }
        }
      }
      __syncwarp();
    }
    __syncthreads();
  }
}

// start[k] = first position of key k in the sorted keys[0, n), for
// k = 0..nbins (start[nbins] = position of the first key >= nbins); also the
// largest segment length over keys < nbins.
__global__ void k_segment_starts(const uint32_t *__restrict__ keys, size_t n, uint32_t nbins,
                                 uint32_t *__restrict__ start) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i <= n;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t prev = (i == 0) ? 0u : min(keys[i - 1], nbins) + 1u;  // first key not yet started
    const uint32_t cur = (i == n) ? nbins : min(keys[i], nbins);
    for (uint32_t k = prev; k <= cur; ++k) start[k] = (uint32_t)i;
  }
}

__global__ void __launch_bounds__(kScanThreads)
    k_segment_max(const uint32_t *__restrict__ start, uint32_t nbins, uint32_t *n_max) {
  __shared__ uint32_t s_max;
  if (threadIdx.x == 0) s_max = 0;
  __syncthreads();
  uint32_t mx = 0;
  for (uint32_t k = threadIdx.x; k < nbins; k += blockDim.x) mx = max(mx, start[k + 1] - start[k]);
  atomicMax(&s_max, mx);
  __syncthreads();
  if (threadIdx.x == 0) *n_max = s_max;
}

// Tile order of particles sorted by cell: the particles of tile t are, row
// by row, the contiguous runs [cell_start[first cell of the row], cell_start
// [one past the last cell]) -- which is the stable counting sort by tile of
// the cell-sorted array.
__global__ void k_tile_counts_from_cells(MeshK m, TilesK T, const uint32_t *__restrict__ cs,
                                         uint32_t *__restrict__ counts) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T.ntiles; t += gridDim.x * blockDim.x) {
    const int tx = t % T.ntx, ty = t / T.ntx;
    const int x0 = m.guard[0] + tx * T.tx;
    const int x1 = min(x0 + T.tx, m.dims[0] - m.guard[0]);
    const int y0 = m.guard[1] + ty * T.ty;
    const int y1 = min(y0 + T.ty, m.dims[1] - m.guard[1]);
    uint32_t n = 0;
    for (int y = y0; y < y1; ++y) n += cs[y * m.dims[0] + x1] - cs[y * m.dims[0] + x0];
    counts[t] = n;
  }
}

__global__ void k_tile_fill_from_cells(MeshK m, TilesK T, const uint32_t *__restrict__ cs,
                                       const uint32_t *__restrict__ tile_start,
                                       uint32_t *__restrict__ order, uint32_t slot0) {
  for (int t = blockIdx.x; t < T.ntiles; t += gridDim.x) {
    const int tx = t % T.ntx, ty = t / T.ntx;
    const int x0 = m.guard[0] + tx * T.tx;
    const int x1 = min(x0 + T.tx, m.dims[0] - m.guard[0]);
    const int y0 = m.guard[1] + ty * T.ty;
    const int y1 = min(y0 + T.ty, m.dims[1] - m.guard[1]);
    uint32_t out = tile_start[t];
    for (int y = y0; y < y1; ++y) {
      const uint32_t a = cs[y * m.dims[0] + x0], b = cs[y * m.dims[0] + x1];
      for (uint32_t i = a + threadIdx.x; i < b; i += blockDim.x) order[out + (i - a)] = slot0 + i;
      out += b - a;
    }
  }
}

// Keys for the full rebuild: tile of a bulk cell, ntiles otherwise; cells
// outside the bulk are emptied as the reference push does (ptc_updater.cu:
// 87-90).
// Keys of slots base + i, i < n (vals = the slots).
__global__ void k_tile_keys(MeshK m, TilesK T, uint32_t *cell, size_t base, size_t n,
                            uint32_t *keys, uint32_t *vals) {
  cell += base;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    uint32_t c = cell[i];
    uint32_t key = (uint32_t)T.ntiles;
    if (c != AP_MAX_CELL) {
      int c1 = (int)(c % (uint32_t)m.dims[0]);
      int c2 = (int)((c / (uint32_t)m.dims[0]) % (uint32_t)m.dims[1]);
      int c3 = (int)(c / ((uint32_t)m.dims[0] * (uint32_t)m.dims[1]));
      bool bulk = c1 >= m.guard[0] && c1 < m.dims[0] - m.guard[0] && c2 >= m.guard[1] &&
                  c2 < m.dims[1] - m.guard[1] && c3 >= m.guard[2] && c3 < m.dims[2] - m.guard[2];
      if (bulk) {
        int tx = (c1 - m.guard[0]) / T.tx;
        int ty = (m.dim > 1) ? (c2 - m.guard[1]) / T.ty : 0;
        key = (uint32_t)(tx + ty * T.ntx);
      } else {
        cell[i] = AP_MAX_CELL;
      }
    }
    keys[i] = key;
    vals[i] = (uint32_t)(base + i);
  }
}

// Exclusive scan of nbins counters into start[0..nbins] with one CTA.
__global__ void __launch_bounds__(kScanThreads)
    k_scan_counts(const uint32_t *counts, int nbins, uint32_t *start, uint32_t *n_max) {
  __shared__ uint32_t s_part[kScanThreads];
  __shared__ uint32_t s_max;
  const int tid = threadIdx.x;
  if (tid == 0) s_max = 0;
  const int per = (nbins + kScanThreads - 1) / kScanThreads;
  const int b0 = tid * per, b1 = min(nbins, b0 + per);
  uint32_t local = 0, mx = 0;
  for (int b = b0; b < b1; ++b) {
    local += counts[b];
    mx = max(mx, counts[b]);
  }
  s_part[tid] = local;
  __syncthreads();
  atomicMax(&s_max, mx);
  for (int off = 1; off < kScanThreads; off <<= 1) {
    uint32_t v = tid >= off ? s_part[tid - off] : 0u;
    __syncthreads();
    s_part[tid] += v;
    __syncthreads();
  }
  uint32_t run = s_part[tid] - local;
  for (int b = b0; b < b1; ++b) {
    start[b] = run;
    run += counts[b];
  }
  if (tid == kScanThreads - 1) start[nbins] = s_part[tid];
  __syncthreads();
  if (tid == 0 && n_max) *n_max = s_max;
}

// Keys of slots base + i, i < n (vals = the slots); slots at or beyond a
// device-side live count are empty.
__global__ void k_cell_keys(const uint32_t *cell, size_t base, size_t n, uint32_t ncells,
                            uint32_t *keys, uint32_t *vals, const uint32_t *d_number) {
  const size_t live = d_number ? (size_t)*d_number : base + n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t c = base + i < live ? cell[base + i] : AP_MAX_CELL;
    keys[i] = (c == AP_MAX_CELL) ? ncells : c;
    vals[i] = (uint32_t)(base + i);
  }
}

template <typename T>
__global__ void k_gather(const T *src, const uint32_t *perm, size_t n, T *dst) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    dst[i] = src[perm[i]];
}

int bits_for(uint32_t maxkey) {
  int b = 1;
  while (b < 32 && (maxkey >> b) != 0) ++b;
  return b;
}

int grid_for(Ctx &c, size_t n, int threads) {
  size_t g = (n + threads - 1) / threads;
  size_t cap = (size_t)c.num_sms * 16;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

// Stable radix sort of (keys[0], vals[0]) -> result pointers (k_radix.cu).
cudaError_t radix_pairs(Ctx &c, size_t n, int end_bit, uint32_t **keys_out,
                        uint32_t **vals_out) {
  return radix_sort_pairs(c, n, end_bit, keys_out, vals_out);
}

}  // namespace

cudaError_t launch_tile_scan(Ctx &c, const uint32_t *dir_count, uint32_t *new_start,
                             uint32_t *grp_off) {
  TileTopo T{c.tiles.ntx, c.tiles.nty, c.tiles.ntiles, c.params.periodic[0],
             c.params.periodic[1]};
  const int nt = c.tiles.ntiles;
  const int g = (nt + 255) / 256;
  k_tile_newcount<<<g, 256, 0, c.stream>>>(T, dir_count, c.newcount);
  k_scan_counts<<<1, kScanThreads, 0, c.stream>>>(c.newcount, nt, new_start, c.n_max);
  k_tile_groups<<<g, 256, 0, c.stream>>>(T, dir_count, new_start, grp_off);
  c.launches += 3;
  return cudaGetLastError();
}

cudaError_t launch_order_scatter(Ctx &c, const uint32_t *old_start, const uint32_t *old_order,
                                 const uint8_t *dir, const uint32_t *grp_off,
                                 uint32_t *new_order, uint32_t slot0) {
  int grid = c.tiles.ntiles < c.num_sms * 8 ? c.tiles.ntiles : c.num_sms * 8;
  if (!c.chunk_count_ok) {
    k_order_scatter<<<grid, kScatterThreads, 0, c.stream>>>(
        c.tiles.ntiles, old_start, old_order, dir, grp_off, new_order, (uint32_t)c.order_cap,
        slot0, nullptr, c.status);
    c.launches++;
    return cudaGetLastError();
  }
  // one pass from the push / deposit kernel's chunk counts; tiles of more
  // than kMaxChunks chunks are listed in big_tiles for the two-pass kernel
  cudaError_t e = cudaMemsetAsync(c.big_tiles, 0, sizeof(uint32_t), c.stream);
  if (e != cudaSuccess) return e;
  k_order_scatter1<<<grid, kScatterThreads, 0, c.stream>>>(
      c.tiles.ntiles, chunk_of(c), old_start, old_order, dir, c.chunk_count, grp_off, new_order,
      (uint32_t)c.order_cap, slot0, c.big_tiles, c.status);
  k_order_scatter<<<c.num_sms, kScatterThreads, 0, c.stream>>>(
      c.tiles.ntiles, old_start, old_order, dir, grp_off, new_order, (uint32_t)c.order_cap,
      slot0, c.big_tiles, c.status);
  c.launches += 2;
  return cudaGetLastError();
}

// Scratch for the radix sorts: two key and two value buffers of n entries,
// the per-CTA digit counts, and an 8-byte-per-slot gather buffer.
int ensure_scratch(Ctx &c, size_t n) {
  if (n <= c.scratch_cap && c.keys[0]) return AP_OK;
  for (int i = 0; i < 2; ++i) {
    cudaFree(c.keys[i]);
    cudaFree(c.vals[i]);
    c.keys[i] = c.vals[i] = nullptr;
  }
  cudaFree(c.rx_counts);
  cudaFree(c.gather_tmp);
  c.rx_counts = nullptr;
  c.gather_tmp = nullptr;
  size_t cap = n < 1024 ? 1024 : n;
  for (int i = 0; i < 2; ++i) {
    if (cudaMalloc(&c.keys[i], cap * sizeof(uint32_t)) != cudaSuccess) return AP_ERR_NOMEM;
    if (cudaMalloc(&c.vals[i], cap * sizeof(uint32_t)) != cudaSuccess) return AP_ERR_NOMEM;
  }
  if (cudaMalloc(&c.rx_counts, radix_count_words(c.num_sms) * sizeof(uint32_t)) != cudaSuccess)
    return AP_ERR_NOMEM;
  if (cudaMalloc(&c.gather_tmp, cap * sizeof(uint64_t)) != cudaSuccess) return AP_ERR_NOMEM;
  c.scratch_cap = cap;
  return AP_OK;
}

// After a compaction: the slots after the live ones are empty.
__global__ void k_compact_tail(const uint32_t *live, uint32_t *cell, size_t n) {
  const uint32_t m = *live;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    if (i >= m) cell[i] = AP_MAX_CELL;
}

namespace {

ap_particles store_layout(void *buf, size_t cap) {
  unsigned char *b = static_cast<unsigned char *>(buf);
  ap_particles s;
  s.id = reinterpret_cast<uint64_t *>(b);
  s.x1 = reinterpret_cast<float *>(b + 8 * cap);
  s.x2 = s.x1 + cap;
  s.x3 = s.x2 + cap;
  s.p1 = s.x3 + cap;
  s.p2 = s.p1 + cap;
  s.p3 = s.p2 + cap;
  s.E = s.p3 + cap;
  s.weight = s.E + cap;
  s.cell = reinterpret_cast<uint32_t *>(s.weight + cap);
  s.flag = s.cell + cap;
  return s;
}

}  // namespace

// The scratch store (48 B per slot, allocated on first use).
static cudaError_t compact_store_scratch(Ctx &c, PtcK *out, uint64_t **out_id) {
  const size_t n = c.capacity > c.number ? c.capacity : c.number;
  if (!c.compact_buf || c.compact_cap < n) {
    cudaFree(c.compact_buf);
    c.compact_buf = nullptr;
    cudaError_t e = cudaMalloc(&c.compact_buf, n * 48);
    if (e != cudaSuccess) return e;
    c.compact_cap = n;
  }
  const ap_particles s = store_layout(c.compact_buf, c.compact_cap);
  *out = PtcK{s.x1, s.x2, s.x3, s.p1, s.p2, s.p3, s.E, s.weight, s.cell, s.flag};
  *out_id = s.id;
  return cudaSuccess;
}

// Output of a compaction. When the caller's capacity leaves a free region
// as large as the occupied one ([store_base, number) holds every particle;
// the other half of the capacity is empty), the push writes the tile-ordered
// copy straight into it and the old region becomes empty slots; otherwise
// into the scratch store, copied back afterwards.
cudaError_t compact_store(Ctx &c, PtcK *out, uint64_t **out_id) {
  const size_t half = c.capacity / 2;
  const size_t used = c.number - c.store_base;
  if (c.store_base == 0 && c.number <= half) {
    c.compact_direct = true;
    c.compact_dst = half;
  } else if (c.store_base >= half && used <= c.store_base) {
    c.compact_direct = true;
    c.compact_dst = 0;
  } else {
    c.compact_direct = false;
    c.compact_dst = 0;
  }
  if (c.compact_direct) {
    const size_t d = c.compact_dst;
    *out = PtcK{c.ptc.x1 + d, c.ptc.x2 + d, c.ptc.x3 + d, c.ptc.p1 + d,  c.ptc.p2 + d,
                c.ptc.p3 + d, c.ptc.E + d,  c.ptc.weight + d, c.ptc.cell + d, c.ptc.flag + d};
    *out_id = c.ptc.id + d;
    return cudaSuccess;
  }
  return compact_store_scratch(c, out, out_id);
}

// After the order update of a compacting push: `live` (device) slots were
// written from compact_dst on. Direct output: the old region becomes empty
// and the new high-water mark is compact_dst + (number - store_base);
// scratch output: copied back to slots [0, number). Either way the slots
// between the written ones and the high-water mark become empty.
cudaError_t compact_finish(Ctx &c, const uint32_t *live) {
  const size_t n = c.number - c.store_base;
  if (n == 0) return cudaSuccess;
  cudaError_t e;
  if (c.compact_direct) {
    e = cudaMemsetAsync(c.ptc.cell + c.store_base, 0xff, n * sizeof(uint32_t), c.stream);
    if (e != cudaSuccess) return e;
  } else {
    const ap_particles s = store_layout(c.compact_buf, c.compact_cap);
    const struct {
      void *dst;
      const void *src;
      size_t bytes;
    } back[11] = {{c.ptc.x1, s.x1, 4}, {c.ptc.x2, s.x2, 4},         {c.ptc.x3, s.x3, 4},
                  {c.ptc.p1, s.p1, 4}, {c.ptc.p2, s.p2, 4},         {c.ptc.p3, s.p3, 4},
                  {c.ptc.E, s.E, 4},   {c.ptc.weight, s.weight, 4}, {c.ptc.cell, s.cell, 4},
                  {c.ptc.id, s.id, 8}, {c.ptc.flag, s.flag, 4}};
    for (const auto &m : back) {
      e = cudaMemcpyAsync(m.dst, m.src, n * m.bytes, cudaMemcpyDeviceToDevice, c.stream);
      if (e != cudaSuccess) return e;
    }
    if (c.store_base > 0) {
      e = cudaMemsetAsync(c.ptc.cell + n, 0xff, (c.number - n) * sizeof(uint32_t), c.stream);
      if (e != cudaSuccess) return e;
    }
  }
  k_compact_tail<<<grid_for(c, n, 256), 256, 0, c.stream>>>(live, c.ptc.cell + c.compact_dst, n);
  c.launches++;
  c.number = c.compact_dst + n;
  c.store_base = c.compact_dst;
  return cudaGetLastError();
}

// Builds the tile order from scratch: stable sort of slots
// [store_base, number) by tile key, then tile offsets from a histogram.
cudaError_t rebuild_tile_order(Ctx &c) {
  const size_t n = c.number - c.store_base;
  const uint32_t nt = (uint32_t)c.tiles.ntiles;
  uint32_t *start = c.tile_start[c.cur];
  cudaError_t e;
  if (n > 0) {
    k_tile_keys<<<grid_for(c, n, 256), 256, 0, c.stream>>>(c.mk, c.tiles, c.ptc.cell,
                                                          c.store_base, n, c.keys[0],
                                                          c.vals[0]);
    c.launches++;
    uint32_t *ko, *vo;
    e = radix_pairs(c, n, bits_for(nt), &ko, &vo);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(c.order[c.cur], vo, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                        c.stream);
    if (e != cudaSuccess) return e;
    k_segment_starts<<<grid_for(c, n + 1, 256), 256, 0, c.stream>>>(ko, n, nt, start);
    c.launches++;
  } else {
    e = cudaMemsetAsync(start, 0, sizeof(uint32_t) * (nt + 1), c.stream);
    if (e != cudaSuccess) return e;
  }
  k_segment_max<<<1, kScanThreads, 0, c.stream>>>(start, nt, c.n_max);
  c.launches++;
  c.order_valid = true;
  return cudaGetLastError();
}

namespace {


// Tile-order derived from the cell starts of a store sorted into slots
// [slot0, slot0 + live).
cudaError_t tile_order_from_cells(Ctx &c, uint32_t slot0) {
  const int nt = c.tiles.ntiles;
  k_tile_counts_from_cells<<<(nt + 255) / 256, 256, 0, c.stream>>>(c.mk, c.tiles, c.cell_start,
                                                                   c.dir_count);
  k_scan_counts<<<1, kScanThreads, 0, c.stream>>>(c.dir_count, nt, c.tile_start[c.cur], c.n_max);
  k_tile_fill_from_cells<<<nt < c.num_sms * 8 ? nt : c.num_sms * 8, 256, 0, c.stream>>>(
      c.mk, c.tiles, c.cell_start, c.tile_start[c.cur], c.order[c.cur], slot0);
  c.launches += 3;
  c.order_valid = true;
  return cudaGetLastError();
}

}  // namespace

cudaError_t sort_by_cell(Ctx &c, size_t *new_number) {
  // a 1D context with a device-side count (pair injection) sorts over its
  // capacity and writes the new count on the device; a 2D store after a
  // compaction into the upper half sorts slots [store_base, number)
  c.order_valid = false;
  const bool device_count = c.pstate && c.mk.dim == 1;
  const size_t base = device_count ? 0 : c.store_base;
  const size_t n = (device_count ? c.capacity : c.number) - base;
  *new_number = 0;
  if (n == 0) {
    c.store_base = 0;
    return cudaSuccess;
  }
  const uint32_t ncells =
      (uint32_t)c.mesh.dims[0] * (uint32_t)c.mesh.dims[1] * (uint32_t)c.mesh.dims[2];
  k_cell_keys<<<grid_for(c, n, 256), 256, 0, c.stream>>>(c.ptc.cell, base, n, ncells, c.keys[0],
                                                        c.vals[0],
                                                        device_count ? &c.pstate->number
                                                                     : nullptr);
  c.launches++;
  uint32_t *ko, *vo;
  cudaError_t e = radix_pairs(c, n, bits_for(ncells), &ko, &vo);
  if (e != cudaSuccess) return e;
  const int g = grid_for(c, n, 256);
  // With compaction on and a free half of the capacity, each member is
  // gathered straight into that half (the store then occupies
  // [out0, out0 + live)); otherwise through the gather buffer and back to
  // slots [0, live) (cuda/core/particle_base_impl.cu:466-487). One member at
  // a time: the random reads of one array stay in L2, those of eleven at once
  // do not.
  const size_t half = c.capacity / 2;
  size_t out0 = 0;
  bool direct = false;
  if (!device_count && c.compact_interval > 0) {
    if (c.store_base == 0 && c.number <= half) {
      direct = true;
      out0 = half;
    } else if (c.store_base >= half && n <= c.store_base) {
      direct = true;
      out0 = 0;
    }
  }
#define AP_GATHER(FIELD, T)                                                                  \
  do {                                                                                        \
    if (direct) {                                                                             \
      k_gather<T><<<g, 256, 0, c.stream>>>(c.ptc.FIELD, vo, n, (T *)c.ptc.FIELD + out0);      \
    } else {                                                                                  \
      k_gather<T><<<g, 256, 0, c.stream>>>(c.ptc.FIELD, vo, n, (T *)c.gather_tmp);           \
      e = cudaMemcpyAsync(c.ptc.FIELD, c.gather_tmp, n * sizeof(T), cudaMemcpyDeviceToDevice, \
                          c.stream);                                                          \
      if (e != cudaSuccess) return e;                                                         \
    }                                                                                         \
    c.launches++;                                                                             \
  } while (0)
  AP_GATHER(x1, float);
  AP_GATHER(x2, float);
  AP_GATHER(x3, float);
  AP_GATHER(p1, float);
  AP_GATHER(p2, float);
  AP_GATHER(p3, float);
  AP_GATHER(E, float);
  AP_GATHER(weight, float);
  AP_GATHER(cell, uint32_t);
  AP_GATHER(id, uint64_t);
  AP_GATHER(flag, uint32_t);
#undef AP_GATHER
  if (direct && out0 > 0) {  // the old particles sat below the new range: empty them
    e = cudaMemsetAsync(c.ptc.cell, 0xff, c.number * sizeof(uint32_t), c.stream);
    if (e != cudaSuccess) return e;
  }
  // cell_start over the sorted keys; cell_start[ncells] is the number of
  // non-empty slots (upper_bound of MAX_CELL - 1, particle_base_impl.cu:454-458)
  if (!c.cell_start) {
    e = cudaMalloc(&c.cell_start, sizeof(uint32_t) * ((size_t)ncells + 1));
    if (e != cudaSuccess) return e;
  }
  k_segment_starts<<<grid_for(c, n + 1, 256), 256, 0, c.stream>>>(ko, n, ncells, c.cell_start);
  c.launches++;
  if (device_count) {
    c.number_stale = true;
    return cudaMemcpyAsync(&c.pstate->number, c.cell_start + ncells, sizeof(uint32_t),
                           cudaMemcpyDeviceToDevice, c.stream);
  }
  uint32_t live = 0;
  e = cudaMemcpyAsync(&live, c.cell_start + ncells, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                      c.stream);
  if (e != cudaSuccess) return e;
  if (c.mk.dim == 2) {
    // the tile order of the cell-sorted particles, without another sort
    e = tile_order_from_cells(c, (uint32_t)out0);
    if (e != cudaSuccess) return e;
  }
  e = cudaStreamSynchronize(c.stream);
  if (e != cudaSuccess) return e;
  c.store_base = out0;
  *new_number = out0 + live;
  return cudaSuccess;
}

// photons.sort_by_cell (sim_data_impl.hpp:81; particle_base_impl.cu:435-487
// for photon_data): the same stable sort of the photon slots [0, number),
// each of the twelve members gathered through the scratch buffer, and the
// empty slots trimmed.
cudaError_t sort_photons(Ctx &c, size_t *new_number) {
  const size_t n = c.ph_number;
  *new_number = 0;
  if (n == 0) return cudaSuccess;
  if (ensure_scratch(c, n) != AP_OK) return cudaErrorMemoryAllocation;
  const uint32_t ncells =
      (uint32_t)c.mesh.dims[0] * (uint32_t)c.mesh.dims[1] * (uint32_t)c.mesh.dims[2];
  k_cell_keys<<<grid_for(c, n, 256), 256, 0, c.stream>>>(c.ph.cell, 0, n, ncells, c.keys[0],
                                                        c.vals[0], nullptr);
  c.launches++;
  uint32_t *ko, *vo;
  cudaError_t e = radix_pairs(c, n, bits_for(ncells), &ko, &vo);
  if (e != cudaSuccess) return e;
  const int g = grid_for(c, n, 256);
#define AP_GATHER_PH(FIELD, T)                                                                \
  do {                                                                                        \
    k_gather<T><<<g, 256, 0, c.stream>>>(c.ph.FIELD, vo, n, (T *)c.gather_tmp);               \
    e = cudaMemcpyAsync(c.ph.FIELD, c.gather_tmp, n * sizeof(T), cudaMemcpyDeviceToDevice,    \
                        c.stream);                                                            \
    if (e != cudaSuccess) return e;                                                           \
    c.launches++;                                                                             \
  } while (0)
  AP_GATHER_PH(x1, float);
  AP_GATHER_PH(x2, float);
  AP_GATHER_PH(x3, float);
  AP_GATHER_PH(p1, float);
  AP_GATHER_PH(p2, float);
  AP_GATHER_PH(p3, float);
  AP_GATHER_PH(E, float);
  AP_GATHER_PH(weight, float);
  AP_GATHER_PH(path_left, float);
  AP_GATHER_PH(cell, uint32_t);
  AP_GATHER_PH(id, uint64_t);
  AP_GATHER_PH(flag, uint32_t);
#undef AP_GATHER_PH
  if (!c.cell_start) {
    e = cudaMalloc(&c.cell_start, sizeof(uint32_t) * ((size_t)ncells + 1));
    if (e != cudaSuccess) return e;
  }
  k_segment_starts<<<grid_for(c, n + 1, 256), 256, 0, c.stream>>>(ko, n, ncells, c.cell_start);
  c.launches++;
  uint32_t live = 0;
  e = cudaMemcpyAsync(&live, c.cell_start + ncells, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                      c.stream);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(c.stream);
  if (e != cudaSuccess) return e;
  *new_number = live;
  return cudaSuccess;
}

}  // namespace apb

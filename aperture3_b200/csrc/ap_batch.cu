// Batched mode: many independent 2D Cartesian runs advanced together.
//
// Each run is an ordinary context. A step of the batch enqueues, on one
// stream and without host synchronisation: each run's zeroing (and tile
// order rebuild when needed), ONE persistent push / deposit launch per
// group of runs that share a tile shape, chunk and field-load path (CTAs
// draw (run, tile) items from one queue over all the group's tiles, so
// small runs fill the GPU together), then each run's order update and
// current finalize. The per-run kernel parameters and tensor maps go to
// the device as an array of RunDesc through a double-buffered pinned
// staging area.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <new>
#include <tuple>
#include <vector>

#include "ap_internal.h"

using namespace apb;

struct ap_ctx : public apb::Ctx {};

namespace {

struct Group {
  int dim;
  int tx, ty, chunk;
  bool tma;
  std::vector<int> members;  // indices into the batch's runs
};

// Work items of a run in a batched launch: tiles (2D) or chunks of
// particle slots (1D).
uint32_t work_items(const Ctx *c) {
  if (c->mk.dim == 1) {
    // with a device-side count the kernel covers the capacity
    const size_t n = c->pstate ? c->capacity : c->number;
    return (uint32_t)((n + kChunk1DSlots - 1) / kChunk1DSlots);
  }
  return (uint32_t)c->tiles.ntiles;
}

}  // namespace

struct ap_batch {
  std::vector<Ctx *> runs;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 148;
  // staging: RunDesc[nruns] then base[nruns + 2 * groups] per slot
  unsigned char *h_stage[2] = {nullptr, nullptr};
  cudaEvent_t stage_ev[2] = {nullptr, nullptr};
  int slot = 0;
  unsigned char *d_stage = nullptr;
  size_t stage_bytes = 0;
  size_t cap_runs = 0;  // runs the staging buffers hold
  uint32_t *queue = nullptr;
  // staging ring for the descriptors of the batched 1D launches
  struct Slot {
    unsigned char *h = nullptr, *d = nullptr;
    size_t cap = 0;
    cudaEvent_t ev = nullptr;
  };
  Slot ring[8];
  int ring_next = 0;
  // graph capture (ap_batch_set_capture): every staging copy comes from its
  // own host / device block, kept until the mode is turned off
  bool capture = false;
  std::vector<unsigned char *> arena_h, arena_d;
  // autotuning: time the push / deposit per class when set
  bool tuning = false;
  std::vector<int> tune_class;   // class of each run
  std::vector<float> tune_ms;    // per class, last step
  std::vector<cudaEvent_t> tune_ev;
};

namespace {

void free_arena(ap_batch *b) {
  for (unsigned char *h : b->arena_h) cudaFreeHost(h);
  for (unsigned char *d : b->arena_d) cudaFree(d);
  b->arena_h.clear();
  b->arena_d.clear();
}

void release(ap_batch *b) {
  if (b->stream) cudaStreamSynchronize(b->stream);
  free_arena(b);
  for (int i = 0; i < 2; ++i) {
    if (b->h_stage[i]) cudaFreeHost(b->h_stage[i]);
    if (b->stage_ev[i]) cudaEventDestroy(b->stage_ev[i]);
  }
  cudaFree(b->d_stage);
  cudaFree(b->queue);
  for (cudaEvent_t e : b->tune_ev) cudaEventDestroy(e);
  for (auto &s : b->ring) {
    if (s.h) cudaFreeHost(s.h);
    cudaFree(s.d);
    if (s.ev) cudaEventDestroy(s.ev);
  }
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
}

std::vector<Group> make_groups(const ap_batch *b, const std::vector<bool> &active,
                               const std::vector<int> *only_class, int cls) {
  std::map<std::tuple<int, int, int, int, bool>, int> idx;
  std::vector<Group> gs;
  for (int r = 0; r < (int)b->runs.size(); ++r) {
    if (!active[r]) continue;
    if (only_class && (*only_class)[r] != cls) continue;
    const Ctx *c = b->runs[r];
    const int dim = c->mk.dim;
    const int chunk = dim == 1 ? kChunk1DSlots : chunk_of(*c);
    const int tx = dim == 1 ? 0 : c->tiles.tx, ty = dim == 1 ? 0 : c->tiles.ty;
    const bool tma = dim == 1 ? false : c->use_tma;
    auto key = std::make_tuple(dim, tx, ty, chunk, tma);
    auto it = idx.find(key);
    if (it == idx.end()) {
      idx[key] = (int)gs.size();
      gs.push_back(Group{dim, tx, ty, chunk, tma, {}});
      it = idx.find(key);
    }
    gs[it->second].members.push_back(r);
  }
  return gs;
}

int fail_cuda(cudaError_t e) {
  return e == cudaErrorMemoryAllocation ? AP_ERR_NOMEM : AP_ERR_CUDA;
}

#define B_TRY(expr)                                 \
  do {                                              \
    cudaError_t _e = (expr);                        \
    if (_e != cudaSuccess) return fail_cuda(_e);    \
  } while (0)

#define B_TRY_ST(expr)               \
  do {                               \
    int _s = (expr);                 \
    if (_s != AP_OK) return _s;      \
  } while (0)

// Copies `bytes` from src to a device staging slot, in stream order; the
// slot's host buffer is reused only after its previous copy completed.
// A host / device block pair of the capture arena.
int arena_block(ap_batch *b, size_t bytes, unsigned char **h, unsigned char **d) {
  *h = *d = nullptr;
  B_TRY(cudaMallocHost(reinterpret_cast<void **>(h), bytes));
  b->arena_h.push_back(*h);
  B_TRY(cudaMalloc(reinterpret_cast<void **>(d), bytes));
  b->arena_d.push_back(*d);
  return AP_OK;
}

int stage(ap_batch *b, const void *src, size_t bytes, const unsigned char **dptr) {
  if (b->capture) {
    unsigned char *h, *d;
    B_TRY_ST(arena_block(b, bytes, &h, &d));
    std::memcpy(h, src, bytes);
    B_TRY(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, b->stream));
    *dptr = d;
    return AP_OK;
  }
  auto &s = b->ring[b->ring_next];
  b->ring_next = (b->ring_next + 1) % 8;
  if (!s.ev) B_TRY(cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming));
  else B_TRY(cudaEventSynchronize(s.ev));
  if (bytes > s.cap) {
    B_TRY(cudaStreamSynchronize(b->stream));
    if (s.h) cudaFreeHost(s.h);
    cudaFree(s.d);
    s.h = s.d = nullptr;
    s.cap = 0;
    const size_t cap = bytes * 2 > 4096 ? bytes * 2 : 4096;
    B_TRY(cudaMallocHost(reinterpret_cast<void **>(&s.h), cap));
    B_TRY(cudaMalloc(reinterpret_cast<void **>(&s.d), cap));
    s.cap = cap;
  }
  std::memcpy(s.h, src, bytes);
  B_TRY(cudaMemcpyAsync(s.d, s.h, bytes, cudaMemcpyHostToDevice, b->stream));
  B_TRY(cudaEventRecord(s.ev, b->stream));
  *dptr = s.d;
  return AP_OK;
}

// Stages 1D run descriptors followed by their work-item offsets (items[r]
// per run) and returns the device addresses and the total.
int stage_run1d(ap_batch *b, const std::vector<Run1D> &d, const std::vector<uint32_t> &items,
                const Run1D **dd, const uint32_t **db, uint32_t *total) {
  const size_t n = d.size();
  std::vector<unsigned char> buf(sizeof(Run1D) * n + sizeof(uint32_t) * (n + 1));
  std::memcpy(buf.data(), d.data(), sizeof(Run1D) * n);
  uint32_t *base = reinterpret_cast<uint32_t *>(buf.data() + sizeof(Run1D) * n);
  uint32_t t = 0;
  for (size_t r = 0; r < n; ++r) {
    base[r] = t;
    t += items[r];
  }
  base[n] = t;
  const unsigned char *dp = nullptr;
  B_TRY_ST(stage(b, buf.data(), buf.size(), &dp));
  *dd = reinterpret_cast<const Run1D *>(dp);
  *db = reinterpret_cast<const uint32_t *>(dp + sizeof(Run1D) * n);
  *total = t;
  return AP_OK;
}

bool is_1d(const Ctx *c) { return c->mk.dim == 1 && c->coord == 0; }

// Launches the push / deposit of the given groups from staged descriptors.
int launch_groups(ap_batch *b, const std::vector<Group> &gs,
                  const std::vector<PushDepositParams> &P, bool do_rho) {
  if (gs.empty()) return AP_OK;
  const int s = b->slot;
  const size_t nr = b->cap_runs;
  unsigned char *hblk = nullptr, *dblk = b->d_stage;
  if (b->capture) {
    B_TRY_ST(arena_block(b, b->stage_bytes, &hblk, &dblk));
  } else {
    b->slot ^= 1;
    B_TRY(cudaEventSynchronize(b->stage_ev[s]));  // the copy that last used this slot is done
    hblk = b->h_stage[s];
  }
  RunDesc *hd = reinterpret_cast<RunDesc *>(hblk);
  uint32_t *hbase = reinterpret_cast<uint32_t *>(hblk + sizeof(RunDesc) * nr);
  size_t k = 0, kb = 0;
  std::vector<size_t> desc_off, base_off;
  std::vector<uint32_t> totals;
  std::vector<int> max_sp;
  for (const Group &g : gs) {
    desc_off.push_back(k);
    base_off.push_back(kb);
    uint32_t total = 0;
    int msp = 1;
    for (int r : g.members) {
      hbase[kb++] = total;
      std::memcpy(&hd[k].maps, &b->runs[r]->maps, sizeof(FieldMaps));
      hd[k].P = P[r];
      total += work_items(b->runs[r]);
      msp = std::max(msp, b->runs[r]->params.num_species);
      ++k;
    }
    hbase[kb++] = total;
    totals.push_back(total);
    max_sp.push_back(msp);
  }
  B_TRY(cudaMemcpyAsync(dblk, hblk, sizeof(RunDesc) * k, cudaMemcpyHostToDevice, b->stream));
  B_TRY(cudaMemcpyAsync(dblk + sizeof(RunDesc) * nr, hblk + sizeof(RunDesc) * nr,
                        sizeof(uint32_t) * kb, cudaMemcpyHostToDevice, b->stream));
  if (!b->capture) B_TRY(cudaEventRecord(b->stage_ev[s], b->stream));
  const RunDesc *dd = reinterpret_cast<const RunDesc *>(dblk);
  const uint32_t *db = reinterpret_cast<const uint32_t *>(dblk + sizeof(RunDesc) * nr);
  for (size_t gi = 0; gi < gs.size(); ++gi) {
    const Group &g = gs[gi];
    if (g.dim == 1)
      B_TRY(launch_push_deposit_1d_batch(b->stream, b->num_sms, do_rho, dd + desc_off[gi],
                                         db + base_off[gi], (int)g.members.size(), totals[gi]));
    else
      B_TRY(launch_push_deposit_2d_batch(b->stream, b->num_sms, g.tx, g.ty, g.chunk, g.tma,
                                         do_rho, max_sp[gi], dd + desc_off[gi],
                                         db + base_off[gi], (int)g.members.size(), totals[gi],
                                         b->queue));
    for (int r : g.members) {
      b->runs[r]->launches++;
      b->runs[r]->pd_launches++;
    }
  }
  return AP_OK;
}

int batch_update(ap_batch *b, const double *dt, const uint32_t *steps) {
  const size_t n = b->runs.size();
  std::vector<PushDepositParams> P(n);
  std::vector<bool> work(n, false);
  bool do_rho = false;
  // 1D runs: accumulator clearing and finalize are batched launches
  std::vector<Run1D> d1;
  std::vector<uint32_t> zero_items, fin_items;
  std::vector<int> idx1;
  for (size_t r = 0; r < n; ++r) {
    Ctx *c = b->runs[r];
    bool w = false;
    const bool one = is_1d(c);
    B_TRY_ST(update_prepare(c, dt[r], steps[r], P[r], &w, one));
    if (one) {
      Run1D d;
      B_TRY_ST(fill_run1d(c, dt[r], steps[r], d));
      d1.push_back(d);
      zero_items.push_back(
          (uint32_t)(((size_t)d.zero_comps * d.acc_comp + 255) / 256));
      fin_items.push_back((uint32_t)((d.n0 + 255) / 256));
      idx1.push_back((int)r);
    }
    work[r] = w;
    // one kernel variant for all: charge deposition when any run needs it
    // (runs without it skip the charge terms through P.do_rho)
    do_rho = do_rho || ((steps[r] + 1) % (uint32_t)c->params.data_interval) == 0;
  }
  const Run1D *dd = nullptr;
  const uint32_t *db = nullptr;
  uint32_t tot = 0;
  if (!d1.empty()) {
    B_TRY_ST(stage_run1d(b, d1, zero_items, &dd, &db, &tot));
    B_TRY(launch_b1_zero(b->stream, b->num_sms, dd, db, (int)d1.size(), tot));
  }
  if (!b->tuning) {
    B_TRY_ST(launch_groups(b, make_groups(b, work, nullptr, 0), P, do_rho));
  } else {
    const int ncls = (int)b->tune_ms.size();
    for (int cl = 0; cl < ncls; ++cl) {
      auto gs = make_groups(b, work, &b->tune_class, cl);
      B_TRY(cudaEventRecord(b->tune_ev[2 * cl], b->stream));
      B_TRY_ST(launch_groups(b, gs, P, do_rho));
      B_TRY(cudaEventRecord(b->tune_ev[2 * cl + 1], b->stream));
    }
    B_TRY(cudaStreamSynchronize(b->stream));
    for (int cl = 0; cl < ncls; ++cl) {
      float ms = 0.0f;
      B_TRY(cudaEventElapsedTime(&ms, b->tune_ev[2 * cl], b->tune_ev[2 * cl + 1]));
      b->tune_ms[cl] = ms;
    }
  }
  for (size_t r = 0; r < n; ++r)
    B_TRY_ST(update_complete(b->runs[r], dt[r], steps[r], work[r], is_1d(b->runs[r])));
  if (!d1.empty()) {
    B_TRY_ST(stage_run1d(b, d1, fin_items, &dd, &db, &tot));
    B_TRY(launch_b1_finalize(b->stream, b->num_sms, dd, db, (int)d1.size(), tot));
    for (size_t k = 0; k < idx1.size(); ++k) {
      Ctx *c = b->runs[idx1[k]];
      if (c->params.current_smoothing > 0) B_TRY_ST(update_smooth(c, steps[idx1[k]]));
      c->launches += 2;
    }
  }
  return AP_OK;
}

bool run_ok(const ap_ctx *c) {
  return c && c->mk.dim <= 2 && c->coord == 0 && c->fields_bound && c->ptc_bound;
}

// Staging for up to n runs (descriptors and work-item offsets), grown
// geometrically; waits for the stream before replacing buffers.
int ensure_stage(ap_batch *b, size_t n) {
  if (n <= b->cap_runs) return AP_OK;
  size_t cap = b->cap_runs ? b->cap_runs : 8;
  while (cap < n) cap *= 2;
  if (b->stream) B_TRY(cudaStreamSynchronize(b->stream));
  const size_t bytes = sizeof(RunDesc) * cap + sizeof(uint32_t) * (2 * cap + 2);
  for (int i = 0; i < 2; ++i) {
    if (b->h_stage[i]) cudaFreeHost(b->h_stage[i]);
    b->h_stage[i] = nullptr;
    B_TRY(cudaMallocHost(reinterpret_cast<void **>(&b->h_stage[i]), bytes));
  }
  cudaFree(b->d_stage);
  b->d_stage = nullptr;
  B_TRY(cudaMalloc(reinterpret_cast<void **>(&b->d_stage), bytes));
  b->stage_bytes = bytes;
  b->cap_runs = cap;
  return AP_OK;
}

void adopt(ap_batch *b, ap_ctx *c) {
  b->runs.push_back(c);
  ap_set_stream(c, b->stream);
  c->sync = false;
}

}  // namespace

extern "C" {

AP_API int ap_batch_create(ap_ctx *const *runs, int nruns, ap_batch **out) {
  if ((nruns > 0 && !runs) || nruns < 0 || !out) return AP_ERR_INVALID;
  *out = nullptr;
  for (int r = 0; r < nruns; ++r) {
    if (!run_ok(runs[r])) return AP_ERR_INVALID;
    for (int q = 0; q < r; ++q)
      if (runs[q] == runs[r]) return AP_ERR_INVALID;
  }
  ap_batch *b = new (std::nothrow) ap_batch();
  if (!b) return AP_ERR_NOMEM;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, dev);
  bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess;
  b->own_stream = ok;
  for (int i = 0; i < 2 && ok; ++i)
    ok = cudaEventCreateWithFlags(&b->stage_ev[i], cudaEventDisableTiming) == cudaSuccess &&
         cudaEventRecord(b->stage_ev[i], b->stream) == cudaSuccess;
  ok = ok && cudaMalloc(reinterpret_cast<void **>(&b->queue), 16) == cudaSuccess &&
       ensure_stage(b, nruns > 8 ? nruns : 8) == AP_OK;
  if (!ok) {
    release(b);
    delete b;
    return AP_ERR_NOMEM;
  }
  for (int r = 0; r < nruns; ++r) adopt(b, runs[r]);
  *out = b;
  return AP_OK;
}

AP_API int ap_batch_add(ap_batch *b, ap_ctx *c) {
  if (!b || !run_ok(c)) return AP_ERR_INVALID;
  if (std::find(b->runs.begin(), b->runs.end(), static_cast<Ctx *>(c)) != b->runs.end())
    return AP_ERR_INVALID;
  B_TRY_ST(ensure_stage(b, b->runs.size() + 1));
  adopt(b, c);
  return AP_OK;
}

AP_API int ap_batch_remove(ap_batch *b, ap_ctx *c) {
  if (!b || !c) return AP_ERR_INVALID;
  auto it = std::find(b->runs.begin(), b->runs.end(), static_cast<Ctx *>(c));
  if (it == b->runs.end()) return AP_ERR_INVALID;
  B_TRY(cudaStreamSynchronize(b->stream));
  b->runs.erase(it);
  // the run goes back to synchronous calls on the default stream
  ap_set_stream(c, nullptr);
  c->sync = true;
  return AP_OK;
}

AP_API int ap_batch_size(const ap_batch *b, int *nruns) {
  if (!b || !nruns) return AP_ERR_INVALID;
  *nruns = (int)b->runs.size();
  return AP_OK;
}

AP_API int ap_batch_destroy(ap_batch *b) {
  if (!b) return AP_ERR_INVALID;
  if (b->stream) cudaStreamSynchronize(b->stream);
  // the runs go back to synchronous calls on the default stream
  for (Ctx *c : b->runs) {
    ap_set_stream(static_cast<ap_ctx *>(c), nullptr);
    c->sync = true;
  }
  release(b);
  delete b;
  return AP_OK;
}

AP_API int ap_batch_set_stream(ap_batch *b, void *stream) {
  if (!b) return AP_ERR_INVALID;
  B_TRY(cudaStreamSynchronize(b->stream));
  if (b->own_stream) cudaStreamDestroy(b->stream);
  b->own_stream = false;
  b->stream = static_cast<cudaStream_t>(stream);
  for (Ctx *c : b->runs) ap_set_stream(static_cast<ap_ctx *>(c), b->stream);
  for (int i = 0; i < 2; ++i) B_TRY(cudaEventRecord(b->stage_ev[i], b->stream));
  return AP_OK;
}

AP_API int ap_batch_set_capture(ap_batch *b, int on) {
  if (!b) return AP_ERR_INVALID;
  if (on) {
    b->capture = true;
    return AP_OK;
  }
  B_TRY(cudaStreamSynchronize(b->stream));
  free_arena(b);
  b->capture = false;
  return AP_OK;
}

AP_API int ap_batch_update_particles(ap_batch *b, const double *dt, const uint32_t *steps) {
  if (!b || !dt || !steps) return AP_ERR_INVALID;
  return batch_update(b, dt, steps);
}

AP_API int ap_batch_update_fields(ap_batch *b, const double *dt, const uint32_t *steps) {
  if (!b || !dt || !steps) return AP_ERR_INVALID;
  // 1D runs: four batched launches (initial E half step where a run is at
  // step 0, B, E, divergences); 2D runs one by one
  std::vector<Run1D> d1;
  std::vector<uint32_t> items;
  bool any_half = false;
  for (size_t r = 0; r < b->runs.size(); ++r) {
    Ctx *c = b->runs[r];
    if (!is_1d(c)) {
      int st = ap_update_fields(static_cast<ap_ctx *>(c), dt[r], steps[r]);
      if (st != AP_OK) return st;
      continue;
    }
    Run1D d;
    B_TRY_ST(fill_run1d(c, dt[r], steps[r], d));
    any_half = any_half || d.dt_half > 0.0f;
    d1.push_back(d);
    items.push_back((uint32_t)((d.r0 + 255) / 256));
    c->launches += 3;
  }
  if (d1.empty()) return AP_OK;
  const Run1D *dd = nullptr;
  const uint32_t *db = nullptr;
  uint32_t tot = 0;
  B_TRY_ST(stage_run1d(b, d1, items, &dd, &db, &tot));
  const int nr = (int)d1.size();
  if (any_half) B_TRY(launch_b1_fields(b->stream, b->num_sms, dd, db, nr, tot, 0));
  B_TRY(launch_b1_fields(b->stream, b->num_sms, dd, db, nr, tot, 1));
  B_TRY(launch_b1_fields(b->stream, b->num_sms, dd, db, nr, tot, 2));
  B_TRY(launch_b1_fields(b->stream, b->num_sms, dd, db, nr, tot, 3));
  return AP_OK;
}

AP_API int ap_batch_sort_by_cell(ap_batch *b) {
  if (!b) return AP_ERR_INVALID;
  for (Ctx *c : b->runs) {
    int st = ap_sort_by_cell(static_cast<ap_ctx *>(c));
    if (st != AP_OK) return st;
  }
  return AP_OK;
}

AP_API int ap_batch_inject_pairs(ap_batch *b, const double *dt, const uint32_t *steps) {
  if (!b || !dt || !steps) return AP_ERR_INVALID;
  // 1D runs: three batched launches over all their chunks; 2D runs one by one
  std::vector<Run1D> d1;
  std::vector<uint32_t> items;
  for (size_t r = 0; r < b->runs.size(); ++r) {
    Ctx *c = b->runs[r];
    if (!c->pair.enabled || !c->pstate) continue;
    if (!is_1d(c)) {
      B_TRY_ST(enqueue_pairs(*c, (float)dt[r], steps[r]));
      continue;
    }
    Run1D d;
    B_TRY_ST(fill_run1d(c, dt[r], steps[r], d));
    d1.push_back(d);
    items.push_back(pair_chunks_of(*c));
    c->number_stale = true;
    c->launches += 3;
  }
  if (d1.empty()) return AP_OK;
  const Run1D *dd = nullptr;
  const uint32_t *db = nullptr;
  uint32_t tot = 0;
  B_TRY_ST(stage_run1d(b, d1, items, &dd, &db, &tot));
  B_TRY(launch_b1_pairs(b->stream, b->num_sms, dd, db, (int)d1.size(), tot));
  return AP_OK;
}

AP_API int ap_batch_advance(ap_batch *b, const double *dt, const uint32_t *steps0, int nsteps,
                            int sort_interval, int inject) {
  if (!b || !dt || !steps0 || nsteps < 0 || sort_interval < 0) return AP_ERR_INVALID;
  std::vector<uint32_t> st(steps0, steps0 + b->runs.size());
  for (int s = 0; s < nsteps; ++s) {
    B_TRY_ST(batch_update(b, dt, st.data()));
    B_TRY_ST(ap_batch_update_fields(b, dt, st.data()));
    if (inject) B_TRY_ST(ap_batch_inject_pairs(b, dt, st.data()));
    for (size_t r = 0; r < b->runs.size(); ++r) {
      if (sort_interval > 0 && st[r] != 0 && st[r] % (uint32_t)sort_interval == 0)
        B_TRY_ST(ap_sort_by_cell(static_cast<ap_ctx *>(b->runs[r])));
      ++st[r];
    }
  }
  return AP_OK;
}

AP_API int ap_batch_sync(ap_batch *b, int *failed_run) {
  if (!b) return AP_ERR_INVALID;
  if (failed_run) *failed_run = -1;
  B_TRY(cudaStreamSynchronize(b->stream));
  // the status words of batched runs accumulate between syncs: read, then
  // clear them
  int first = AP_OK;
  for (size_t r = 0; r < b->runs.size(); ++r) {
    int st = ctx_check_status(b->runs[r]);
    B_TRY(cudaMemsetAsync(b->runs[r]->status, 0, sizeof(DevStatus), b->stream));
    if (st != AP_OK && first == AP_OK) {
      if (failed_run) *failed_run = (int)r;
      first = st;
    }
  }
  return first;
}

AP_API int ap_batch_autotune(ap_batch *b, const double *dt, const uint32_t *steps,
                             int *steps_used) {
  if (!b || !dt || !steps) return AP_ERR_INVALID;
  std::vector<uint32_t> cur(steps, steps + b->runs.size());
  // classes: runs with the same grid size
  std::map<std::pair<int, int>, int> cls;
  b->tune_class.assign(b->runs.size(), 0);
  for (size_t r = 0; r < b->runs.size(); ++r) {
    auto key = std::make_pair(b->runs[r]->mesh.dims[0], b->runs[r]->mesh.dims[1]);
    auto it = cls.find(key);
    if (it == cls.end()) it = cls.emplace(key, (int)cls.size()).first;
    b->tune_class[r] = it->second;
  }
  const int ncls = (int)cls.size();
  for (cudaEvent_t e : b->tune_ev) cudaEventDestroy(e);
  b->tune_ev.assign(2 * ncls, nullptr);
  for (auto &e : b->tune_ev) B_TRY(cudaEventCreate(&e));
  b->tune_ms.assign(ncls, 0.0f);
  // Candidates: every compiled tile shape with 256-particle chunks, and the
  // two large shapes with 512-particle chunks. Each runs kSteps steps; the
  // first includes the order rebuild after the shape change and the next
  // one still reads a freshly sorted store (which flatters small tiles,
  // whose particles change tiles more often in steady state), so only the
  // last kSteps - 2 are timed.
  constexpr int kCand = 7, kSteps = 5;
  const int cand[kCand][3] = {{16, 16, 256}, {32, 16, 256}, {16, 8, 256}, {8, 8, 256},
                              {4, 4, 256},   {16, 16, 512}, {32, 16, 512}};
  std::vector<float> best(ncls, 1e30f);
  std::vector<int> best_k(ncls, 0);
  int used = 0;
  b->tuning = true;
  int st = AP_OK;
  for (int k = 0; k < kCand && st == AP_OK; ++k) {
    // a candidate needs three tiles per dim for the per-step order update
    std::vector<bool> ok(ncls, false);
    for (size_t r = 0; r < b->runs.size(); ++r) {
      const Ctx *c = b->runs[r];
      if (c->mk.dim != 2) continue;  // 1D runs have no tiles
      const bool fits = (c->mk.red[0] + cand[k][0] - 1) / cand[k][0] >= 3 &&
                        (c->mk.red[1] + cand[k][1] - 1) / cand[k][1] >= 3;
      if (fits) {
        ok[b->tune_class[r]] = true;
        st = ap_set_tile_shape(static_cast<ap_ctx *>(b->runs[r]), cand[k][0], cand[k][1]);
        if (st != AP_OK) break;
        b->runs[r]->params.chunk = cand[k][2];
      }
    }
    // the first step after a shape change includes the order rebuild: time
    // the push / deposit of the following ones
    std::vector<float> sum(ncls, 0.0f);
    for (int rep = 0; rep < kSteps && st == AP_OK; ++rep) {
      st = batch_update(b, dt, cur.data());
      if (st == AP_OK) st = ap_batch_update_fields(b, dt, cur.data());
      for (uint32_t &x : cur) ++x;
      ++used;
      if (rep > 1)
        for (int cl = 0; cl < ncls; ++cl) sum[cl] += b->tune_ms[cl];
    }
    if (st != AP_OK) break;
    for (int cl = 0; cl < ncls; ++cl)
      if (ok[cl] && sum[cl] < best[cl]) {
        best[cl] = sum[cl];
        best_k[cl] = k;
      }
  }
  b->tuning = false;
  if (st == AP_OK)
    for (size_t r = 0; r < b->runs.size() && st == AP_OK; ++r) {
      if (b->runs[r]->mk.dim != 2) continue;
      const int k = best_k[b->tune_class[r]];
      int tx = 0, ty = 0;
      ap_get_tile_shape(static_cast<ap_ctx *>(b->runs[r]), &tx, &ty);
      if (tx != cand[k][0] || ty != cand[k][1])
        st = ap_set_tile_shape(static_cast<ap_ctx *>(b->runs[r]), cand[k][0], cand[k][1]);
      b->runs[r]->params.chunk = cand[k][2];
    }
  if (steps_used) *steps_used = used;
  return st;
}

}  // extern "C"

// Internal declarations shared by the CUDA translation units of
// libaperture_b200.so. Nothing here is part of the public ABI.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <vector>
#include <stdint.h>

#include "../../include/aperture_b200.h"

namespace apb {

// Status-word bits written by kernels (device side, atomicOr) and counters
// (atomicAdd) in DevStatus.
struct DevStatus {
  unsigned long long nan_momenta;
  unsigned long long moved_far;
  unsigned long long lost;
  unsigned long long tile_faults;
  unsigned long long timeouts;
};

// Grid constants a kernel needs (a copy of the host ap_mesh, in the
// forms the kernels use).
struct MeshK {
  int dims[3];
  int guard[3];
  int red[3];
  float delta[3];
  float inv_delta[3];
  float lower[3];
  int dim;
  unsigned long long div0;  // floor(2^64 / dims[0]) + 1: c / dims[0] = umul64hi(c, div0)
};

// Fixed-point format of the current/charge accumulators (see
// k_push_deposit.cu): a contribution v becomes X = rint(v * 2^S), split into
// hi = X >> L (int32) and lo = X mod 2^L (uint32) in shared memory.
struct FixedFmt {
  int S;
  int L;
};

struct PtcK {
  float *x1, *x2, *x3, *p1, *p2, *p3, *E, *w;
  uint32_t *cell;
  uint32_t *flag;
};

struct FieldArr {
  float *ptr;
  int pitch;  // in floats
};

// Six tensor maps for the E/B tiles (E1, E2, E3, B1, B2, B3).
struct alignas(64) FieldMaps {
  CUtensorMap m[6];
};

// Tile geometry of the 2D sort.
struct TilesK {
  int tx, ty;    // tile size in cells
  int ntx, nty;  // tiles per dim
  int ntiles;
};

struct PushDepositParams {
  MeshK m;
  PtcK p;
  FieldArr F[6];     // E1..E3, B1..B3 (used when tensor maps are off)
  FieldArr J[3];
  FieldArr Rho[AP_MAX_SPECIES];
  // Fixed-point accumulators of J1..J3 then Rho[0..num_species): component k
  // at acc + k * acc_comp, row-major with row length acc_pitch. A value v is
  // stored as the 64-bit integer rint(v * 2^S) (two's complement), S from
  // the FixedFmt the kernel writes to fx_used.
  unsigned long long *acc;
  int acc_pitch;
  size_t acc_comp;
  FixedFmt *fx_used;      // device: format used by this update (read by finalize)
  const uint32_t *n_max;  // device: largest tile population (2D)
  const float *wmax;      // device: largest |weight|
  float qmax;             // largest |charge|
  float dt;
  float qm[AP_MAX_SPECIES];      // dt * 0.5f * q / m, evaluated as the reference does
  float charge[AP_MAX_SPECIES];
  int num_species;
  int do_rho;
  int periodic[3];
  // 2D tile order
  TilesK t;
  const uint32_t *order;
  const uint32_t *tile_start;
  uint8_t *dir;
  uint32_t *dir_count;   // ntiles * 10
  // per staged chunk of the tile lists, its direction counts (10 each):
  // chunk k of tile t is entry tile_start[t] / CH + t + k (null: not kept)
  uint32_t *chunk_count;
  uint32_t *queue;
  DevStatus *status;
  size_t number;         // 1D: particle slots (an upper bound when d_number is set)
  const uint32_t *d_number;  // 1D: live slots kept on the device, or null
  // 2D compaction step: every member of the particle at tile-list position
  // q is written to slot q of this scratch store (null pointers otherwise)
  PtcK cout;
  uint64_t *cout_id;
  const uint64_t *id;
  // log-spherical push / move (ap_logsph_params)
  float ls_compactness, ls_omega, ls_gravity, ls_rad_coef, ls_B0;
  int ls_rad_on;
  int ls_outflow_c1;     // dims[0] - damping_length + 2
  float mass[AP_MAX_SPECIES];
  FieldArr dV;           // cell volumes (J3 and Rho are divided by them)
};

// Device-side particle bookkeeping of a context with pair injection: the
// live slot count (updated by injection and sort on the device, so that the
// step loop needs no host round trip), counters of the last injection and
// running totals. The host copy Ctx::number is refreshed at sync points.
struct PairState {
  uint32_t number;
  uint32_t emitted;        // last injection
  uint32_t dropped;        // last injection, over capacity
  uint32_t old_number;     // last injection: live slots before it
  unsigned long long next_id;
  unsigned long long particle_steps;  // sum of live slots over injections
  unsigned long long emitted_total;
  unsigned long long dropped_total;
};

// A 1D run in the batched per-step launches other than the push / deposit
// (accumulator clearing, current finalize, field update, pair injection):
// everything a kernel needs, so that one launch serves all 1D runs.
struct Run1D {
  int n0, g0, r0, per0;
  float id0;
  FieldArr E[3], B[3], Eb[3], Bb[3], J[3], Rho[AP_MAX_SPECIES], divE, divB;
  unsigned long long *acc;
  size_t acc_comp;
  const FixedFmt *fx;
  int zero_comps;  // accumulator components to clear before the push
  int ncomp;       // components the finalize rounds (3 + species on charge steps)
  float dt;        // field update
  float dt_half;   // the initial E half step (step 0), else 0
  int has_divs;
  // pair injection
  float gamma_thr, free_path, pair_energy, pair_dt;
  uint32_t key[2];
  uint32_t step;
  PtcK p;
  uint64_t *ids;
  PairState *pst;
  uint8_t *emit;
  uint32_t *counts, *offs, *tot;
  size_t capacity;
};

// Batched 1D launches (k_fields.cu, k_pairs.cu). base has nruns + 1
// entries: run r owns work items [base[r], base[r + 1]). Items are blocks
// of 256 accumulator words (zero), 256 cells (finalize), 256 bulk cells
// (fields), 1024 particle slots (pairs).
cudaError_t launch_b1_zero(cudaStream_t s, int num_sms, const Run1D *runs, const uint32_t *base,
                           int nruns, uint32_t total);
cudaError_t launch_b1_finalize(cudaStream_t s, int num_sms, const Run1D *runs,
                               const uint32_t *base, int nruns, uint32_t total);
// which: 0 initial E half step, 1 B, 2 E, 3 divergences
cudaError_t launch_b1_fields(cudaStream_t s, int num_sms, const Run1D *runs, const uint32_t *base,
                             int nruns, uint32_t total, int which);
cudaError_t launch_b1_pairs(cudaStream_t s, int num_sms, const Run1D *runs,
                            const uint32_t *base, int nruns, uint32_t total);

// One run of a batched launch: its tensor maps and its parameters, in
// device memory (the maps must be 64-byte aligned).
struct alignas(64) RunDesc {
  FieldMaps maps;
  PushDepositParams P;
};

// Per-context state.
struct Ctx {
  int device = 0;
  ap_mesh mesh{};
  ap_params params{};
  MeshK mk{};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bool sync = true;
  int last_error = AP_OK;
  uint64_t launches = 0;
  int num_sms = 148;

  bool fields_bound = false;
  ap_fields fields{};
  bool use_tma = false;
  FieldMaps maps{};

  bool ptc_bound = false;
  ap_particles ptc{};
  size_t number = 0;
  size_t capacity = 0;

  // 2D tile order (ping-pong)
  TilesK tiles{};
  uint32_t *order[2] = {nullptr, nullptr};
  uint32_t *tile_start[2] = {nullptr, nullptr};
  int cur = 0;
  bool order_valid = false;
  uint8_t *dir = nullptr;
  uint32_t *dir_count = nullptr;
  uint32_t *grp_off = nullptr;
  uint32_t *newcount = nullptr;  // per-tile population after the step
  uint32_t *queue = nullptr;
  size_t order_cap = 0;
  // per-chunk direction counts of the push / deposit (one-pass order update)
  uint32_t *chunk_count = nullptr;
  size_t chunk_count_cap = 0;  // entries of 10 counts
  uint32_t *big_tiles = nullptr;  // count, then tiles left to the two-pass kernel
  size_t big_tiles_cap = 0;
  bool chunk_count_ok = false;  // the last push / deposit recorded them

  // rebuild / sort scratch
  uint32_t *keys[2] = {nullptr, nullptr};
  uint32_t *vals[2] = {nullptr, nullptr};
  uint32_t *rx_counts = nullptr;  // radix sort: per-CTA digit counts
  void *gather_tmp = nullptr;
  size_t scratch_cap = 0;
  uint32_t *cell_start = nullptr;  // ncells + 1 entries, set by sort_by_cell
  uint32_t *cell_count = nullptr;  // ncells + 1 entries (tile-local sort)
  uint32_t *sort_max = nullptr;    // device: largest cell population (tile-local sort)

  // fixed-point current / charge accumulators (3 + num_species components)
  unsigned long long *acc = nullptr;
  size_t acc_comp = 0;
  FixedFmt *fx_used = nullptr;  // device: format of the last deposit
  uint32_t *n_max = nullptr;    // device: largest tile population
  float *wmax = nullptr;        // device: max |weight| over the bound particles
  bool scale_valid = false;

  // filter scratch
  float *tmp_j = nullptr;
  int tmp_pitch = 0;

  // pair injection (ap_set_pair_params)
  ap_pair_params pair{};
  uint32_t *pair_chunks = nullptr;  // per-chunk counts then offsets, then totals
  size_t pair_cap_chunks = 0;
  PairState *pstate = nullptr;      // device (allocated with the pair parameters)
  PairState *pstate_host = nullptr; // pinned mirror
  bool number_stale = false;        // the device count moved since the last read
  bool rho_is_zero = false;         // Rho arrays hold zeros (skip re-zeroing)
  int compact_interval = 0;         // 2D: rewrite the store in tile order every n updates
  int since_compact = 0;
  void *compact_buf = nullptr;      // scratch copy of the store (48 B per slot)
  size_t compact_cap = 0;
  bool compact_now = false;         // this update writes the store in tile order
  size_t store_base = 0;            // lowest slot that may hold a particle
  size_t compact_dst = 0;           // first slot of this compaction's output
  bool compact_direct = false;      // output in the caller's free half, no copy back

  // log-spherical grid (ap_ctx_create_logsph)
  int coord = 0;                // 0 Cartesian, 1 log-spherical, 2 1D gap, 3 1D GR
  ap_gap_params gap{};          // 1D gap lab parameters
  ap_gr_params gr{};            // 1D GR lab parameters (coefficients in coef)
  float gr_kfac = 1.0f;         // bound of |J1, Rho contribution| / (|q| w) in the GR deposit
  double *ls_surface = nullptr;  // log-spherical injection: surface densities
  uint32_t inject_calls = 0;
  uint64_t inject_next_id = 1ull << 62;
  ap_logsph_params lsp{};
  float *coef = nullptr;        // AP_NUM_COEF arrays of dims[0] x dims[1]
  size_t coef_pitch = 0;        // bytes per row
  float ls_kfac = 1.0f;         // bound of |J3 contribution| / (|q| w)

  // photons and pair production (ap_bind_photons, ap_set_rad_params)
  bool ph_bound = false;
  ap_photons ph{};
  size_t ph_number = 0;
  size_t ph_capacity = 0;
  bool rad_on = false;
  ap_rad_params rad{};
  uint32_t rad_emit_calls = 0;
  uint32_t rad_pair_calls = 0;
  uint64_t rad_next_photon_id = 0;
  uint64_t rad_next_ptc_id = 0;
  uint8_t *rad_mark = nullptr;     // one byte per slot of the larger store
  size_t rad_mark_cap = 0;
  uint32_t *rad_chunks = nullptr;  // per-chunk counts, offsets, then the total
  size_t rad_chunks_cap = 0;
  uint32_t *rad_total_host = nullptr;  // pinned: marked count of the last pass
  // inverse-Compton tables (ap_ic_init; k_ic.cu), device arrays
  float *ic_buf = nullptr;  // ic_rate, gg_rate, gammas, dNde, dNde_thomson
  int ic_n_gamma = 0, ic_n_ep = 0;
  float ic_dep = 0.0f, ic_dg = 0.0f, ic_dlep = 0.0f;
  bool ic_ready = false;
  ap_spectrum ic_spec{};     // what the tables were built for
  double ic_emin = 0.0, ic_emax = 0.0, ic_n0 = 0.0;

  // per-phase event timing (ap_set_profiling)
  bool profiling = false;
  struct EventPair {
    cudaEvent_t a, b;
    int phase;
  };
  EventPair *ev = nullptr;
  int ev_used = 0, ev_cap = 0;
  uint64_t pd_launches = 0;

  DevStatus *status = nullptr;     // device
  DevStatus *status_host = nullptr;  // pinned
  double *diag_dev = nullptr;
  double *diag_host = nullptr;
  // FP64 continuity check (ap_set_continuity_check): the total charge
  // density of the last update with Rho output, and its step
  bool cont_on = false;
  double *rho_prev = nullptr;  // dims[0] * dims[1] doubles
  long long last_rho_step = -2;
  bool cont_snap = false;      // this update took the snapshot
};

// --- launchers (defined in the .cu files) ---
cudaError_t launch_push_deposit_2d(Ctx &c, const PushDepositParams &P);
cudaError_t launch_push_deposit_1d(Ctx &c, const PushDepositParams &P);
cudaError_t launch_selftest_wait(Ctx &c, uint32_t limit);
cudaError_t launch_tile_scan(Ctx &c, const uint32_t *dir_count,
                             uint32_t *new_start, uint32_t *grp_off);
// old_order null: the particle at list position p sits in slot slot0 + p.
cudaError_t launch_order_scatter(Ctx &c, const uint32_t *old_start,
                                 const uint32_t *old_order, const uint8_t *dir,
                                 const uint32_t *grp_off, uint32_t *new_order,
                                 uint32_t slot0 = 0);
cudaError_t rebuild_tile_order(Ctx &c);
// Stable LSD radix sort of (c.keys[0], c.vals[0])[0, n) by the low end_bit
// bits of the keys, ping-ponging with keys[1] / vals[1] (k_radix.cu).
cudaError_t radix_sort_pairs(Ctx &c, size_t n, int end_bit, uint32_t **keys_out,
                             uint32_t **vals_out);
size_t radix_count_words(int num_sms);
cudaError_t sort_by_cell(Ctx &c, size_t *new_number);
cudaError_t sort_photons(Ctx &c, size_t *new_number);
// Compaction: the scratch store the push / deposit writes into (allocated on
// first use), and the copy back into the caller's arrays; `live` is the
// device-side count of written slots, the slots after it become empty.
cudaError_t compact_store(Ctx &c, PtcK *out, uint64_t **out_id);
cudaError_t compact_finish(Ctx &c, const uint32_t *live);

cudaError_t launch_fold_guards(Ctx &c, ap_array a);
cudaError_t launch_copy_guards(Ctx &c, ap_array a);
cudaError_t launch_update_e(Ctx &c, float dt);
cudaError_t launch_update_b(Ctx &c, float dt);
cudaError_t launch_divs(Ctx &c);
cudaError_t launch_filter(Ctx &c, ap_array a, int bnd[4]);
cudaError_t launch_zero(Ctx &c, ap_array a);
cudaError_t launch_finalize_current(Ctx &c, int ncomp);
cudaError_t launch_fixed_scale(Ctx &c);
cudaError_t launch_diagnostics(Ctx &c, double *out_dev);
// rho_prev = sum over species of Rho (FP64)
cudaError_t launch_rho_snapshot(Ctx &c);
// *out = max over the bulk of |sum_s Rho_s - rho_prev + div J| (FP64)
cudaError_t launch_continuity(Ctx &c, double *out);

// photons and pair production (k_rad.cu): the photon move of an update, and
// the emit / produce passes; *marked receives the emitters of the pass
// (waits for the stream).
int rad_move_photons(Ctx &c, float dt, uint32_t step);
int rad_emit_photons(Ctx &c, ap_array produced, ap_rad_counts *out);
int rad_produce_pairs(Ctx &c, ap_array produced, ap_rad_counts *out);
void rad_free(Ctx &c);
// inverse_compton (k_ic.cu): builds the tables on the device; frees them
int ic_init(Ctx &c, const ap_spectrum &s, double emin, double emax, double n0, int n_gamma,
            int n_ep);
void ic_free(Ctx &c);

// pair injection (k_pairs.cu): enqueue mark / scan / append on the device
// count (no host synchronisation); refresh_number reads the device state
// back when it moved (waits for the stream); push_number writes the host
// count to the device.
int enqueue_pairs(Ctx &c, float dt, uint32_t step);
int ensure_pair_scratch(Ctx &c);
uint32_t pair_chunks_of(const Ctx &c);
int refresh_number(Ctx *c);
int push_number(Ctx *c);

// log-spherical (k_logsph.cu)
int logsph_setup(Ctx &c);  // coefficients on the host, upload, J3 bound
ap_array coef_array(const Ctx &c, int which);
// 1D gap lab (k_gap.cu)
cudaError_t launch_gap_push_deposit(Ctx &c, const PushDepositParams &P);
cudaError_t launch_gap_filter(Ctx &c, const float *src, float *dst, int bnd_lower,
                              int bnd_upper);
cudaError_t launch_gap_update_e(Ctx &c, float j0, float dt);

// 1D GR lab (k_gr.cu): coefficient pointers and parameters of the pusher.
struct GrK {
  const float *D1, *D2, *D3, *alpha, *theta, *K1, *K1_j, *agrr, *B3B1;
  float a, omega;
  uint32_t step;
  int data_interval;
};
void host_gr_coef(const ap_mesh &m, const ap_gr_params &gp, const ap_gr_table &t,
                  std::vector<float> *co);
cudaError_t launch_gr_push_deposit(Ctx &c, const PushDepositParams &P, const GrK &G);
cudaError_t launch_gr_filter(Ctx &c, const float *src, float *dst, const float *k1,
                             int bnd_lower, int bnd_upper);
cudaError_t launch_gr_update_e(Ctx &c, const float *j0, float dt);

cudaError_t launch_ls_finalize(Ctx &c, float dt, bool do_rho, bool zero_axis);
cudaError_t launch_ls_smooth(Ctx &c, bool do_rho);
cudaError_t launch_ls_update_b(Ctx &c, float dt);
cudaError_t launch_ls_update_e(Ctx &c, float dt);
cudaError_t launch_ls_divs(Ctx &c);
cudaError_t launch_ls_field_boundary(Ctx &c, float omega);
cudaError_t launch_ls_inject(Ctx &c, int inj, float p1, float w, uint64_t seed, uint32_t call,
                             uint64_t first_id, double *surface);

MeshK make_meshk(const ap_mesh &m);

// Particles staged per chunk by the 2D push / deposit of this context: 1024
// for log-spherical grids, else the configured 256, 1024 or 2048, or 512.
inline int chunk_of(const Ctx &c) {
  if (c.coord == 1) return 256;
  const int ch = c.params.chunk;
  return (ch == 512 || ch == 1024 || ch == 2048) ? ch : 256;
}

// The update of one context in three parts (ap_api.cu): prepare (zeroing,
// tile-order rebuild, kernel parameters), the push / deposit launch, and
// complete (order update, finalize, smoothing). ctx_check_status reads the
// device status word back (waits for the stream).
// batched: the caller clears the accumulators (and, for 1D runs, runs the
// finalize) in batched launches; the device status word is not cleared, so
// it accumulates until the batch reads it.
int update_prepare(Ctx *c, double dt, uint32_t step, PushDepositParams &P, bool *has_work,
                   bool batched = false);
int update_complete(Ctx *c, double dt, uint32_t step, bool had_work, bool batched = false);
// Smoothing after a finalize done elsewhere (batched 1D runs).
int update_smooth(Ctx *c, uint32_t step);
// Fills the 1D batch descriptor of a context (fields, accumulators, pair
// scratch) for the given step and dt.
int fill_run1d(Ctx *c, double dt, uint32_t step, Run1D &d);

int ctx_check_status(Ctx *c);

// One persistent push / deposit launch over the tiles of several 2D
// Cartesian runs with the same tile shape, chunk and field-load path.
// runs / base are device arrays (base has nruns + 1 entries).
cudaError_t launch_push_deposit_2d_batch(cudaStream_t stream, int num_sms, int tx, int ty,
                                         int chunk, bool tma, bool do_rho, int max_species,
                                         const RunDesc *runs, const uint32_t *base, int nruns,
                                         uint32_t total_tiles, uint32_t *queue);
// The same for 1D runs: work items are chunks of 2048 particle slots
// (base[r] = first chunk of run r).
cudaError_t launch_push_deposit_1d_batch(cudaStream_t stream, int num_sms, bool do_rho,
                                         const RunDesc *runs, const uint32_t *base, int nruns,
                                         uint32_t total_chunks);
constexpr int kChunk1DSlots = 2048;
int ensure_scratch(Ctx &c, size_t n);

}  // namespace apb

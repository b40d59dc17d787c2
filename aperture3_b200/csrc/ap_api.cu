// C ABI of libaperture_b200.so: context management, binding of the
// caller's arrays, and the orchestration of ptc_updater::update_particles /
// field_solver::update_fields for one rank.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>

#include "ap_internal.h"

using namespace apb;

struct ap_ctx : public apb::Ctx {};

namespace apb {

MeshK make_meshk(const ap_mesh &m) {
  MeshK k;
  for (int i = 0; i < 3; ++i) {
    k.dims[i] = m.dims[i];
    k.guard[i] = m.guard[i];
    k.red[i] = m.dims[i] - 2 * m.guard[i];
    k.delta[i] = m.delta[i];
    k.inv_delta[i] = m.inv_delta[i];
    k.lower[i] = m.lower[i];
  }
  k.div0 = (m.dims[0] > 1) ? (~0ull / (unsigned long long)m.dims[0]) + 1ull : 0ull;
  if (m.dims[1] <= 1 && m.dims[2] <= 1)
    k.dim = 1;
  else if (m.dims[2] <= 1)
    k.dim = 2;
  else
    k.dim = 3;
  return k;
}

}  // namespace apb

namespace {

int fail(Ctx *c, int st) {
  if (c) c->last_error = st;
  return st;
}

int cuda_fail(Ctx *c, cudaError_t e) {
  if (e == cudaSuccess) return AP_OK;
  if (e == cudaErrorMemoryAllocation) return fail(c, AP_ERR_NOMEM);
  return fail(c, AP_ERR_CUDA);
}

#define AP_TRY(expr)                              \
  do {                                            \
    cudaError_t _e = (expr);                      \
    if (_e != cudaSuccess) return cuda_fail(c, _e); \
  } while (0)

#define AP_TRY_ST(expr)              \
  do {                               \
    int _s = (expr);                 \
    if (_s != AP_OK) return fail(c, _s); \
  } while (0)

bool is_supported_tile(int tx, int ty) {
  return (tx == 16 && ty == 16) || (tx == 32 && ty == 16) || (tx == 8 && ty == 8) ||
         (tx == 16 && ty == 8) || (tx == 4 && ty == 4);
}

void choose_tiles(Ctx &c) {
  const int r0 = c.mk.red[0], r1 = c.mk.dim > 1 ? c.mk.red[1] : 1;
  int tx = c.params.tile[0], ty = c.params.tile[1];
  if (c.mk.dim == 1) {
    tx = 1;
    ty = 1;
  } else if (!is_supported_tile(tx, ty)) {
    const int cand[4][2] = {{16, 16}, {8, 8}, {4, 4}, {4, 4}};
    tx = 4;
    ty = 4;
    for (auto &t : cand)
      if ((r0 + t[0] - 1) / t[0] >= 3 && (r1 + t[1] - 1) / t[1] >= 3) {
        tx = t[0];
        ty = t[1];
        break;
      }
  }
  c.tiles.tx = tx;
  c.tiles.ty = ty;
  c.tiles.ntx = (r0 + tx - 1) / tx;
  c.tiles.nty = c.mk.dim > 1 ? (r1 + ty - 1) / ty : 1;
  c.tiles.ntiles = c.tiles.ntx * c.tiles.nty;
}

// The per-step order update needs at least three tiles per dim so that the
// eight neighbours of a tile are distinct; smaller grids rebuild the order
// with the full sort every step.
bool incremental_order(const Ctx &c) { return c.tiles.ntx >= 3 && c.tiles.nty >= 3; }

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// Tensor maps for the E/B tiles: a box of (tx + 8) x (ty + 2) floats whose
// x start is rounded down to a multiple of four floats (16 bytes).
bool setup_tensor_maps(Ctx &c) {
  if (c.mk.dim != 2) return false;
  auto enc = encode_fn();
  if (!enc) return false;
  const ap_array *src[6] = {&c.fields.E[0], &c.fields.E[1], &c.fields.E[2],
                            &c.fields.B[0], &c.fields.B[1], &c.fields.B[2]};
  for (int k = 0; k < 6; ++k) {
    const ap_array &a = *src[k];
    if ((reinterpret_cast<uintptr_t>(a.ptr) & 15u) || (a.pitch & 15u)) return false;
    cuuint64_t gdim[2] = {(cuuint64_t)c.mesh.dims[0], (cuuint64_t)c.mesh.dims[1]};
    cuuint64_t gstride[1] = {(cuuint64_t)a.pitch};
    cuuint32_t box[2] = {(cuuint32_t)(c.tiles.tx + 8), (cuuint32_t)(c.tiles.ty + 2)};
    cuuint32_t estride[2] = {1, 1};
    CUresult r = enc(&c.maps.m[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, a.ptr, gdim, gstride, box,
                     estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
  }
  return true;
}

bool valid_array(const ap_array &a, const ap_mesh &m) {
  return a.ptr != nullptr && a.pitch >= sizeof(float) * (size_t)m.dims[0] &&
         (a.pitch % sizeof(float)) == 0;
}

int finish(Ctx *c) {
  if (!c->sync) return AP_OK;
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e);
  return AP_OK;
}

int check_status(Ctx *c) {
  if (refresh_number(c) != AP_OK) return fail(c, AP_ERR_CUDA);
  cudaError_t e = cudaMemcpyAsync(c->status_host, c->status, sizeof(DevStatus),
                                  cudaMemcpyDeviceToHost, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e);
  e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e);
  const DevStatus &s = *c->status_host;
  if (s.tile_faults) c->order_valid = false;
  if (s.timeouts) return fail(c, AP_ERR_TIMEOUT);
  if (s.tile_faults) return fail(c, AP_ERR_TILE);
  if (s.nan_momenta) return fail(c, AP_ERR_NAN);
  if (s.moved_far) return fail(c, AP_ERR_MOVED_FAR);
  return AP_OK;
}

int alloc_particle_state(Ctx *c, size_t cap) {
  if (cap <= c->order_cap && c->order[0]) return AP_OK;
  for (int i = 0; i < 2; ++i) {
    cudaFree(c->order[i]);
    c->order[i] = nullptr;
  }
  cudaFree(c->dir);
  c->dir = nullptr;
  size_t n = cap < 1 ? 1 : cap;
  for (int i = 0; i < 2; ++i)
    if (cudaMalloc(&c->order[i], n * sizeof(uint32_t)) != cudaSuccess) return AP_ERR_NOMEM;
  if (cudaMalloc(&c->dir, n) != cudaSuccess) return AP_ERR_NOMEM;
  c->order_cap = n;
  // sort_by_cell's cell starts, here rather than at the first sort, so that
  // no allocation falls between the updates of a run
  if (!c->cell_start) {
    const size_t ncells =
        (size_t)c->mesh.dims[0] * (size_t)c->mesh.dims[1] * (size_t)c->mesh.dims[2];
    if (cudaMalloc(&c->cell_start, sizeof(uint32_t) * (ncells + 1)) != cudaSuccess)
      return AP_ERR_NOMEM;
  }
  return ensure_scratch(*c, n);
}

enum Phase { kPhPushDeposit = 0, kPhOrder, kPhRebuild, kPhFinalize, kPhFields, kPhSort, kPhN };

// Starts a timed phase; returns the slot to close with phase_end, or -1.
int phase_begin(Ctx *c, int phase) {
  if (!c->profiling) return -1;
  if (c->ev_used == c->ev_cap) {
    int cap = c->ev_cap ? 2 * c->ev_cap : 256;
    auto *nv = new (std::nothrow) Ctx::EventPair[cap];
    if (!nv) return -1;
    for (int i = 0; i < c->ev_used; ++i) nv[i] = c->ev[i];
    for (int i = c->ev_used; i < cap; ++i) {
      cudaEventCreate(&nv[i].a);
      cudaEventCreate(&nv[i].b);
    }
    delete[] c->ev;
    c->ev = nv;
    c->ev_cap = cap;
  }
  int k = c->ev_used++;
  c->ev[k].phase = phase;
  cudaEventRecord(c->ev[k].a, c->stream);
  return k;
}

void phase_end(Ctx *c, int k) {
  if (k >= 0) cudaEventRecord(c->ev[k].b, c->stream);
}

}  // namespace

extern "C" {

AP_API const char *ap_version(void) { return "aperture_b200 0.1 (sm_100a)"; }

AP_API const char *ap_status_string(int s) {
  switch (s) {
    case AP_OK: return "ok";
    case AP_ERR_INVALID: return "invalid argument or state";
    case AP_ERR_CUDA: return "CUDA runtime error";
    case AP_ERR_NAN: return "NaN momentum in push";
    case AP_ERR_MOVED_FAR: return "particle moved more than one cell";
    case AP_ERR_CAPACITY: return "size exceeds a fixed limit";
    case AP_ERR_TIMEOUT: return "bounded device wait timed out";
    case AP_ERR_UNSUPPORTED: return "unsupported grid or option";
    case AP_ERR_NOMEM: return "device allocation failed";
    case AP_ERR_TILE: return "particle outside its sort tile";
    default: return "unknown status";
  }
}

AP_API int ap_ctx_create(const ap_mesh *mesh, const ap_params *params, ap_ctx **out) {
  if (!mesh || !params || !out) return AP_ERR_INVALID;
  *out = nullptr;
  MeshK mk = make_meshk(*mesh);
  if (mk.dim == 3) return AP_ERR_UNSUPPORTED;
  for (int d = 0; d < mk.dim; ++d) {
    if (mesh->guard[d] < 2) return AP_ERR_INVALID;  // the deposit reaches two cells out
    if (mk.red[d] < 1) return AP_ERR_INVALID;
    if (params->periodic[d] && mk.red[d] < 2 * mesh->guard[d]) return AP_ERR_INVALID;
  }
  if (params->num_species < 1 || params->num_species > AP_MAX_SPECIES) return AP_ERR_INVALID;
  if (params->data_interval < 1 || params->current_smoothing < 0) return AP_ERR_INVALID;
  if ((uint64_t)mesh->dims[0] * mesh->dims[1] * mesh->dims[2] >= AP_MAX_CELL - 1ull)
    return AP_ERR_CAPACITY;
  ap_ctx *c = new (std::nothrow) ap_ctx();
  if (!c) return AP_ERR_NOMEM;
  c->mesh = *mesh;
  c->params = *params;
  c->mk = mk;
  choose_tiles(*c);
  cudaGetDevice(&c->device);
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return AP_ERR_CUDA;
  }
  c->own_stream = true;
  const int nt = c->tiles.ntiles;
  bool ok = cudaMalloc(&c->status, sizeof(DevStatus)) == cudaSuccess &&
            cudaMallocHost(&c->status_host, sizeof(DevStatus)) == cudaSuccess &&
            cudaMalloc(&c->dir_count, sizeof(uint32_t) * ((size_t)nt * 10 + 16)) == cudaSuccess &&
            cudaMalloc(&c->grp_off, sizeof(uint32_t) * ((size_t)nt * 9 + 16)) == cudaSuccess &&
            cudaMalloc(&c->newcount, sizeof(uint32_t) * ((size_t)nt + 16)) == cudaSuccess &&
            cudaMalloc(&c->tile_start[0], sizeof(uint32_t) * (nt + 1)) == cudaSuccess &&
            cudaMalloc(&c->tile_start[1], sizeof(uint32_t) * (nt + 1)) == cudaSuccess &&
            cudaMalloc(&c->queue, sizeof(uint32_t) * 4) == cudaSuccess &&
            cudaMalloc(&c->diag_dev, sizeof(double) * 16) == cudaSuccess &&
            cudaMalloc(&c->fx_used, sizeof(FixedFmt)) == cudaSuccess &&
            cudaMalloc(&c->n_max, sizeof(uint32_t)) == cudaSuccess &&
            cudaMalloc(&c->wmax, sizeof(float)) == cudaSuccess &&
            cudaMallocHost(&c->diag_host, sizeof(double) * 16) == cudaSuccess;
  if (!ok) {
    ap_ctx_destroy(c);
    return AP_ERR_NOMEM;
  }
  cudaMemset(c->status, 0, sizeof(DevStatus));
  cudaMemset(c->diag_dev, 0xFF, sizeof(double) * 16);  // NaN: nothing recorded yet
  std::memset(c->status_host, 0, sizeof(DevStatus));
  cudaMemset(c->fx_used, 0, sizeof(FixedFmt));
  cudaMemset(c->n_max, 0, sizeof(uint32_t));
  cudaMemset(c->wmax, 0, sizeof(float));
  *out = c;
  return AP_OK;
}

AP_API int ap_ctx_destroy(ap_ctx *c) {
  if (!c) return AP_ERR_INVALID;
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (int i = 0; i < 2; ++i) {
    cudaFree(c->order[i]);
    cudaFree(c->tile_start[i]);
    cudaFree(c->keys[i]);
    cudaFree(c->vals[i]);
  }
  cudaFree(c->dir);
  cudaFree(c->dir_count);
  cudaFree(c->grp_off);
  cudaFree(c->newcount);
  cudaFree(c->queue);
  cudaFree(c->rx_counts);
  cudaFree(c->gather_tmp);
  cudaFree(c->cell_start);
  cudaFree(c->cell_count);
  cudaFree(c->chunk_count);
  cudaFree(c->big_tiles);
  cudaFree(c->ls_surface);
  cudaFree(c->sort_max);
  cudaFree(c->tmp_j);
  cudaFree(c->coef);
  cudaFree(c->compact_buf);
  cudaFree(c->pair_chunks);
  cudaFree(c->pstate);
  if (c->pstate_host) cudaFreeHost(c->pstate_host);
  cudaFree(c->acc);
  cudaFree(c->fx_used);
  cudaFree(c->n_max);
  cudaFree(c->wmax);
  cudaFree(c->status);
  cudaFree(c->diag_dev);
  cudaFree(c->rho_prev);
  rad_free(*c);
  ic_free(*c);
  if (c->status_host) cudaFreeHost(c->status_host);
  if (c->diag_host) cudaFreeHost(c->diag_host);
  for (int i = 0; i < c->ev_cap; ++i) {
    cudaEventDestroy(c->ev[i].a);
    cudaEventDestroy(c->ev[i].b);
  }
  delete[] c->ev;
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return AP_OK;
}

AP_API int ap_set_stream(ap_ctx *c, void *stream) {
  if (!c) return AP_ERR_INVALID;
  if (c->own_stream && c->stream) {
    cudaStreamSynchronize(c->stream);
    cudaStreamDestroy(c->stream);
  }
  c->own_stream = false;
  c->stream = static_cast<cudaStream_t>(stream);
  return AP_OK;
}

AP_API int ap_set_sync(ap_ctx *c, int sync) {
  if (!c) return AP_ERR_INVALID;
  c->sync = sync != 0;
  return AP_OK;
}

AP_API int ap_sync(ap_ctx *c) {
  if (!c) return AP_ERR_INVALID;
  return check_status(c);
}

AP_API int ap_bind_fields(ap_ctx *c, const ap_fields *f) {
  if (!c || !f) return AP_ERR_INVALID;
  const ap_mesh &m = c->mesh;
  for (int k = 0; k < 3; ++k)
    if (!valid_array(f->E[k], m) || !valid_array(f->B[k], m) || !valid_array(f->Ebg[k], m) ||
        !valid_array(f->Bbg[k], m) || !valid_array(f->J[k], m))
      return fail(c, AP_ERR_INVALID);
  for (int s = 0; s < c->params.num_species; ++s)
    if (!valid_array(f->Rho[s], m)) return fail(c, AP_ERR_INVALID);
  c->fields = *f;
  c->fields_bound = true;
  c->rho_is_zero = false;
  c->use_tma = setup_tensor_maps(*c);
  if (!c->acc) {
    c->acc_comp = (size_t)m.dims[0] * m.dims[1] * m.dims[2];
    AP_TRY(cudaMalloc(&c->acc, sizeof(unsigned long long) * c->acc_comp *
                                   (3 + c->params.num_species)));
  }
  if (!c->tmp_j) {
    size_t pitch = sizeof(float) * (size_t)m.dims[0];
    AP_TRY(cudaMalloc(&c->tmp_j, pitch * (size_t)m.dims[1] * m.dims[2]));
    AP_TRY(cudaMemset(c->tmp_j, 0, pitch * (size_t)m.dims[1] * m.dims[2]));
    c->tmp_pitch = m.dims[0];
  }
  return AP_OK;
}

AP_API int ap_bind_particles(ap_ctx *c, const ap_particles *p, size_t number, size_t capacity) {
  if (!c || !p) return AP_ERR_INVALID;
  if (number > capacity || capacity >= (size_t)UINT32_MAX) return fail(c, AP_ERR_CAPACITY);
  if (!p->x1 || !p->x2 || !p->x3 || !p->p1 || !p->p2 || !p->p3 || !p->E || !p->weight ||
      !p->cell || !p->id || !p->flag)
    return fail(c, AP_ERR_INVALID);
  c->ptc = *p;
  c->number = number;
  c->store_base = 0;
  c->capacity = capacity;
  c->ptc_bound = true;
  c->order_valid = false;
  c->scale_valid = false;
  AP_TRY_ST(alloc_particle_state(c, capacity));
  AP_TRY_ST(push_number(c));
  return AP_OK;
}

AP_API int ap_particles_modified(ap_ctx *c, size_t number) {
  if (!c || !c->ptc_bound) return AP_ERR_INVALID;
  if (number > c->capacity) return fail(c, AP_ERR_CAPACITY);
  c->number = number;
  c->store_base = 0;
  c->order_valid = false;
  c->scale_valid = false;
  AP_TRY_ST(push_number(c));
  return AP_OK;
}

AP_API int ap_get_number(const ap_ctx *c, size_t *n) {
  if (!c || !n) return AP_ERR_INVALID;
  if (refresh_number(const_cast<ap_ctx *>(c)) != AP_OK) return AP_ERR_CUDA;
  *n = c->number;
  return AP_OK;
}

AP_API int ap_get_slot_range(const ap_ctx *c, size_t *first, size_t *end) {
  if (!c || !first || !end) return AP_ERR_INVALID;
  if (refresh_number(const_cast<ap_ctx *>(c)) != AP_OK) return AP_ERR_CUDA;
  *first = c->store_base;
  *end = c->number;
  return AP_OK;
}

AP_API int ap_smooth_array(ap_ctx *c, ap_array a) {
  if (!c || !c->fields_bound || !valid_array(a, c->mesh)) return AP_ERR_INVALID;
  int bnd[4] = {!c->params.periodic[0], !c->params.periodic[0], !c->params.periodic[1],
                !c->params.periodic[1]};
  AP_TRY(launch_filter(*c, a, bnd));
  return finish(c);
}

static int smooth_current_async(Ctx *c, uint32_t step) {
  int bnd[4] = {!c->params.periodic[0], !c->params.periodic[0], !c->params.periodic[1],
                !c->params.periodic[1]};
  const bool out = ((step + 1) % (uint32_t)c->params.data_interval) == 0;
  for (int it = 0; it < c->params.current_smoothing; ++it) {
    for (int k = 0; k < 3; ++k) AP_TRY(launch_filter(*c, c->fields.J[k], bnd));
    for (int k = 0; k < 3; ++k) AP_TRY(launch_copy_guards(*c, c->fields.J[k]));
    if (out)
      for (int s = 0; s < c->params.num_species; ++s) {
        AP_TRY(launch_filter(*c, c->fields.Rho[s], bnd));
        AP_TRY(launch_copy_guards(*c, c->fields.Rho[s]));
      }
  }
  return AP_OK;
}

AP_API int ap_smooth_current(ap_ctx *c, uint32_t step) {
  if (!c || !c->fields_bound) return AP_ERR_INVALID;
  if (c->coord == 1) {
    AP_TRY(launch_ls_smooth(*c, ((step + 1) % (uint32_t)c->params.data_interval) == 0));
    return finish(c);
  }
  AP_TRY_ST(smooth_current_async(c, step));
  return finish(c);
}

}  // extern "C"

namespace apb {

// ptc_updater_1dgap::update_particles (ptc_updater_1dgap.cu:219-272).
int update_particles_gap(Ctx *c, double dt, uint32_t step) {
  const ap_params &pr = c->params;
  // without particles nothing but the photons moves (:226, :272-278)
  if (c->number == 0) {
    if (c->ph_bound) AP_TRY_ST(rad_move_photons(*c, (float)dt, step));
    return finish(c);
  }
  const int ncomp = 3 + pr.num_species;
  const int n = c->mesh.dims[0];
  const int bl = !pr.periodic[0], bu = !pr.periodic[0];  // is_boundary(0), (1)
  int ph = phase_begin(c, kPhFinalize);
  // J and Rho are zeroed (:227-230); the finalize writes every component
  AP_TRY(cudaMemsetAsync(c->acc, 0, sizeof(unsigned long long) * c->acc_comp * ncomp,
                         c->stream));
  if (!c->scale_valid) AP_TRY(launch_fixed_scale(*c));
  AP_TRY(cudaMemsetAsync(c->status, 0, sizeof(DevStatus), c->stream));
  // E3 = E1, smoothed current_smoothing times through E2 (:232-240)
  float *E1 = c->fields.E[0].ptr, *E2 = c->fields.E[1].ptr, *E3 = c->fields.E[2].ptr;
  AP_TRY(cudaMemcpyAsync(E3, E1, sizeof(float) * n, cudaMemcpyDeviceToDevice, c->stream));
  for (int it = 0; it < pr.current_smoothing; ++it) {
    AP_TRY(launch_gap_filter(*c, E3, E2, bl, bu));
    AP_TRY(cudaMemcpyAsync(E3, E2, sizeof(float) * n, cudaMemcpyDeviceToDevice, c->stream));
  }
  phase_end(c, ph);
  PushDepositParams P;
  std::memset(&P, 0, sizeof(P));
  P.m = c->mk;
  P.p = PtcK{c->ptc.x1, c->ptc.x2, c->ptc.x3, c->ptc.p1, c->ptc.p2,
             c->ptc.p3, c->ptc.E,  c->ptc.weight, c->ptc.cell, c->ptc.flag};
  P.F[2] = FieldArr{E3, (int)(c->fields.E[2].pitch / 4)};
  P.acc = c->acc;
  P.acc_pitch = c->mesh.dims[0];
  P.acc_comp = c->acc_comp;
  P.fx_used = c->fx_used;
  P.n_max = c->n_max;
  P.wmax = c->wmax;
  P.number = c->number;
  P.status = c->status;
  P.num_species = pr.num_species;
  P.dt = (float)dt;
  P.qmax = 0.0f;
  for (int s = 0; s < AP_MAX_SPECIES; ++s) {
    P.qmax = fmaxf(P.qmax, fabsf(pr.charges[s]));
    P.charge[s] = pr.charges[s];
    P.mass[s] = pr.masses[s];
  }
  // J1 contributions carry delta / dt (:143-144)
  const float kj = c->mesh.delta[0] / (float)dt;
  if (kj > 1.0f) P.qmax *= kj;
  ph = phase_begin(c, kPhPushDeposit);
  AP_TRY(launch_gap_push_deposit(*c, P));
  phase_end(c, ph);
  ph = phase_begin(c, kPhFinalize);
  AP_TRY(launch_finalize_current(*c, ncomp));
  // J1 and each Rho smoothed current_smoothing times (:254-268)
  float *tmp = c->tmp_j;
  for (int it = 0; it < pr.current_smoothing; ++it) {
    AP_TRY(launch_gap_filter(*c, c->fields.J[0].ptr, tmp, bl, bu));
    AP_TRY(cudaMemcpyAsync(c->fields.J[0].ptr, tmp, sizeof(float) * n, cudaMemcpyDeviceToDevice,
                           c->stream));
    for (int s = 0; s < pr.num_species; ++s) {
      AP_TRY(launch_gap_filter(*c, c->fields.Rho[s].ptr, tmp, bl, bu));
      AP_TRY(cudaMemcpyAsync(c->fields.Rho[s].ptr, tmp, sizeof(float) * n,
                             cudaMemcpyDeviceToDevice, c->stream));
    }
  }
  c->rho_is_zero = false;
  phase_end(c, ph);
  // the photons after the particles (:272-278)
  if (c->ph_bound) AP_TRY_ST(rad_move_photons(*c, (float)dt, step));
  return finish(c);
}

// ptc_updater_1dgr::update_particles (ptc_updater_1dgr.cu:418-473).
int update_particles_gr(Ctx *c, double dt, uint32_t step) {
  const ap_params &pr = c->params;
  if (c->number == 0) {
    // without particles nothing but the photons moves (:422, :492-499)
    if (c->ph_bound) AP_TRY_ST(rad_move_photons(*c, (float)dt, step));
    return finish(c);
  }
  const int ncomp = 3 + pr.num_species;
  const int n = c->mesh.dims[0];
  const int bl = !pr.periodic[0], bu = !pr.periodic[0];  // is_boundary(0), (1)
  const float *K1 = coef_array(*c, AP_GR_K1).ptr, *K1j = coef_array(*c, AP_GR_K1_J).ptr;
  int ph = phase_begin(c, kPhFinalize);
  // J and Rho are zeroed (:423-426); the finalize writes every component
  AP_TRY(cudaMemsetAsync(c->acc, 0, sizeof(unsigned long long) * c->acc_comp * ncomp,
                         c->stream));
  if (!c->scale_valid) AP_TRY(launch_fixed_scale(*c));
  AP_TRY(cudaMemsetAsync(c->status, 0, sizeof(DevStatus), c->stream));
  // E3 = E1, smoothed current_smoothing times through E2 with K1_j (:428-435)
  float *E1 = c->fields.E[0].ptr, *E2 = c->fields.E[1].ptr, *E3 = c->fields.E[2].ptr;
  AP_TRY(cudaMemcpyAsync(E3, E1, sizeof(float) * n, cudaMemcpyDeviceToDevice, c->stream));
  for (int it = 0; it < pr.current_smoothing; ++it) {
    AP_TRY(launch_gr_filter(*c, E3, E2, K1j, bl, bu));
    AP_TRY(cudaMemcpyAsync(E3, E2, sizeof(float) * n, cudaMemcpyDeviceToDevice, c->stream));
  }
  phase_end(c, ph);
  PushDepositParams P;
  std::memset(&P, 0, sizeof(P));
  P.m = c->mk;
  P.p = PtcK{c->ptc.x1, c->ptc.x2, c->ptc.x3, c->ptc.p1, c->ptc.p2,
             c->ptc.p3, c->ptc.E,  c->ptc.weight, c->ptc.cell, c->ptc.flag};
  P.F[2] = FieldArr{E3, (int)(c->fields.E[2].pitch / 4)};
  P.acc = c->acc;
  P.acc_pitch = c->mesh.dims[0];
  P.acc_comp = c->acc_comp;
  P.fx_used = c->fx_used;
  P.n_max = c->n_max;
  P.wmax = c->wmax;
  P.number = c->number;
  P.status = c->status;
  P.num_species = pr.num_species;
  P.dt = (float)dt;
  P.qmax = 0.0f;
  for (int s = 0; s < AP_MAX_SPECIES; ++s) {
    P.qmax = fmaxf(P.qmax, fabsf(pr.charges[s]));
    P.charge[s] = pr.charges[s];
    P.mass[s] = pr.masses[s];
  }
  // J1 contributions carry delta / (dt K1_j), Rho ones 1 / K1 (:280-288)
  const float kj = c->gr_kfac * c->mesh.delta[0] / (float)dt;
  P.qmax *= fmaxf(1.0f, fmaxf(kj, c->gr_kfac));
  GrK G;
  G.D1 = coef_array(*c, AP_GR_D1).ptr;
  G.D2 = coef_array(*c, AP_GR_D2).ptr;
  G.D3 = coef_array(*c, AP_GR_D3).ptr;
  G.alpha = coef_array(*c, AP_GR_ALPHA).ptr;
  G.theta = coef_array(*c, AP_GR_THETA).ptr;
  G.K1 = K1;
  G.K1_j = K1j;
  G.agrr = coef_array(*c, AP_GR_AGRR).ptr;
  G.B3B1 = coef_array(*c, AP_GR_B3B1).ptr;
  G.a = c->gr.a;
  G.omega = c->gr.omega;
  G.step = step;
  G.data_interval = pr.data_interval;
  ph = phase_begin(c, kPhPushDeposit);
  AP_TRY(launch_gr_push_deposit(*c, P, G));
  phase_end(c, ph);
  ph = phase_begin(c, kPhFinalize);
  AP_TRY(launch_finalize_current(*c, ncomp));
  // J1 (K1_j) and each Rho (K1) smoothed current_smoothing times (:447-466)
  float *tmp = c->tmp_j;
  for (int it = 0; it < pr.current_smoothing; ++it) {
    AP_TRY(launch_gr_filter(*c, c->fields.J[0].ptr, tmp, K1j, bl, bu));
    AP_TRY(cudaMemcpyAsync(c->fields.J[0].ptr, tmp, sizeof(float) * n, cudaMemcpyDeviceToDevice,
                           c->stream));
    for (int s = 0; s < pr.num_species; ++s) {
      AP_TRY(launch_gr_filter(*c, c->fields.Rho[s].ptr, tmp, K1, bl, bu));
      AP_TRY(cudaMemcpyAsync(c->fields.Rho[s].ptr, tmp, sizeof(float) * n,
                             cudaMemcpyDeviceToDevice, c->stream));
    }
  }
  c->rho_is_zero = false;
  phase_end(c, ph);
  // the photons after the particles (:492-499)
  if (c->ph_bound) AP_TRY_ST(rad_move_photons(*c, (float)dt, step));
  if (!c->sync) return AP_OK;
  return check_status(c);  // AP_ERR_MOVED_FAR
}

// First part of an update: zero the accumulators, refresh the weight bound
// and the tile order if needed, and fill the kernel parameters. Returns
// AP_OK; *has_work is false when there are no particles.
int update_prepare(Ctx *c, double dt, uint32_t step, PushDepositParams &P, bool *has_work,
                   bool batched) {
  const ap_params &pr = c->params;
  const bool do_rho = ((step + 1) % (uint32_t)pr.data_interval) == 0;
  // data.J.initialize(); data.Rho[i].initialize() (ptc_updater.cu:752-755):
  // the FP64 accumulators start at zero; J (and Rho on output steps) are
  // overwritten by the finalize pass, Rho is zeroed on other steps.
  const int ncomp = 3 + (do_rho ? pr.num_species : 0);
  const bool ls = c->coord == 1;
  int ph = phase_begin(c, kPhFinalize);
  if (!batched)
    AP_TRY(cudaMemsetAsync(c->acc, 0, sizeof(unsigned long long) * c->acc_comp * ncomp,
                           c->stream));
  if (!c->scale_valid) AP_TRY(launch_fixed_scale(*c));
  // Rho keeps the zeros of the last step without charge deposition
  if (!do_rho && !ls && !c->rho_is_zero) {
    for (int s = 0; s < pr.num_species; ++s) AP_TRY(launch_zero(*c, c->fields.Rho[s]));
    c->rho_is_zero = true;
  }
  if (!batched) AP_TRY(cudaMemsetAsync(c->status, 0, sizeof(DevStatus), c->stream));
  // continuity check: rho(t) of the previous update, before it is replaced
  c->cont_snap = false;
  if (c->cont_on && !batched && !ls && do_rho && c->last_rho_step == (long long)step - 1) {
    AP_TRY(launch_rho_snapshot(*c));
    c->cont_snap = true;
  }
  phase_end(c, ph);

  std::memset(&P, 0, sizeof(P));
  // with a device-side count, 1D kernels work over the capacity and read
  // the live count on the device; 2D needs the host count for the order
  const bool device_count = c->pstate && c->mk.dim == 1;
  if (c->pstate && !device_count) AP_TRY_ST(refresh_number(c));
  *has_work = device_count ? c->capacity > 0 : c->number > 0;
  if (*has_work) {
    P.m = c->mk;
    P.p = PtcK{c->ptc.x1, c->ptc.x2, c->ptc.x3, c->ptc.p1, c->ptc.p2,
               c->ptc.p3, c->ptc.E,  c->ptc.weight, c->ptc.cell, c->ptc.flag};
    const ap_array *fa[6] = {&c->fields.E[0], &c->fields.E[1], &c->fields.E[2],
                             &c->fields.B[0], &c->fields.B[1], &c->fields.B[2]};
    for (int k = 0; k < 6; ++k) P.F[k] = FieldArr{fa[k]->ptr, (int)(fa[k]->pitch / 4)};
    for (int k = 0; k < 3; ++k)
      P.J[k] = FieldArr{c->fields.J[k].ptr, (int)(c->fields.J[k].pitch / 4)};
    for (int s = 0; s < pr.num_species; ++s)
      P.Rho[s] = FieldArr{c->fields.Rho[s].ptr, (int)(c->fields.Rho[s].pitch / 4)};
    P.acc = c->acc;
    P.acc_pitch = c->mesh.dims[0];
    P.acc_comp = c->acc_comp;
    P.fx_used = c->fx_used;
    P.n_max = c->n_max;
    P.wmax = c->wmax;
    P.qmax = 0.0f;
    for (int s = 0; s < AP_MAX_SPECIES; ++s) P.qmax = fmaxf(P.qmax, fabsf(pr.charges[s]));
    // The kernel receives dt as float (Scalar dt); q_over_m is evaluated as
    // dt * 0.5f * q / m (ptc_updater.cu:42, 101).
    const float dtf = (float)dt;
    P.dt = dtf;
    for (int s = 0; s < AP_MAX_SPECIES; ++s) {
      volatile float a = dtf * 0.5f;
      volatile float b = a * pr.charges[s];
      P.qm[s] = pr.masses[s] != 0.0f ? b / pr.masses[s] : 0.0f;
      P.charge[s] = pr.charges[s];
    }
    P.num_species = pr.num_species;
    P.do_rho = do_rho ? 1 : 0;
    for (int d = 0; d < 3; ++d) P.periodic[d] = pr.periodic[d];
    P.status = c->status;
    P.number = device_count ? c->capacity : c->number;
    P.d_number = device_count ? &c->pstate->number : nullptr;
    if (ls) {
      // user_push_2d_logsph / deposit_and_move_2d_log_sph parameters; the
      // J3 contributions are divided by the cell volume, which widens the
      // fixed-point range by ls_kfac
      P.ls_compactness = c->lsp.compactness;
      P.ls_omega = c->lsp.omega;
      P.ls_gravity = c->lsp.gravity;
      P.ls_rad_coef = c->lsp.rad_cooling_coef;
      P.ls_B0 = c->lsp.B0;
      P.ls_rad_on = c->lsp.rad_cooling_on;
      P.ls_outflow_c1 = c->mesh.dims[0] - c->lsp.damping_length + 2;
      for (int s = 0; s < AP_MAX_SPECIES; ++s) P.mass[s] = pr.masses[s];
      const ap_array dv = coef_array(*c, AP_COEF_DV);
      P.dV = FieldArr{dv.ptr, (int)(dv.pitch / 4)};
      P.qmax *= c->ls_kfac;
    }
    if (c->mk.dim == 2) {
      if (!c->order_valid) {
        ph = phase_begin(c, kPhRebuild);
        AP_TRY(rebuild_tile_order(*c));
        phase_end(c, ph);
        c->since_compact = 0;
      }
      c->compact_now = false;
      if (c->compact_interval > 0 && incremental_order(*c) &&
          ++c->since_compact >= c->compact_interval) {
        // this update writes the store in tile order (into the scratch
        // store, copied back after the order update)
        AP_TRY(compact_store(*c, &P.cout, &P.cout_id));
        P.id = c->ptc.id;
        c->compact_now = true;
        c->since_compact = 0;
      }
      // per-chunk direction counts for the one-pass order update
      c->chunk_count_ok = false;
      if (incremental_order(*c)) {
        const size_t need = c->order_cap / (size_t)chunk_of(*c) + c->tiles.ntiles + 2;
        if (c->chunk_count_cap < need) {
          cudaFree(c->chunk_count);
          c->chunk_count = nullptr;
          c->chunk_count_cap = 0;
          AP_TRY(cudaMalloc(&c->chunk_count, sizeof(uint32_t) * 10 * need));
          c->chunk_count_cap = need;
        }
        if (c->big_tiles_cap < (size_t)c->tiles.ntiles + 1) {
          cudaFree(c->big_tiles);
          c->big_tiles = nullptr;
          c->big_tiles_cap = 0;
          AP_TRY(cudaMalloc(&c->big_tiles, sizeof(uint32_t) * (c->tiles.ntiles + 1)));
          c->big_tiles_cap = c->tiles.ntiles + 1;
        }
        P.chunk_count = c->chunk_count;
        c->chunk_count_ok = true;
      }
      P.t = c->tiles;
      P.order = c->order[c->cur];
      P.tile_start = c->tile_start[c->cur];
      P.dir = c->dir;
      P.dir_count = c->dir_count;
      P.queue = c->queue;
    }
  }
  return AP_OK;
}

// Last part: the tile-order update from the directions the kernel wrote,
// then rounding (and folding / process_j) of the current and smoothing.
int update_complete(Ctx *c, double dt, uint32_t step, bool had_work, bool batched) {
  const ap_params &pr = c->params;
  const bool do_rho = ((step + 1) % (uint32_t)pr.data_interval) == 0;
  const int ncomp = 3 + (do_rho ? pr.num_species : 0);
  const bool ls = c->coord == 1;
  if (do_rho || ls) c->rho_is_zero = false;  // the finalize writes Rho
  int ph;
  if (had_work && c->mk.dim == 2) {
    if (incremental_order(*c)) {
      const int nxt = c->cur ^ 1;
      ph = phase_begin(c, kPhOrder);
      AP_TRY(launch_tile_scan(*c, c->dir_count, c->tile_start[nxt], c->grp_off));
      // after a compacting push the particle at list position q sits in
      // slot compact_dst + q
      AP_TRY(launch_order_scatter(*c, c->tile_start[c->cur],
                                  c->compact_now ? nullptr : c->order[c->cur], c->dir,
                                  c->grp_off, c->order[nxt], (uint32_t)c->compact_dst));
      phase_end(c, ph);
      if (c->compact_now) {
        ph = phase_begin(c, kPhSort);
        AP_TRY(compact_finish(*c, c->tile_start[c->cur] + c->tiles.ntiles));
        phase_end(c, ph);
        c->compact_now = false;
        c->compact_dst = 0;
      }
      c->cur = nxt;
    } else {
      c->order_valid = false;
    }
  }
  if (batched && c->mk.dim == 1 && !ls) return AP_OK;  // batched finalize and smoothing
  ph = phase_begin(c, kPhFinalize);
  if (ls) {
    // process_j, then (ptc_updater_logsph::apply_boundary) axis_rho after
    // the smoothing; particles that left the bulk were dropped by the move
    // and ptc_outflow was applied there too
    AP_TRY(launch_ls_finalize(*c, (float)dt, do_rho, pr.current_smoothing == 0));
    if (pr.current_smoothing > 0) AP_TRY(launch_ls_smooth(*c, do_rho));
    phase_end(c, ph);
  } else {
    // send_add_guard_cells(J), and Rho on output steps (ptc_updater.cu:800-805),
    // fused with the rounding of the exact sums
    AP_TRY(launch_finalize_current(*c, ncomp));
    phase_end(c, ph);
    AP_TRY_ST(smooth_current_async(c, step));
    if (c->cont_on && !batched) {
      if (c->cont_snap)
        AP_TRY(launch_continuity(*c, c->diag_dev + 6));
      else
        AP_TRY(cudaMemsetAsync(c->diag_dev + 6, 0xFF, sizeof(double), c->stream));  // NaN
      c->last_rho_step = do_rho ? (long long)step : -2;
    }
  }
  return AP_OK;
}

int ctx_check_status(Ctx *c) { return check_status(c); }

int update_smooth(Ctx *c, uint32_t step) { return smooth_current_async(c, step); }

int fill_run1d(Ctx *c, double dt, uint32_t step, Run1D &d) {
  std::memset(&d, 0, sizeof(d));
  const ap_mesh &m = c->mesh;
  const ap_fields &f = c->fields;
  auto fa = [](const ap_array &a) { return FieldArr{a.ptr, (int)(a.pitch / sizeof(float))}; };
  d.n0 = m.dims[0];
  d.g0 = m.guard[0];
  d.r0 = m.dims[0] - 2 * m.guard[0];
  d.per0 = c->params.periodic[0];
  d.id0 = m.inv_delta[0];
  for (int k = 0; k < 3; ++k) {
    d.E[k] = fa(f.E[k]);
    d.B[k] = fa(f.B[k]);
    d.Eb[k] = fa(f.Ebg[k]);
    d.Bb[k] = fa(f.Bbg[k]);
    d.J[k] = fa(f.J[k]);
  }
  for (int s = 0; s < c->params.num_species; ++s) d.Rho[s] = fa(f.Rho[s]);
  d.divE = fa(f.divE);
  d.divB = fa(f.divB);
  d.has_divs = f.divE.ptr && f.divB.ptr;
  d.acc = c->acc;
  d.acc_comp = c->acc_comp;
  d.fx = c->fx_used;
  const bool do_rho = ((step + 1) % (uint32_t)c->params.data_interval) == 0;
  d.ncomp = 3 + (do_rho ? c->params.num_species : 0);
  d.zero_comps = d.ncomp;
  d.dt = (float)dt;
  d.dt_half = step == 0 ? (float)(0.5 * dt) : 0.0f;
  d.step = step;
  if (c->pstate && c->pair.enabled) {
    if (ensure_pair_scratch(*c) != AP_OK) return AP_ERR_NOMEM;
    d.counts = c->pair_chunks;
    d.offs = c->pair_chunks + c->pair_cap_chunks;
    d.tot = d.offs + c->pair_cap_chunks;
    d.gamma_thr = c->pair.gamma_thr;
    d.free_path = c->pair.free_path;
    d.pair_energy = c->pair.pair_energy;
    d.pair_dt = (float)dt;
    d.key[0] = (uint32_t)c->pair.seed;
    d.key[1] = (uint32_t)(c->pair.seed >> 32);
    d.p = PtcK{c->ptc.x1, c->ptc.x2, c->ptc.x3, c->ptc.p1, c->ptc.p2,
               c->ptc.p3, c->ptc.E,  c->ptc.weight, c->ptc.cell, c->ptc.flag};
    d.ids = c->ptc.id;
    d.pst = c->pstate;
    d.emit = c->dir;
    d.capacity = c->capacity;
  }
  return AP_OK;
}

}  // namespace apb

extern "C" {

AP_API int ap_update_particles(ap_ctx *c, double dt, uint32_t step) {
  if (!c || !c->fields_bound || !c->ptc_bound) return AP_ERR_INVALID;
  if (c->coord == 2) return update_particles_gap(c, dt, step);
  if (c->coord == 3) return update_particles_gr(c, dt, step);
  PushDepositParams P;
  bool has_work = false;
  AP_TRY_ST(update_prepare(c, dt, step, P, &has_work));
  if (has_work) {
    const int ph = phase_begin(c, kPhPushDeposit);
    AP_TRY(c->mk.dim == 1 ? launch_push_deposit_1d(*c, P) : launch_push_deposit_2d(*c, P));
    phase_end(c, ph);
    c->pd_launches++;
  }
  AP_TRY_ST(update_complete(c, dt, step, has_work));
  // photons move after the particles (ptc_updater.cu:814-833,
  // ptc_updater_logsph.cu:793-803)
  if (c->ph_bound) AP_TRY_ST(rad_move_photons(*c, (float)dt, step));
  if (!c->sync) return AP_OK;
  return check_status(c);
}

AP_API int ap_update_e_field(ap_ctx *c, double dt) {
  if (!c || !c->fields_bound) return AP_ERR_INVALID;
  AP_TRY(c->coord == 1 ? launch_ls_update_e(*c, (float)dt) : launch_update_e(*c, (float)dt));
  return finish(c);
}

AP_API int ap_update_b_field(ap_ctx *c, double dt) {
  if (!c || !c->fields_bound) return AP_ERR_INVALID;
  AP_TRY(c->coord == 1 ? launch_ls_update_b(*c, (float)dt) : launch_update_b(*c, (float)dt));
  return finish(c);
}

AP_API int ap_compute_divs(ap_ctx *c) {
  if (!c || !c->fields_bound) return AP_ERR_INVALID;
  AP_TRY(c->coord == 1 ? launch_ls_divs(*c) : launch_divs(*c));
  return finish(c);
}

AP_API int ap_update_fields(ap_ctx *c, double dt, uint32_t step) {
  if (!c || !c->fields_bound) return AP_ERR_INVALID;
  const int ph = phase_begin(c, kPhFields);
  if (c->coord == 2) {
    // field_solver_1dgap::update_fields (field_solver_1dgap.cu:28-40)
    AP_TRY(launch_gap_update_e(*c, (float)(c->gap.B0 * 1.6), (float)dt));
    phase_end(c, ph);
    return finish(c);
  }
  if (c->coord == 3) {
    // field_solver_1dgr::update_fields (field_solver_1dgr.cu:29-44)
    AP_TRY(launch_gr_update_e(*c, coef_array(*c, AP_GR_J0).ptr, (float)dt));
    phase_end(c, ph);
    return finish(c);
  }
  if (c->coord == 1) {
    // field_solver_logsph::update_fields (field_solver_logsph.cu:354-398):
    // B, then E, then the divergences; no guard exchange on a
    // non-periodic grid (EdotB is not computed)
    AP_TRY(launch_ls_update_b(*c, (float)dt));
    AP_TRY(launch_ls_update_e(*c, (float)dt));
    AP_TRY(launch_ls_divs(*c));
    phase_end(c, ph);
    return finish(c);
  }
  // field_solver::update_fields (field_solver.cu:334-358)
  if (step == 0) AP_TRY(launch_update_e(*c, (float)(0.5 * dt)));
  AP_TRY(launch_update_b(*c, (float)dt));
  AP_TRY(launch_update_e(*c, (float)dt));
  AP_TRY(launch_divs(*c));
  phase_end(c, ph);
  return finish(c);
}

AP_API int ap_send_guard_cells(ap_ctx *c, ap_array a) {
  if (!c || !valid_array(a, c->mesh)) return AP_ERR_INVALID;
  AP_TRY(launch_copy_guards(*c, a));
  return finish(c);
}

AP_API int ap_send_add_guard_cells(ap_ctx *c, ap_array a) {
  if (!c || !valid_array(a, c->mesh)) return AP_ERR_INVALID;
  AP_TRY(launch_fold_guards(*c, a));
  return finish(c);
}

AP_API int ap_sort_by_cell(ap_ctx *c) {
  if (!c || !c->ptc_bound) return AP_ERR_INVALID;
  size_t n = 0;
  // a 1D context with a device-side count sorts over its capacity and keeps
  // the count on the device (no host synchronisation)
  const bool device_count = c->pstate && c->mk.dim == 1;
  if (!device_count) AP_TRY_ST(refresh_number(c));
  const int ph = phase_begin(c, kPhSort);
  AP_TRY(sort_by_cell(*c, &n));  // also leaves the 2D tile order of the sorted store
  if (c->ph_bound) {
    // sim_data::sort_particles sorts the photons too (sim_data_impl.hpp:78-82)
    size_t nph = 0;
    AP_TRY(sort_photons(*c, &nph));
    c->ph_number = nph;
  }
  phase_end(c, ph);
  if (!device_count) {
    c->number = n;  // sort_by_cell set store_base
    AP_TRY_ST(push_number(c));
  }
  return AP_OK;
}

AP_API int ap_get_tile_order(ap_ctx *c, const uint32_t **order, const uint32_t **tile_start,
                             uint32_t *ntiles, size_t *live) {
  if (!c || !c->ptc_bound || c->mk.dim != 2) return AP_ERR_INVALID;
  if (!c->order_valid) AP_TRY(rebuild_tile_order(*c));
  uint32_t n = 0;
  AP_TRY(cudaMemcpyAsync(&n, c->tile_start[c->cur] + c->tiles.ntiles, sizeof(uint32_t),
                         cudaMemcpyDeviceToHost, c->stream));
  AP_TRY(cudaStreamSynchronize(c->stream));
  if (order) *order = c->order[c->cur];
  if (tile_start) *tile_start = c->tile_start[c->cur];
  if (ntiles) *ntiles = (uint32_t)c->tiles.ntiles;
  if (live) *live = n;
  return AP_OK;
}

AP_API int ap_get_stats(ap_ctx *c, ap_step_stats *s) {
  if (!c || !s) return AP_ERR_INVALID;
  AP_TRY_ST(refresh_number(c));
  AP_TRY(cudaMemcpyAsync(c->status_host, c->status, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                         c->stream));
  AP_TRY(cudaStreamSynchronize(c->stream));
  s->nan_momenta = c->status_host->nan_momenta;
  s->moved_far = c->status_host->moved_far;
  s->lost = c->status_host->lost;
  s->tile_faults = c->status_host->tile_faults;
  s->live = 0;
  if (c->mk.dim == 2 && c->order_valid) {
    uint32_t n = 0;
    AP_TRY(cudaMemcpy(&n, c->tile_start[c->cur] + c->tiles.ntiles, sizeof(uint32_t),
                      cudaMemcpyDeviceToHost));
    s->live = n;
  }
  return AP_OK;
}

AP_API int ap_diagnostics(ap_ctx *c, ap_diag *out) {
  if (!c || !out || !c->fields_bound || !c->ptc_bound) return AP_ERR_INVALID;
  AP_TRY_ST(refresh_number(c));
  AP_TRY(launch_diagnostics(*c, c->diag_dev));
  AP_TRY(cudaMemcpyAsync(c->diag_host, c->diag_dev, sizeof(double) * 7, cudaMemcpyDeviceToHost,
                         c->stream));
  AP_TRY(cudaStreamSynchronize(c->stream));
  out->kinetic = c->diag_host[0];
  out->charge = c->diag_host[1];
  out->field_energy = c->diag_host[2];
  out->max_abs_rho = c->diag_host[3];
  out->gauss_residual = c->diag_host[4];
  out->max_abs_j = c->diag_host[5];
  out->continuity_residual = c->diag_host[6];
  return AP_OK;
}

AP_API int ap_diagnostics_async(ap_ctx *c, double *host_out) {
  if (!c || !host_out || !c->fields_bound || !c->ptc_bound) return AP_ERR_INVALID;
  if (c->pstate && c->mk.dim == 1 && c->number_stale) return fail(c, AP_ERR_INVALID);
  AP_TRY(launch_diagnostics(*c, c->diag_dev));
  AP_TRY(cudaMemcpyAsync(host_out, c->diag_dev, sizeof(double) * 7, cudaMemcpyDeviceToHost,
                         c->stream));
  return AP_OK;
}

AP_API int ap_selftest_wait_timeout(ap_ctx *c) {
  if (!c) return AP_ERR_INVALID;
  AP_TRY(cudaMemsetAsync(c->status, 0, sizeof(DevStatus), c->stream));
  AP_TRY(launch_selftest_wait(*c, 1u << 12));
  return check_status(c);
}

AP_API int ap_set_profiling(ap_ctx *c, int on) {
  if (!c) return AP_ERR_INVALID;
  c->profiling = on != 0;
  return AP_OK;
}

AP_API int ap_get_phase_times(ap_ctx *c, ap_phase_times *out, int reset) {
  if (!c || !out) return AP_ERR_INVALID;
  AP_TRY(cudaStreamSynchronize(c->stream));
  double t[kPhN] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < c->ev_used; ++i) {
    float ms = 0.0f;
    AP_TRY(cudaEventElapsedTime(&ms, c->ev[i].a, c->ev[i].b));
    t[c->ev[i].phase] += ms;
  }
  out->push_deposit_ms = t[kPhPushDeposit];
  out->order_ms = t[kPhOrder];
  out->rebuild_ms = t[kPhRebuild];
  out->finalize_ms = t[kPhFinalize];
  out->fields_ms = t[kPhFields];
  out->sort_ms = t[kPhSort];
  out->push_deposit_launches = c->pd_launches;
  if (reset) {
    c->ev_used = 0;
    c->pd_launches = 0;
  }
  return AP_OK;
}

AP_API int ap_ctx_create_logsph(const ap_mesh *mesh, const ap_params *params,
                                const ap_logsph_params *lsp, ap_ctx **out) {
  if (!mesh || !params || !lsp || !out) return AP_ERR_INVALID;
  *out = nullptr;
  const MeshK mk = make_meshk(*mesh);
  if (mk.dim != 2) return AP_ERR_UNSUPPORTED;
  if (params->periodic[0] || params->periodic[1]) return AP_ERR_UNSUPPORTED;
  if (lsp->damping_length < 0 || lsp->damping_length > mesh->dims[0]) return AP_ERR_INVALID;
  ap_ctx *c = nullptr;
  int st = ap_ctx_create(mesh, params, &c);
  if (st != AP_OK) return st;
  c->coord = 1;
  c->lsp = *lsp;
  st = logsph_setup(*c);
  if (st != AP_OK) {
    ap_ctx_destroy(c);
    return st;
  }
  *out = c;
  return AP_OK;
}

AP_API int ap_ctx_create_1dgap(const ap_mesh *mesh, const ap_params *params,
                               const ap_gap_params *gap, ap_ctx **out) {
  if (!mesh || !params || !gap || !out) return AP_ERR_INVALID;
  *out = nullptr;
  if (make_meshk(*mesh).dim != 1) return AP_ERR_UNSUPPORTED;
  ap_ctx *c = nullptr;
  int st = ap_ctx_create(mesh, params, &c);
  if (st != AP_OK) return st;
  c->coord = 2;
  c->gap = *gap;
  *out = c;
  return AP_OK;
}

AP_API int ap_ctx_create_1dgr(const ap_mesh *mesh, const ap_params *params,
                              const ap_gr_params *gr, const ap_gr_table *table, ap_ctx **out) {
  if (!mesh || !params || !gr || !table || !out) return AP_ERR_INVALID;
  *out = nullptr;
  if (make_meshk(*mesh).dim != 1) return AP_ERR_UNSUPPORTED;
  if (table->n < 2 || !table->r || !table->B1 || !table->B3 || !table->jr || !table->rho ||
      !table->theta || !table->dpsidth)
    return AP_ERR_INVALID;
  std::vector<float> co[AP_GR_NCOEF];
  host_gr_coef(*mesh, *gr, *table, co);
  // largest 1 / |K1| and 1 / |K1_j| the deposit can divide by
  float kfac = 0.0f;
  for (int k : {AP_GR_K1, AP_GR_K1_J})
    for (float v : co[k])
      if (v != 0.0f && std::isfinite(1.0f / v)) kfac = fmaxf(kfac, fabsf(1.0f / v));
  ap_ctx *c = nullptr;
  int st = ap_ctx_create(mesh, params, &c);
  if (st != AP_OK) return st;
  c->coord = 3;
  c->gr = *gr;
  c->gr_kfac = kfac > 0.0f ? kfac : 1.0f;
  const size_t n0 = (size_t)mesh->dims[0];
  c->coef_pitch = n0 * sizeof(float);
  if (cudaMalloc(&c->coef, c->coef_pitch * AP_GR_NCOEF) != cudaSuccess) {
    c->coef = nullptr;
    ap_ctx_destroy(c);
    return AP_ERR_NOMEM;
  }
  for (int k = 0; k < AP_GR_NCOEF; ++k)
    if (cudaMemcpy(reinterpret_cast<char *>(c->coef) + k * c->coef_pitch, co[k].data(),
                   c->coef_pitch, cudaMemcpyHostToDevice) != cudaSuccess) {
      ap_ctx_destroy(c);
      return AP_ERR_CUDA;
    }
  *out = c;
  return AP_OK;
}

AP_API int ap_gr_coef(ap_ctx *c, int which, ap_array *out) {
  if (!c || !out || c->coord != 3 || which < 0 || which >= AP_GR_NCOEF) return AP_ERR_INVALID;
  *out = coef_array(*c, which);
  return AP_OK;
}

AP_API int ap_logsph_coef(ap_ctx *c, int which, ap_array *out) {
  if (!c || !out || c->coord != 1 || which < 0 || which >= AP_NUM_COEF) return AP_ERR_INVALID;
  *out = coef_array(*c, which);
  return AP_OK;
}

AP_API int ap_logsph_inject(ap_ctx *c, int inj_per_cell, float p1, float p2, float p3,
                            float w, float omega, uint64_t seed) {
  (void)p2;  // the reference's kernel sets p2 from p1 and theta, p3 to 0,
  (void)p3;  // and leaves omega unused (ptc_updater_logsph.cu:341-367)
  (void)omega;
  if (!c || c->coord != 1 || !c->ptc_bound || inj_per_cell < 0) return AP_ERR_INVALID;
  const int red = c->mesh.dims[1] - 2 * c->mesh.guard[1];
  const size_t add = (size_t)2 * inj_per_cell * red;
  if (c->number + add > c->capacity) return fail(c, AP_ERR_CAPACITY);
  if (!c->ls_surface) AP_TRY(cudaMalloc(&c->ls_surface, sizeof(double) * 2 * red));
  AP_TRY(launch_ls_inject(*c, inj_per_cell, p1, w, seed, c->inject_calls, c->inject_next_id,
                          c->ls_surface));
  c->inject_calls++;
  c->inject_next_id += add;
  c->number += add;
  c->order_valid = false;
  c->scale_valid = false;
  return finish(c);
}

AP_API int ap_logsph_field_boundary(ap_ctx *c, double omega) {
  if (!c || !c->fields_bound || c->coord != 1) return AP_ERR_INVALID;
  AP_TRY(launch_ls_field_boundary(*c, (float)omega));
  return finish(c);
}

AP_API int ap_set_pair_params(ap_ctx *c, const ap_pair_params *pp) {
  if (!c || !pp) return AP_ERR_INVALID;
  if (pp->enabled && (!(pp->free_path > 0.0f) || !(pp->pair_energy >= 0.0f) ||
                      !(pp->gamma_thr > pp->pair_energy + 1.0f)))
    return fail(c, AP_ERR_INVALID);
  AP_TRY_ST(refresh_number(c));
  if (!c->pstate) {
    AP_TRY(cudaMalloc(&c->pstate, sizeof(PairState)));
    AP_TRY(cudaMallocHost(reinterpret_cast<void **>(&c->pstate_host), sizeof(PairState)));
  }
  c->pair = *pp;
  // the device state starts from the host count and the given first id
  PairState s{};
  s.number = (uint32_t)c->number;
  s.next_id = pp->first_id;
  AP_TRY(cudaStreamSynchronize(c->stream));
  AP_TRY(cudaMemcpy(c->pstate, &s, sizeof(s), cudaMemcpyHostToDevice));
  c->number_stale = false;
  return AP_OK;
}

AP_API int ap_get_pair_stats(ap_ctx *c, uint64_t *particle_steps, uint64_t *emitted_total,
                             uint64_t *dropped_total) {
  if (!c) return AP_ERR_INVALID;
  if (!c->pstate) {
    if (particle_steps) *particle_steps = 0;
    if (emitted_total) *emitted_total = 0;
    if (dropped_total) *dropped_total = 0;
    return AP_OK;
  }
  c->number_stale = true;
  AP_TRY_ST(refresh_number(c));
  if (particle_steps) *particle_steps = c->pstate_host->particle_steps;
  if (emitted_total) *emitted_total = c->pstate_host->emitted_total;
  if (dropped_total) *dropped_total = c->pstate_host->dropped_total;
  return AP_OK;
}

AP_API int ap_inject_pairs(ap_ctx *c, double dt, uint32_t step, uint64_t *emitted,
                           uint64_t *dropped) {
  if (!c || !c->ptc_bound) return AP_ERR_INVALID;
  if (emitted) *emitted = 0;
  if (dropped) *dropped = 0;
  if (!c->pair.enabled) return AP_OK;
  AP_TRY_ST(enqueue_pairs(*c, (float)dt, step));
  AP_TRY_ST(refresh_number(c));
  if (emitted) *emitted = c->pstate_host->emitted;
  if (dropped) *dropped = c->pstate_host->dropped;
  return AP_OK;
}

AP_API int ap_bind_photons(ap_ctx *c, const ap_photons *ph, size_t number, size_t capacity) {
  if (!c || !ph) return AP_ERR_INVALID;
  if (number > capacity || capacity >= (size_t)UINT32_MAX) return fail(c, AP_ERR_CAPACITY);
  if (!ph->x1 || !ph->x2 || !ph->x3 || !ph->p1 || !ph->p2 || !ph->p3 || !ph->E ||
      !ph->weight || !ph->path_left || !ph->cell || !ph->id || !ph->flag)
    return fail(c, AP_ERR_INVALID);
  c->ph = *ph;
  c->ph_number = number;
  c->ph_capacity = capacity;
  c->ph_bound = true;
  return AP_OK;
}

AP_API int ap_get_photon_number(const ap_ctx *c, size_t *n) {
  if (!c || !n) return AP_ERR_INVALID;
  *n = c->ph_bound ? c->ph_number : 0;
  return AP_OK;
}

AP_API int ap_set_rad_params(ap_ctx *c, const ap_rad_params *rp) {
  if (!c || !rp) return AP_ERR_INVALID;
  if (rp->model != AP_RAD_DEFAULT && rp->model != AP_RAD_PULSAR && rp->model != AP_RAD_GR1D &&
      rp->model != AP_RAD_GAP1D)
    return fail(c, AP_ERR_INVALID);
  // the pulsar lab's functions read (ln r, theta) positions and Rho[0], Rho[1]
  if (rp->model == AP_RAD_PULSAR && (c->coord != 1 || c->params.num_species < 2))
    return fail(c, AP_ERR_UNSUPPORTED);
  // the 1D GR lab's read Grid_1dGR's arrays; its photons move with the GR
  // mover, the others' with the Cartesian or log-spherical one
  if ((rp->model == AP_RAD_GR1D) != (c->coord == 3)) return fail(c, AP_ERR_UNSUPPORTED);
  // the 1D gap lab's functions, with its photon mover, on a 1D gap context
  if ((rp->model == AP_RAD_GAP1D) != (c->coord == 2)) return fail(c, AP_ERR_UNSUPPORTED);
  if (rp->model == AP_RAD_GR1D || rp->model == AP_RAD_GAP1D) {
    // user_rt_init of either lab (labs/1dgr/src/cuda/radiation/
    // user_radiative_functions.cuh:191-203, labs/1dgap/...:135-144):
    // broken_power_law(1.25, 1.1, e_min, 1e-10, 0.1) over [emin(), emax()]
    // with n0 = 1.5e24 / ic_path
    if (!(rp->ic_path > 0.0f) || !(rp->e_min > 0.0f)) return fail(c, AP_ERR_INVALID);
    ap_spectrum sp{};
    sp.kind = AP_SPEC_BROKEN_POWER_LAW;
    sp.p[0] = 1.25f;
    sp.p[1] = 1.1f;
    sp.p[2] = rp->e_min;
    sp.p[3] = 1.0e-10f;
    sp.p[4] = 0.1f;
    const double n0 = 1.50e24 / rp->ic_path;
    const bool same = c->ic_ready && c->ic_n_gamma == rp->n_gamma && c->ic_n_ep == rp->n_ep &&
                      std::memcmp(&c->ic_spec, &sp, sizeof(sp)) == 0 && c->ic_n0 == n0 &&
                      c->ic_emin == (double)sp.p[3] && c->ic_emax == (double)sp.p[4];
    if (!same) AP_TRY_ST(ic_init(*c, sp, sp.p[3], sp.p[4], n0, rp->n_gamma, rp->n_ep));
  }
  c->rad = *rp;
  c->rad_on = true;
  c->rad_emit_calls = c->rad_pair_calls = 0;
  c->rad_next_photon_id = rp->first_photon_id;
  c->rad_next_ptc_id = rp->first_particle_id;
  return AP_OK;
}

AP_API int ap_ic_init(ap_ctx *c, const ap_spectrum *sp, double emin, double emax, double n0,
                      int n_gamma, int n_ep) {
  if (!c || !sp || sp->kind < AP_SPEC_POWER_LAW_HARD || sp->kind > AP_SPEC_MONO_ENERGETIC ||
      !(emin > 0.0) || !(emax > emin))
    return AP_ERR_INVALID;
  AP_TRY_ST(ic_init(*c, *sp, emin, emax, n0, n_gamma, n_ep));
  return finish(c);
}

AP_API int ap_ic_tables(ap_ctx *c, float *ic_rate, float *gg_rate, float *gammas, float *dNde,
                        float *dNde_thomson, float *steps) {
  if (!c || !c->ic_ready) return AP_ERR_INVALID;
  const size_t ng = (size_t)c->ic_n_gamma, ne = (size_t)c->ic_n_ep;
  const float *src[5] = {c->ic_buf, c->ic_buf + ng, c->ic_buf + 2 * ng, c->ic_buf + 3 * ng,
                         c->ic_buf + 3 * ng + ng * ne};
  float *dst[5] = {ic_rate, gg_rate, gammas, dNde, dNde_thomson};
  const size_t len[5] = {ng, ng, ng, ng * ne, ng * ne};
  for (int k = 0; k < 5; ++k)
    if (dst[k])
      AP_TRY(cudaMemcpyAsync(dst[k], src[k], len[k] * sizeof(float), cudaMemcpyDeviceToHost,
                             c->stream));
  AP_TRY(cudaStreamSynchronize(c->stream));
  if (steps) {
    steps[0] = c->ic_dep;
    steps[1] = c->ic_dg;
    steps[2] = c->ic_dlep;
  }
  return AP_OK;
}

static bool produced_ok(const Ctx *c, ap_array a) {
  return a.ptr == nullptr || valid_array(a, c->mesh);
}

AP_API int ap_emit_photons(ap_ctx *c, ap_array produced, ap_rad_counts *out) {
  if (!c || !out || !c->rad_on || !c->ph_bound || !c->ptc_bound || !c->fields_bound ||
      !produced_ok(c, produced))
    return AP_ERR_INVALID;
  AP_TRY_ST(refresh_number(c));
  AP_TRY_ST(rad_emit_photons(*c, produced, out));
  return AP_OK;
}

AP_API int ap_produce_pairs(ap_ctx *c, ap_array produced, ap_rad_counts *out) {
  if (!c || !out || !c->rad_on || !c->ph_bound || !c->ptc_bound || !c->fields_bound ||
      !produced_ok(c, produced))
    return AP_ERR_INVALID;
  AP_TRY_ST(refresh_number(c));
  const size_t before = c->number;
  AP_TRY_ST(rad_produce_pairs(*c, produced, out));
  if (c->number != before) {
    // the new pairs are in no tile list and may carry a larger weight
    c->order_valid = false;
    c->scale_valid = false;
    AP_TRY_ST(push_number(c));
  }
  return AP_OK;
}

AP_API int ap_move_photons(ap_ctx *c, double dt) {
  if (!c || !c->ph_bound) return AP_ERR_INVALID;
  AP_TRY_ST(rad_move_photons(*c, (float)dt, 0));
  return finish(c);
}

AP_API int ap_set_continuity_check(ap_ctx *c, int on) {
  if (!c) return AP_ERR_INVALID;
  if (c->coord != 0) return AP_ERR_UNSUPPORTED;
  if (on && !c->rho_prev) {
    const size_t n = (size_t)c->mesh.dims[0] * (c->mk.dim > 1 ? c->mesh.dims[1] : 1);
    if (cudaMalloc(&c->rho_prev, sizeof(double) * n) != cudaSuccess) {
      c->rho_prev = nullptr;
      return fail(c, AP_ERR_NOMEM);
    }
  }
  c->cont_on = on != 0;
  c->last_rho_step = -2;
  return AP_OK;
}

AP_API int ap_set_compaction(ap_ctx *c, int interval) {
  if (!c || interval < 0) return AP_ERR_INVALID;
  c->compact_interval = interval;
  c->since_compact = 0;
  return AP_OK;
}

AP_API int ap_set_tile_shape(ap_ctx *c, int tx, int ty) {
  if (!c || c->mk.dim != 2 || !is_supported_tile(tx, ty)) return AP_ERR_INVALID;
  if (c->stream) AP_TRY(cudaStreamSynchronize(c->stream));
  c->params.tile[0] = tx;
  c->params.tile[1] = ty;
  choose_tiles(*c);
  const size_t nt = (size_t)c->tiles.ntiles;
  cudaFree(c->dir_count);
  cudaFree(c->grp_off);
  cudaFree(c->newcount);
  cudaFree(c->tile_start[0]);
  cudaFree(c->tile_start[1]);
  c->dir_count = c->grp_off = c->newcount = c->tile_start[0] = c->tile_start[1] = nullptr;
  AP_TRY(cudaMalloc(&c->dir_count, sizeof(uint32_t) * (nt * 10 + 16)));
  AP_TRY(cudaMalloc(&c->grp_off, sizeof(uint32_t) * (nt * 9 + 16)));
  AP_TRY(cudaMalloc(&c->newcount, sizeof(uint32_t) * (nt + 16)));
  AP_TRY(cudaMalloc(&c->tile_start[0], sizeof(uint32_t) * (nt + 1)));
  AP_TRY(cudaMalloc(&c->tile_start[1], sizeof(uint32_t) * (nt + 1)));
  if (c->fields_bound) c->use_tma = setup_tensor_maps(*c);
  c->order_valid = false;
  return AP_OK;
}

AP_API int ap_get_tile_shape(const ap_ctx *c, int *tx, int *ty) {
  if (!c || !tx || !ty) return AP_ERR_INVALID;
  *tx = c->tiles.tx;
  *ty = c->tiles.ty;
  return AP_OK;
}

AP_API int ap_last_error(const ap_ctx *c) { return c ? c->last_error : AP_ERR_INVALID; }

AP_API uint64_t ap_launch_count(const ap_ctx *c) { return c ? c->launches : 0; }

}  // extern "C"

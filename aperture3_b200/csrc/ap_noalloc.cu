// Allocation-free variant of the 1D particle update.
//
// ap_update_particles_1d_noalloc runs the same work as ap_update_particles
// on a 1D context (push, Esirkepov deposit, periodic fold, rounding of J and
// Rho to FP32, wrap through periodic sides) without a context and without
// allocating device memory. It is meant for callers that cannot call
// cudaMalloc at the point where they update particles: for example a host
// process whose device memory is fully reserved by another allocator (a
// framework's caching allocator or a serving runtime that pre-reserves HBM
// at start-up), where an allocation inside the call would fail or fragment
// that pool. The caller passes the particle and field arrays; the only other
// device memory used is the fixed-size file-scope array below, which every
// GPU that loads this library keeps until the process exits.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "ap_internal.h"

namespace {

using namespace apb;

constexpr size_t kAccWords = (size_t)(3 + AP_NOALLOC_MAX_SPECIES) * AP_NOALLOC_MAX_CELLS;
constexpr size_t kTailWords = 32;  // format word, weight maximum, status counters

// Fixed-point current/charge accumulators followed by the small state words.
// Shared by every call on a device: the accumulators and the status are
// cleared at the start of each call.
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kAccWords + kTailWords];

// Device address of g_noalloc_scratch per CUDA context. The host-side
// symbol is only a stand-in: kernels must be given the address that
// cudaGetSymbolAddress returns in the context they run in. The cache is
// keyed by the context's unique id (cuCtxGetId), not by the device
// ordinal, so a context that is destroyed and re-created (cudaDeviceReset,
// or a caller's own driver-API context on the same device) gets its own
// lookup instead of a stale address.
struct ScratchEntry {
  unsigned long long ctx_id;
  unsigned long long *ptr;
};
constexpr int kMaxContexts = 64;
std::mutex g_mu;
ScratchEntry g_scratch_cache[kMaxContexts] = {};
int g_scratch_cached = 0;
int g_scratch_next = 0;

// The two driver calls, reached through the runtime's entry-point query so
// that the library does not link the driver library directly.
template <typename F>
F driver_fn(const char *name) {
  void *p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess)
    return nullptr;
  return reinterpret_cast<F>(p);
}

int scratch_in_current_context(unsigned long long **out) {
  static const PFN_cuCtxGetCurrent_v4000 get_current =
      driver_fn<PFN_cuCtxGetCurrent_v4000>("cuCtxGetCurrent");
  static const PFN_cuCtxGetId_v12000 get_id = driver_fn<PFN_cuCtxGetId_v12000>("cuCtxGetId");
  if (!get_current || !get_id) return AP_ERR_CUDA;
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS) return AP_ERR_CUDA;
  void *p = nullptr;
  if (!ctx) {
    // No context current on this thread yet: the runtime call below makes
    // the device's primary context current.
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return AP_ERR_CUDA;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return AP_ERR_CUDA;
  }
  unsigned long long id = 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return AP_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_mu);
  for (int i = 0; i < g_scratch_cached; ++i)
    if (g_scratch_cache[i].ctx_id == id) {
      *out = g_scratch_cache[i].ptr;
      return AP_OK;
    }
  if (!p && (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p))
    return AP_ERR_CUDA;
  // a full table is reused round-robin; a dropped entry is looked up again
  ScratchEntry &slot = g_scratch_cache[g_scratch_cached < kMaxContexts ? g_scratch_cached++
                                                                       : g_scratch_next];
  if (g_scratch_cached == kMaxContexts) g_scratch_next = (g_scratch_next + 1) % kMaxContexts;
  slot.ctx_id = id;
  slot.ptr = static_cast<unsigned long long *>(p);
  *out = slot.ptr;
  return AP_OK;
}

bool array_ok(const ap_array &a, const ap_mesh &m) {
  return a.ptr != nullptr && a.pitch >= sizeof(float) * (size_t)m.dims[0] &&
         (a.pitch % sizeof(float)) == 0;
}

}  // namespace

extern "C" AP_API int ap_update_particles_1d_noalloc(const ap_mesh *mesh,
                                                     const ap_params *params,
                                                     const ap_particles *ptc, size_t number,
                                                     const ap_fields *fields, double dt,
                                                     uint32_t step, void *cuda_stream) {
  if (!mesh || !params || !ptc || !fields) return AP_ERR_INVALID;
  const MeshK mk = make_meshk(*mesh);
  if (mk.dim != 1) return AP_ERR_UNSUPPORTED;
  if (mesh->dims[0] > AP_NOALLOC_MAX_CELLS) return AP_ERR_CAPACITY;
  if (params->num_species < 1) return AP_ERR_INVALID;
  if (params->num_species > AP_NOALLOC_MAX_SPECIES) return AP_ERR_CAPACITY;
  if (number > 0x7fffffffu) return AP_ERR_CAPACITY;
  if (mesh->guard[0] < 2 || mk.red[0] < 1) return AP_ERR_INVALID;
  if (params->periodic[0] && mk.red[0] < 2 * mesh->guard[0]) return AP_ERR_INVALID;
  if (params->data_interval < 1) return AP_ERR_INVALID;
  if (params->current_smoothing != 0) return AP_ERR_UNSUPPORTED;
  if (number > 0 && (!ptc->x1 || !ptc->x2 || !ptc->x3 || !ptc->p1 || !ptc->p2 || !ptc->p3 ||
                     !ptc->E || !ptc->weight || !ptc->cell || !ptc->flag))
    return AP_ERR_INVALID;
  for (int k = 0; k < 3; ++k)
    if (!array_ok(fields->E[k], *mesh) || !array_ok(fields->B[k], *mesh) ||
        !array_ok(fields->J[k], *mesh))
      return AP_ERR_INVALID;
  for (int s = 0; s < params->num_species; ++s)
    if (!array_ok(fields->Rho[s], *mesh)) return AP_ERR_INVALID;

  unsigned long long *scratch = nullptr;
  int st = scratch_in_current_context(&scratch);
  if (st != AP_OK) return st;

  // A context on the stack: only plain fields, no allocation.
  Ctx c;
  c.mesh = *mesh;
  c.params = *params;
  c.mk = mk;
  c.stream = static_cast<cudaStream_t>(cuda_stream);
  cudaGetDevice(&c.device);
  if (cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, c.device) !=
      cudaSuccess)
    return AP_ERR_CUDA;
  c.fields = *fields;
  c.fields_bound = true;
  c.ptc = *ptc;
  c.number = number;
  c.ptc_bound = true;
  c.acc = scratch;
  c.acc_comp = (size_t)mesh->dims[0];
  unsigned long long *tail = scratch + kAccWords;
  c.fx_used = reinterpret_cast<FixedFmt *>(tail);
  c.wmax = reinterpret_cast<float *>(tail + 1);
  c.status = reinterpret_cast<DevStatus *>(tail + 2);

  const bool do_rho = ((step + 1) % (uint32_t)params->data_interval) == 0;
  const int ncomp = 3 + (do_rho ? params->num_species : 0);
  cudaError_t e =
      cudaMemsetAsync(c.acc, 0, sizeof(unsigned long long) * c.acc_comp * ncomp, c.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c.status, 0, sizeof(DevStatus), c.stream);
  if (!do_rho)
    for (int s = 0; s < params->num_species && e == cudaSuccess; ++s)
      e = launch_zero(c, c.fields.Rho[s]);
  if (e == cudaSuccess && number == 0)  // nothing deposited: a neutral format word
    e = cudaMemsetAsync(c.fx_used, 0, sizeof(FixedFmt), c.stream);
  if (e == cudaSuccess && number > 0) e = launch_fixed_scale(c);
  if (e == cudaSuccess && number > 0) {
    PushDepositParams P;
    std::memset(&P, 0, sizeof(P));
    P.m = c.mk;
    P.p = PtcK{ptc->x1, ptc->x2, ptc->x3, ptc->p1, ptc->p2,
               ptc->p3, ptc->E,  ptc->weight, ptc->cell, ptc->flag};
    const ap_array *fa[6] = {&fields->E[0], &fields->E[1], &fields->E[2],
                             &fields->B[0], &fields->B[1], &fields->B[2]};
    for (int k = 0; k < 6; ++k) P.F[k] = FieldArr{fa[k]->ptr, (int)(fa[k]->pitch / 4)};
    for (int k = 0; k < 3; ++k) P.J[k] = FieldArr{fields->J[k].ptr, (int)(fields->J[k].pitch / 4)};
    for (int s = 0; s < params->num_species; ++s)
      P.Rho[s] = FieldArr{fields->Rho[s].ptr, (int)(fields->Rho[s].pitch / 4)};
    P.acc = c.acc;
    P.acc_pitch = mesh->dims[0];
    P.acc_comp = c.acc_comp;
    P.fx_used = c.fx_used;
    P.wmax = c.wmax;
    P.qmax = 0.0f;
    for (int s = 0; s < AP_MAX_SPECIES; ++s) P.qmax = fmaxf(P.qmax, fabsf(params->charges[s]));
    const float dtf = (float)dt;
    P.dt = dtf;
    for (int s = 0; s < AP_MAX_SPECIES; ++s) {
      volatile float a = dtf * 0.5f;
      volatile float b = a * params->charges[s];
      P.qm[s] = params->masses[s] != 0.0f ? b / params->masses[s] : 0.0f;
      P.charge[s] = params->charges[s];
    }
    P.num_species = params->num_species;
    P.do_rho = do_rho ? 1 : 0;
    for (int d = 0; d < 3; ++d) P.periodic[d] = params->periodic[d];
    P.status = c.status;
    P.number = number;
    e = launch_push_deposit_1d(c, P);
  }
  if (e == cudaSuccess) e = launch_finalize_current(c, ncomp);
  DevStatus hs;
  std::memset(&hs, 0, sizeof(hs));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&hs, c.status, sizeof(DevStatus), cudaMemcpyDeviceToHost, c.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
  if (e != cudaSuccess) {
    // Work enqueued before the failure may still use the shared array: wait
    // for it, so that a retry (on any stream) cannot overlap with it.
    cudaStreamSynchronize(c.stream);
    return AP_ERR_CUDA;
  }
  if (hs.timeouts) return AP_ERR_TIMEOUT;
  if (hs.nan_momenta) return AP_ERR_NAN;
  if (hs.moved_far) return AP_ERR_MOVED_FAR;
  return AP_OK;
}

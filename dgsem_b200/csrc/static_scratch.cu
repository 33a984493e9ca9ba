// dgsem_ssprk3_step_static_scratch: one SSPRK3 step whose two stage states
// live in a file-scope device array instead of the context's temporaries.
// The entry point allocates nothing (no cudaMalloc/cudaFree, no allocating
// library routine); it drives the same fused stage kernels as
// dgsem_ssprk3_step through the public dgsem_ssprk3_stage.
//
// The scratch is a static __device__ array in this translation unit, so it
// belongs to this file's module alone: a process that never calls this entry
// point does not pay for it under lazy module loading.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "context.hpp"
#include "dgsem_b200.h"

// Two stage states of at most DGSEM_STATIC_SCRATCH_MAX_STATE doubles each
// (2 x 16 MiB).  Nothing here has to start at zero: stage 1 writes every
// entry of the first state before stage 2 reads it, and stage 2 every entry
// of the second before stage 3 reads it.
static __device__ __align__(256) double dgsem_stage_scratch[2 * DGSEM_STATIC_SCRATCH_MAX_STATE];

namespace {

constexpr int kMaxDevices = 64;

// Per-device address of the scratch, looked up with that device current.
// Only a successful look-up is kept: a failed one (which leaves nothing
// cached) is retried by the next call on that device.
std::mutex g_slot_mutex;
double* g_slots[kMaxDevices] = {};

dgsem_status scratch_on_device(int device, double** out) {
  if (device < 0 || device >= kMaxDevices) return DGSEM_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lock(g_slot_mutex);
  if (!g_slots[device]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, dgsem_stage_scratch) != cudaSuccess || !p) {
      cudaGetLastError();  // leave no stale error for the next launch check
      return DGSEM_ERR_CUDA;
    }
    g_slots[device] = static_cast<double*>(p);
  }
  *out = g_slots[device];
  return DGSEM_OK;
}

}  // namespace

extern "C" dgsem_status dgsem_ssprk3_step_static_scratch(dgsem_ctx* ctx, double* u, double t,
                                                         double dt) {
  if (!ctx || !u) return DGSEM_ERR_INVALID_ARG;
  int64_t nelem = 0, state_len = 0;
  int nodes = 0, nvars = 0;
  dgsem_status st = dgsem_get_sizes(ctx, &nelem, &nodes, &nvars, &state_len);
  if (st != DGSEM_OK) return st;
  if (state_len > DGSEM_STATIC_SCRATCH_MAX_STATE) return DGSEM_ERR_SCRATCH_LIMIT;
  // The scratch address is per device: u and the context must belong to
  // the current device.
  int device = -1;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return DGSEM_ERR_CUDA;
  }
  if (ctx->device != device) return DGSEM_ERR_INVALID_ARG;
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, u) != cudaSuccess) {
    cudaGetLastError();
    return DGSEM_ERR_INVALID_ARG;
  }
  if ((attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) ||
      attr.device != device)
    return DGSEM_ERR_INVALID_ARG;
  double* scratch = nullptr;
  st = scratch_on_device(device, &scratch);
  if (st != DGSEM_OK) return st;
  double* s1 = scratch;
  double* s2 = scratch + DGSEM_STATIC_SCRATCH_MAX_STATE;
  st = dgsem_ssprk3_stage(ctx, 1, nullptr, u, s1, t, dt);
  if (st == DGSEM_OK) st = dgsem_ssprk3_stage(ctx, 2, u, s1, s2, t, dt);
  if (st == DGSEM_OK) st = dgsem_ssprk3_stage(ctx, 3, u, s2, u, t, dt);
  return st;
}

extern "C" dgsem_status dgsem_static_scratch_state(int k, const double** out) {
  if (!out || k < 0 || k > 1) return DGSEM_ERR_INVALID_ARG;
  *out = nullptr;
  int device = -1;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return DGSEM_ERR_CUDA;
  }
  double* scratch = nullptr;
  const dgsem_status st = scratch_on_device(device, &scratch);
  if (st != DGSEM_OK) return st;
  *out = scratch + (int64_t)k * DGSEM_STATIC_SCRATCH_MAX_STATE;
  return DGSEM_OK;
}

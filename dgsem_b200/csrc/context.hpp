// Internal definition of the C ABI context (shared by the translation units
// that implement include/dgsem_b200.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <vector>

#include "../../include/dgsem_b200.h"
#include "engine.cuh"

struct dgsem_ctx {
  dgsem_mesh_desc mesh;
  dgsem_scheme_desc scheme;
  cudaStream_t stream = nullptr;
  int device = 0;
  dgsem::EngineConfig cfg{};
  std::unique_ptr<dgsem::EngineBase> engine;
  int nodes = 0;     // n^d
  int nvars = 0;
  int64_t state_len = 0;
  std::vector<void*> allocations;
  double* tmp1 = nullptr;  // SSPRK3 stage states
  double* tmp2 = nullptr;
  double* staging = nullptr;  // device copy for the host-buffer entry point
  double* tdev = nullptr;     // device clock for graph replay
  double* table_block = nullptr;
  unsigned int* flag = nullptr;
  int64_t launches = 0;
  // fused diagnostics (dgsem_set_diagnostics): per-block partial volume
  // integrals of the stage-3 output and the reduced (volume, KE, entropy)
  double* diag_partials = nullptr;  // non-null while enabled
  double* diag_store = nullptr;
  double* diag_result = nullptr;
  // failure-path testing: allocation number that fails (0 = none)
  int alloc_calls = 0;
  int fail_alloc_at = 0;
};

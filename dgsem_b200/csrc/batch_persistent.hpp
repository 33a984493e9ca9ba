// Persistent batched stage launch (batch_persistent.cu): one launch per
// SSPRK3 stage over the meshes of every degree of a 2D batch.
#pragma once

#include <cuda_runtime.h>

#include "engine.cuh"

namespace dgsem {

// One degree's share of a persistent launch (deg[k] describes n = k + 2).
struct PersistentDegree {
  const EngineConfig* cfg = nullptr;  // null: no mesh of this degree
  const MeshView* meshes = nullptr;   // the stage's mesh views (device)
  const int* tile_mesh = nullptr;     // device tile list of this degree
  const int* tile_e0 = nullptr;
};

bool persistent_supported(int ndims, int vf, int sf);
// elements per tile of degree n (the node-parallel tile)
int persistent_elements_per_tile(int n);
// dynamic shared memory of the launch for the degrees present
size_t persistent_smem(int vf, const PersistentDegree* deg);
// resident blocks on the device at that shared-memory size
int persistent_grid(int vf, size_t smem);
// out = a*u_n + b*u_in + c*RHS for every tile of the work list
cudaError_t launch_persistent_stage(int vf, const PersistentDegree* deg, const int* work,
                                    int nwork, double a, double b, double t, const double* t_dev,
                                    int grid, size_t smem, cudaStream_t s);

}  // namespace dgsem

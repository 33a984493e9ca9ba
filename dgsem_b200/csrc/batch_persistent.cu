// One persistent launch per SSPRK3 stage over all meshes of a 2D batch, of
// every polynomial degree: each block walks a work list of (degree, tile)
// items, cost-ordered (higher degrees first), and runs the node-parallel
// stage body of that item's degree (stage_node_kernel.cuh) with 256 threads;
// degrees whose tiles use fewer threads leave the rest idle at the barriers.
// The per-degree launch arguments (basis tables, mesh tables, tile lists)
// travel in the kernel parameters.  No reference counterpart (the reference
// advances one mesh per solver instance).
#include <cuda_runtime.h>

#include "batch_persistent.hpp"
#include "engine.cuh"

namespace dgsem {
namespace {

// 256 threads per block (every degree's work item then fills at least 95 %
// of its warp lanes) and 4 resident blocks per SM (64 registers): on the
// batched vortex workload 17.6 ms per step against 20.1 ms for 128 threads
// at 72 registers and 22.6 ms at 96; occupancy outweighs the spills.
constexpr int kThreads = 256;
constexpr int kMinBlocks = 4;

// Elements per work item of degree n: as many as fit in the kThreads threads of
// the persistent block (at least 95 % of its lanes for every degree).
template <int N>
struct PersistLaunch {
  static constexpr int EPB = kThreads / (N * N) > 0 ? kThreads / (N * N) : 1;
  static constexpr int NT = EPB * N * N;
};

template <int VF, int SF>
struct PersistArgs {
  StageArgs<2> a2;
  StageArgs<3> a3;
  StageArgs<4> a4;
  StageArgs<5> a5;
  StageArgs<6> a6;
  StageArgs<7> a7;
  StageArgs<8> a8;
  const int* work;  // per item: (n << 24) | tile index within the degree's tile list
  int nwork;
};

template <int N, int VF, int SF>
__device__ __forceinline__ void run_item(const StageArgs<N>& a, int tile) {
  using NL = PersistLaunch<N>;
  static_assert(NL::NT <= kThreads, "tile wider than the persistent block");
  stage_node_body<2, N, VF, SF, NL::EPB, true, false, false, kThreads, true>(a, tile);
}

// The kernel inlines the bodies of all seven degrees, so its register count
// is their maximum (168 uncapped); the cap of kMinBlocks blocks per SM
// spills in every body.
template <int VF, int SF>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
    batch_persistent_kernel(const PersistArgs<VF, SF> P) {
  for (int w = blockIdx.x; w < P.nwork; w += gridDim.x) {
    const int item = P.work[w];
    const int n = item >> 24, tile = item & 0xffffff;
    switch (n) {
      case 2: run_item<2, VF, SF>(P.a2, tile); break;
      case 3: run_item<3, VF, SF>(P.a3, tile); break;
      case 4: run_item<4, VF, SF>(P.a4, tile); break;
      case 5: run_item<5, VF, SF>(P.a5, tile); break;
      case 6: run_item<6, VF, SF>(P.a6, tile); break;
      case 7: run_item<7, VF, SF>(P.a7, tile); break;
      default: run_item<8, VF, SF>(P.a8, tile); break;
    }
    // the next item reuses the shared memory: every thread of the block has
    // finished this one (threads that left the body early wait here)
    __syncthreads();
  }
}

template <int N>
constexpr size_t smem_of(int vf) {
  using NL = PersistLaunch<N>;
  return vf == VF_CHANDRASHEKAR ? NodeShape<2, N, VF_CHANDRASHEKAR, NL::EPB>::smem_bytes_base
         : vf == VF_RANOCHA     ? NodeShape<2, N, VF_RANOCHA, NL::EPB>::smem_bytes_base
                                : NodeShape<2, N, VF_KENNEDY_GRUBER, NL::EPB>::smem_bytes_base;
}

size_t max_smem(int vf, const int* present) {
  const size_t s[7] = {smem_of<2>(vf), smem_of<3>(vf), smem_of<4>(vf), smem_of<5>(vf),
                       smem_of<6>(vf), smem_of<7>(vf), smem_of<8>(vf)};
  size_t m = 0;
  for (int k = 0; k < 7; ++k)
    if (present[k] && s[k] > m) m = s[k];
  return m;
}

template <int N>
void set_degree(StageArgs<N>& dst, const PersistentDegree& d, double a, double b, double t,
                const double* t_dev) {
  if (!d.cfg) return;
  dst = stage_args_common<N>(*d.cfg, a, b, t, t_dev, nullptr);
  dst.meshes = d.meshes;
  dst.tile_mesh = d.tile_mesh;
  dst.tile_e0 = d.tile_e0;
}

template <int VF, int SF>
cudaError_t launch_vf(const PersistentDegree* deg, const int* work, int nwork, double a, double b,
                      double t, const double* t_dev, int grid, size_t smem, cudaStream_t s) {
  PersistArgs<VF, SF> P{};
  set_degree<2>(P.a2, deg[0], a, b, t, t_dev);
  set_degree<3>(P.a3, deg[1], a, b, t, t_dev);
  set_degree<4>(P.a4, deg[2], a, b, t, t_dev);
  set_degree<5>(P.a5, deg[3], a, b, t, t_dev);
  set_degree<6>(P.a6, deg[4], a, b, t, t_dev);
  set_degree<7>(P.a7, deg[5], a, b, t, t_dev);
  set_degree<8>(P.a8, deg[6], a, b, t, t_dev);
  P.work = work;
  P.nwork = nwork;
  auto k = batch_persistent_kernel<VF, SF>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  launch_stage_kernel(k, (unsigned)grid, kThreads, smem, s, P);
  return cudaGetLastError();
}

template <int VF, int SF>
int occupancy_vf(size_t smem) {
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaFuncSetAttribute(batch_persistent_kernel<VF, SF>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_persistent_kernel<VF, SF>,
                                                kThreads, smem);
  return (nsm > 0 ? nsm : 1) * (per_sm > 0 ? per_sm : 1);
}

}  // namespace

bool persistent_supported(int ndims, int vf, int sf) {
  return ndims == 2 && vf >= 0 && vf <= 2 && sf == SF_LLF;
}

int persistent_elements_per_tile(int n) {
  switch (n) {
    case 2: return PersistLaunch<2>::EPB;
    case 3: return PersistLaunch<3>::EPB;
    case 4: return PersistLaunch<4>::EPB;
    case 5: return PersistLaunch<5>::EPB;
    case 6: return PersistLaunch<6>::EPB;
    case 7: return PersistLaunch<7>::EPB;
    default: return PersistLaunch<8>::EPB;
  }
}

size_t persistent_smem(int vf, const PersistentDegree* deg) {
  int present[7];
  for (int k = 0; k < 7; ++k) present[k] = deg[k].cfg != nullptr;
  return max_smem(vf, present);
}

int persistent_grid(int vf, size_t smem) {
  switch (vf) {
    case VF_RANOCHA: return occupancy_vf<VF_RANOCHA, SF_LLF>(smem);
    case VF_KENNEDY_GRUBER: return occupancy_vf<VF_KENNEDY_GRUBER, SF_LLF>(smem);
    default: return occupancy_vf<VF_CHANDRASHEKAR, SF_LLF>(smem);
  }
}

cudaError_t launch_persistent_stage(int vf, const PersistentDegree* deg, const int* work,
                                    int nwork, double a, double b, double t, const double* t_dev,
                                    int grid, size_t smem, cudaStream_t s) {
  switch (vf) {
    case VF_RANOCHA:
      return launch_vf<VF_RANOCHA, SF_LLF>(deg, work, nwork, a, b, t, t_dev, grid, smem, s);
    case VF_KENNEDY_GRUBER:
      return launch_vf<VF_KENNEDY_GRUBER, SF_LLF>(deg, work, nwork, a, b, t, t_dev, grid, smem,
                                                  s);
    default:
      return launch_vf<VF_CHANDRASHEKAR, SF_LLF>(deg, work, nwork, a, b, t, t_dev, grid, smem,
                                                 s);
  }
}

}  // namespace dgsem

// FP64 fused-multiply-add throughput of this GPU, measured with CUDA events:
// the FP64-pipe bound beside the HBM bound of the stage kernels' roofline.
// (No counterpart in the reference, which has no timers.)
//
// Every thread runs kChains independent FMA chains, x_c <- x_c * a + b, so
// the pipe, not the FMA latency, bounds the loop; the grid fills every SM
// with resident blocks.  One FMA counts as 2 floating-point operations.  The
// result of each thread is summed and written so the chains cannot be
// removed; with a = 1 - 2^-20 and b = 2^-20 they stay finite and bounded.
// Runs on the clocks the GPU has: nothing here changes a clock or a limit.
#include <cuda_runtime.h>

#include "dgsem_b200.h"

namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;

// written only under a condition that never holds (keeps the chains live)
__device__ double g_fp64_sink;

__global__ void __launch_bounds__(kThreads) fp64_fma_kernel(int iters, double a, double b) {
  double x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) x[c] = 1.0 + 1e-3 * (threadIdx.x + c);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k)
#pragma unroll
      for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += x[c];
  if (s == 12345.678) g_fp64_sink = s;  // the chains converge to 1: never true
}

}  // namespace

extern "C" dgsem_status dgsem_fp64_fma_peak(void* stream, int iters, double* flops_per_s,
                                            double* ms) {
  if (!flops_per_s || iters < 1) return DGSEM_ERR_INVALID_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int dev = 0, nsm = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fp64_fma_kernel, kThreads, 0) !=
          cudaSuccess) {
    cudaGetLastError();
    return DGSEM_ERR_CUDA;
  }
  const int blocks = nsm * (per_sm > 0 ? per_sm : 1);
  const double a = 1.0 - 1.0 / 1048576.0, b = 1.0 / 1048576.0;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return DGSEM_ERR_CUDA;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return DGSEM_ERR_CUDA;
  }
  // warm-up launch, then the timed one
  fp64_fma_kernel<<<blocks, kThreads, 0, s>>>(iters / 4 + 1, a, b);
  cudaEventRecord(e0, s);
  fp64_fma_kernel<<<blocks, kThreads, 0, s>>>(iters, a, b);
  cudaEventRecord(e1, s);
  cudaError_t err = cudaEventSynchronize(e1);
  float t = 0.f;
  if (err == cudaSuccess) err = cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess || t <= 0.f) {
    cudaGetLastError();
    return DGSEM_ERR_CUDA;
  }
  const double fmas = (double)blocks * kThreads * (double)iters * 16.0 * kChains;
  *flops_per_s = 2.0 * fmas / (t * 1e-3);
  if (ms) *ms = t;
  return DGSEM_OK;
}

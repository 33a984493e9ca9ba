// Persistent, pipelined form of the node-parallel stage kernel
// (stage_node_kernel.cuh): the same arithmetic, with the element tiles
// streamed through shared memory by TMA bulk copies so that HBM latency
// overlaps computation.
//
// Each block loops over tiles t = blockIdx.x, blockIdx.x + gridDim.x, ...
// (a tile = EPB consecutive elements; u[e][var][node] makes a tile one
// contiguous range of the state).  Per tile:
//   - u_in(t) has been requested by the previous iteration (or the prologue)
//     as one bulk copy into `stage_in`, u_n(t) likewise into `stage_n`;
//   - phase 1 converts stage_in into the shared-memory tile + node data, after
//     which one thread requests u_in(t + gridDim.x) into stage_in: the copy
//     runs while faces, volume term and lifting of tile t are computed;
//   - the epilogue waits for u_n(t), stores, and after the closing barrier
//     u_n(t + gridDim.x) is requested.
// Every wait on an mbarrier is bounded; the block votes on the outcome, and
// on a timeout it sets bit 1 of the status flag and returns as a whole.
// Requirements (checked by the host): u_in and u_n 16-byte aligned and an
// even number of doubles per element (2D, or 3D with even n), so every tile
// copy is 16-byte aligned and a multiple of 16 bytes.
#pragma once

#include "stage_node_kernel.cuh"
#include "tma.cuh"

namespace dgsem {

template <int DIM, int N, int VF, int EPB>
struct PipeShape {
  using B = NodeShape<DIM, N, VF, EPB>;
  static constexpr int NV = B::NV, ND = B::ND, NDP = B::NDP, NF = B::NF, NFACE = B::NFACE,
                       NQ = B::NQ, NI = B::NI, NT = B::NT;
  static constexpr int SM_T = EPB * NV * ND;  // one staged tile (unpadded)
  static constexpr size_t smem_bytes =
      sizeof(double) * (2 * SM_T + B::SM_U + B::SM_P + B::SM_F + B::SM_X) +
      sizeof(int) * EPB * NI;
  static constexpr bool kSupported = (NV * ND) % 2 == 0;
  // resident blocks per SM allowed by shared memory (228 KB, 1 KB reserved
  // per block), capped at 72 registers per thread (7 blocks of 128 threads)
  static constexpr int MINB_SMEM = int((228 * 1024) / (smem_bytes + 1024));
  static constexpr int MINB_REG = 65536 / (NT * 72) > 1 ? 65536 / (NT * 72) : 1;
  static constexpr int MINB_CAP = MINB_SMEM < MINB_REG ? MINB_SMEM : MINB_REG;
  static constexpr int MINB = MINB_CAP > 0 ? MINB_CAP : 1;
};

template <int DIM, int N, int VF, int SF, int EPB>
__device__ __forceinline__ void stage_pipe_body(const StageArgs<N>& p, int ntiles) {
  using S = PipeShape<DIM, N, VF, EPB>;
  using K = NodeKernelSlots<DIM, VF>;
  constexpr int NV = S::NV, ND = S::ND, NDP = S::NDP, NF = S::NF, NFACE = S::NFACE,
                NQ = S::NQ, NI = S::NI, NT = S::NT;
  extern __shared__ __align__(128) double smem_pipe[];
  double* stage_in = smem_pipe;                    // [el][var][node], bulk-copy target
  double* stage_n = stage_in + S::SM_T;            // [el][var][node], bulk-copy target
  double* us = stage_n + S::SM_T;                  // [el][var][pnode]
  double* pr = us + S::B::SM_U;                    // [el][slot][pnode]
  double* sf = pr + S::B::SM_P;                    // [el][face][fn][var]
  double* xbuf = sf + S::B::SM_F;                  // volume-term exchange
  int* info = reinterpret_cast<int*>(xbuf + S::B::SM_X);
  __shared__ uint64_t bar_in, bar_n;

  stage_dependency_sync();
  const MeshView& M = p.mesh;
  const int tid = threadIdx.x;
  const int nelem = M.nelem;
  const double gamma = p.gamma;
  const double t_stage = p.t_dev ? (*p.t_dev + p.t) : p.t;
  const int c0 = M.cells[0], c1 = M.cells[1], c2 = M.cells[2];
  const bool with_n = p.a != 0.0;
  constexpr uint32_t kElemBytes = NV * ND * sizeof(double);

  auto request = [&](uint64_t* bar, double* dst, const double* src_state, int tile) {
    const int te0 = tile * EPB;
    const int tne = min(EPB, nelem - te0);
    const uint32_t bytes = (uint32_t)tne * kElemBytes;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(bar, bytes);
    bulk_copy_g2s(dst, src_state + (int64_t)te0 * NV * ND, bytes, bar);
  };

  if (tid == 0) {
    mbar_init(&bar_in, 1);
    mbar_init(&bar_n, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (tid == 0 && (int)blockIdx.x < ntiles) {
    request(&bar_in, stage_in, M.u_in, blockIdx.x);
    if (with_n) request(&bar_n, stage_n, M.u_n, blockIdx.x);
  }

  const int el = tid / ND, node = tid % ND;
  const int pn = padn<N, S::B::PAD>(node);
  uint32_t phase = 0;
  double dacc[3] = {0.0, 0.0, 0.0};  // fused diagnostics of this block's tiles
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, phase ^= 1u) {
    const int e0 = t * EPB;
    const int ne = min(EPB, nelem - e0);
    const bool active = el < ne;

    // ---- element info ------------------------------------------------------
    if (M.info) {
      for (int k = tid; k < ne * NI; k += NT) info[k] = __ldg(M.info + (int64_t)e0 * NI + k);
    } else {
      node_element_info<DIM, NI>(M, info, e0, ne, tid, NT);
    }
    // -1/J of this thread's node from the mesh's table, requested before
    // the wait for the tile
    double mij_node = 0.0;
    if (M.mij && active) mij_node = __ldg(M.mij + (int64_t)(e0 + el) * ND + node);
    // the block agrees on a timeout (vote) so that all of it leaves together
    if (__syncthreads_or(!mbar_wait_bounded(&bar_in, phase, p.wait_limit_ns))) {
      if (tid == 0) atomicOr(p.nonfinite, 2u);
      return;
    }

    // ---- phase 1: tile -> shared tile + node data, a^2, -1/J --------------
    if (active) {
      double u[NV];
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        u[q] = stage_in[(el * NV + q) * ND + node];
        us[(el * NV + q) * NDP + pn] = u[q];
      }
      node_prepare<DIM, N, VF, NDP>(M, u, gamma, info + el * NI, node, pr + el * NQ * NDP + pn,
                                    M.mij ? &mij_node : nullptr);
    }
    __syncthreads();
    // stage_in is consumed: request the next tile's u_in
    if (tid == 0 && t + (int)gridDim.x < ntiles)
      request(&bar_in, stage_in, M.u_in, t + gridDim.x);

    // ---- phase 2a: face fluxes ---------------------------------------------
    node_face_tasks<DIM, N, VF, SF, false, NDP, NT, NQ, NI>(p, M, us, pr, nullptr, info, sf, ne,
                                                            tid, gamma, t_stage, c0, c1, c2);

    // ---- phase 2b: volume term ---------------------------------------------
    double acc[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] = 0.0;
    // whole-warp volume term (see stage_node_body): lanes past the last
    // element of a partial tile read element 0 and discard the result
    constexpr bool WARP_ALL = NT % 32 == 0;
    constexpr bool XB = S::B::XCHG;  // exchange buffer: every thread takes part
    if (active || WARP_ALL || XB) {
      const int ev = active ? el : 0;
      const int* I = info + ev * NI;
      const double* U = us + ev * NV * NDP;
      const double* P = pr + ev * NQ * NDP;
      const NodeFluxState<DIM> own = load_flux_state<DIM, VF>(U, P, NDP, pn);
      const double hgm1 = 0.5 * p.inv_gm1;
      node_volume_direction<0, DIM, N, VF, NDP, WARP_ALL, XB>(p, M, U, P, I, node, pn, own, hgm1,
                                                              acc, xbuf, tid, NT);
      node_volume_direction<1, DIM, N, VF, NDP, WARP_ALL, XB>(p, M, U, P, I, node, pn, own, hgm1,
                                                              acc, xbuf, tid, NT);
      if constexpr (DIM == 3)
        node_volume_direction<2, DIM, N, VF, NDP, WARP_ALL, XB>(p, M, U, P, I, node, pn, own,
                                                                hgm1, acc, xbuf, tid, NT);
    }
    __syncthreads();

    // ---- phase 3: lifting, -1/J, SSPRK3 combination, store -----------------
    if (with_n && __syncthreads_or(!mbar_wait_bounded(&bar_n, phase, p.wait_limit_ns))) {
      if (tid == 0) atomicOr(p.nonfinite, 2u);
      return;
    }
    if (active) {
      node_lift<DIM, N>(sf + el * NFACE * NF * NV, node, p.basis.lhat_l0, p.basis.lhat_rN, acc);
      const double mij = pr[(el * NQ + K::MIJ) * NDP + pn];
      const int64_t gbase = (int64_t)(e0 + el) * NV * ND + node;
      bool bad = false;
      double vals[NV];
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        const double du = acc[q] * mij;
        double val = M.c * du;
        if (p.b != 0.0) val = p.b * us[(el * NV + q) * NDP + pn] + val;
        if (with_n) val = p.a * stage_n[(el * NV + q) * ND + node] + val;
        bad |= !isfinite(val);
        M.out[gbase + (int64_t)q * ND] = val;
        vals[q] = val;
      }
      if (bad) atomicOr(p.nonfinite, 1u);
      if (p.diag) diag_add_node<DIM, N>(vals, p.basis, node, -mij, gamma, p.inv_gm1, dacc);
    }
    __syncthreads();
    // stage_n, shared tile, node data and face buffer are free again
    if (tid == 0 && with_n && t + (int)gridDim.x < ntiles)
      request(&bar_n, stage_n, M.u_n, t + gridDim.x);
  }
  // fused diagnostics: one partial per block over all of its tiles
  // the state tile is free after the last tile (NV * NT >= 3 * NT doubles)
  if (p.diag) diag_block_store<NT>(dacc, us, p.diag + 3 * (int64_t)blockIdx.x);
}

template <int DIM, int N, int VF, int SF, int EPB, int MINB>
__global__ void __launch_bounds__(EPB* ipow(N, DIM), MINB)
    stage_pipe_kernel(const StageArgs<N> p, int ntiles) {
  stage_pipe_body<DIM, N, VF, SF, EPB>(p, ntiles);
}

}  // namespace dgsem

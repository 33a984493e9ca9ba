// Two-nodes-per-thread form of the node-parallel stage kernel (launch shape
// 6) for 3D meshes with n = 2 or 4 nodes per direction, split form without
// shock capturing or viscous terms: the same right-hand side and SSPRK3
// epilogue as stage_node_kernel.cuh.
//
// Thread h of an element (n^3 / 2 threads per element) owns the nodes
// h = (i, j, k0) and h + n^3/2 = (i, j, k0 + n/2), k0 < n/2.  For n = 4 an
// element is one warp (lane = h), for n = 2 four lanes.  Then:
//   * x and y lines of both nodes lie inside the warp, with the pair sharing
//     of node_volume_direction (warp shuffles) per node;
//   * the z line of the two nodes is split between the n/2 threads with the
//     same (i, j): the pair (k0, k0 + n/2) is evaluated once inside the
//     thread, and (n = 4) each thread evaluates the pairs (m, m+1 mod 4) of its
//     two nodes and hands them to the thread that owns node m+1 (lane ^ 16) by
//     shuffle, so every z pair is evaluated exactly once: 1.5 two-point fluxes
//     per node along z instead of n - 1 = 3;
//   * per-thread work outside the flux loops (indices, tile and face-task
//     bookkeeping, branches) is shared by two nodes, and the two nodes' flux
//     evaluations are independent instruction streams.
// The two-point flux and its pair normal are symmetric in the two nodes
// (node_volume_direction relies on the same fact), so each node's sum
// sum_k Dsplit(m, k) f(u_m, u_k) equals the reference's k > i pair loop up to
// summation order.
#pragma once

#include "stage_node_kernel.cuh"

namespace dgsem {

template <int N>
struct Node2Launch {
  static_assert(N == 2 || N == 4, "two nodes per thread: n = 2 or 4");
  static constexpr int ND = N * N * N;
  static constexpr int NH = ND / 2;    // threads per element
  static constexpr int NT = 128;
  static constexpr int EPB = NT / NH;  // 4 elements (n = 4), 32 (n = 2)
};

template <int N, int VF>
using Node2Shape = NodeShape<3, N, VF, Node2Launch<N>::EPB>;

// z-direction volume term of the thread's two nodes nA = (i, j, kA) and
// nB = (i, j, kA + n/2).
template <int N, int VF>
__device__ __forceinline__ void node2_volume_z(const StageArgs<N>& p, const MeshView& M,
                                               const double* U, const double* P, const int* I,
                                               int nA, const NodeFluxState<3>& ownA,
                                               const NodeFluxState<3>& ownB, double hgm1,
                                               double* accA, double* accB) {
  constexpr int DIM = 3, NV = 5, ND = N * N * N, N2 = N * N;
  constexpr bool HALF = NodeKernelSlots<DIM, VF>::HALF;
  const int kA = nA / N2, kB = kA + N / 2;
  const int nB = nA + N2 * (N / 2);
  // the nodes' own (halved when HALF) Ja^z
  double hA[DIM], hB[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    const double* jrow = M.tab.ja[2][c] + (int64_t)I[3 + c] * ND;
    const double ja = __ldg(jrow + nA), jb = __ldg(jrow + nB);
    hA[c] = HALF ? 0.5 * ja : ja;
    hB[c] = HALF ? 0.5 * jb : jb;
  }
  // the pair (kA, kB) inside the thread
  {
    double nrm[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) nrm[c] = HALF ? hA[c] + hB[c] : 0.5 * (hA[c] + hB[c]);
    double f[NV];
    node_volume_flux<DIM, VF>(ownA, ownB, nrm, p.inv_gm1, hgm1, f);
    const double da = p.basis.Dsplit[kA][kB], db = p.basis.Dsplit[kB][kA];
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      accA[q] += da * f[q];
      accB[q] += db * f[q];
    }
  }
  if constexpr (N == 4) {
    // the pairs (m, m+1 mod 4) of both nodes; the partner node m+1 belongs
    // to the other thread of the z line (lane ^ 16): its state from shared
    // memory, its metric by shuffle
    const bool low = kA == 0;
    double oA[DIM], oB[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      const double xa = __shfl_xor_sync(0xffffffffu, hA[c], 16);
      const double xb = __shfl_xor_sync(0xffffffffu, hB[c], 16);
      // partner of kA is kA+1 (the other thread's slot A when kA = 0, its
      // slot B when kA = 1); partner of kB is kB+1 mod 4 (slot B, slot A)
      oA[c] = low ? xa : xb;
      oB[c] = low ? xb : xa;
    }
    double fA[NV], fB[NV];
    {
      const NodeFluxState<DIM> other = load_flux_state<DIM, VF>(U, P, ND, nA + N2);
      double nrm[DIM];
#pragma unroll
      for (int c = 0; c < DIM; ++c) nrm[c] = HALF ? hA[c] + oA[c] : 0.5 * (hA[c] + oA[c]);
      node_volume_flux<DIM, VF>(ownA, other, nrm, p.inv_gm1, hgm1, fA);
    }
    {
      const int nk = low ? nB + N2 : nB - 3 * N2;  // node kB + 1 mod 4
      const NodeFluxState<DIM> other = load_flux_state<DIM, VF>(U, P, ND, nk);
      double nrm[DIM];
#pragma unroll
      for (int c = 0; c < DIM; ++c) nrm[c] = HALF ? hB[c] + oB[c] : 0.5 * (hB[c] + oB[c]);
      node_volume_flux<DIM, VF>(ownB, other, nrm, p.inv_gm1, hgm1, fB);
    }
    const double dA = p.basis.Dsplit[kA][kA + 1], dB = p.basis.Dsplit[kB][(kB + 1) & 3];
    // node m receives f(m-1, m) from the owner of m-1: node kA = 0 from the
    // other's slot B (node 3), kA = 1 from its slot A (node 0); node kB = 2
    // from the other's slot A (node 1), kB = 3 from its slot B (node 2)
    const double rA_d = p.basis.Dsplit[kA][(kA + 3) & 3];
    const double rB_d = p.basis.Dsplit[kB][kB - 1];
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      accA[q] += dA * fA[q];
      accB[q] += dB * fB[q];
      const double gA = __shfl_xor_sync(0xffffffffu, fA[q], 16);
      const double gB = __shfl_xor_sync(0xffffffffu, fB[q], 16);
      accA[q] += rA_d * (low ? gB : gA);
      accB[q] += rB_d * (low ? gA : gB);
    }
  }
}

template <int N, int VF, int SF>
__device__ __forceinline__ void stage_node2_body(const StageArgs<N>& p) {
  constexpr int DIM = 3;
  using NL = Node2Launch<N>;
  using S = Node2Shape<N, VF>;
  using K = NodeKernelSlots<DIM, VF>;
  constexpr int EPB = NL::EPB, NT = NL::NT, NH = NL::NH;
  constexpr int NV = S::NV, ND = S::ND, NDP = S::NDP, NF = S::NF, NFACE = S::NFACE,
                NQ = S::NQ, NI = S::NI;
  static_assert(NDP == ND && !S::XCHG && S::NT == 2 * NT, "shape");
  static_assert(S::SM_A == 0 && S::SM_VINV == 0 && S::SM_X == 0 && S::SM_W == 0, "layout");
  extern __shared__ __align__(128) double smem_node2[];
  double* us = smem_node2;     // [el][var][node]
  double* pr = us + S::SM_U;   // [el][slot][node]
  double* sf = pr + S::SM_P;   // [el][face][fn][var]
  int* info = reinterpret_cast<int*>(sf + S::SM_F);
  // [el][var][node] u_n tile (bulk-copy target; present when p.a != 0)
  double* stage_n =
      reinterpret_cast<double*>(reinterpret_cast<char*>(smem_node2) + S::off_n_bytes);

  stage_dependency_sync();
  const int tid = threadIdx.x;
  const MeshView& M = p.mesh;
  const int nelem = M.nelem;
  const int e0 = (int)blockIdx.x * EPB;
  if (e0 >= nelem) return;
  const int ne = min(EPB, nelem - e0);
  const double gamma = p.gamma;
  const double t_stage = p.t_dev ? (*p.t_dev + p.t) : p.t;
  const int c0 = M.cells[0], c1 = M.cells[1], c2 = M.cells[2];

  // ---- phases 0 and 1: the u_in tile, the u_n tile, element info, node
  // data (as in stage_node_body: with the mesh's tables every thread reads
  // its own two nodes and computes their data before the one barrier) -----
  const int el = tid / NH, h = tid % NH;
  const int nA = h, nB = h + NH;
  const bool active = el < ne;
  const bool own_node = M.mij != nullptr && M.info != nullptr;
  const double* tile_src = M.u_in + (int64_t)e0 * NV * ND;
  ElementTileLoad<N, NV, ND, NDP, EPB, NT> tload;
  double u2[2][NV];
  double mij_ab[2] = {0.0, 0.0};
  if (own_node) {
    if (active) {
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const int node = s ? nB : nA;
#pragma unroll
        for (int q = 0; q < NV; ++q)
          u2[s][q] = __ldg(M.u_in + ((int64_t)(e0 + el) * NV + q) * ND + node);
        mij_ab[s] = __ldg(M.mij + (int64_t)(e0 + el) * ND + node);
      }
    }
  } else {
    tload.issue(tile_src, ne, tid);
  }
  __shared__ uint64_t bar_n;
  bool bulk_n = false;
  if constexpr (S::SM_N > 0)
    bulk_n = p.a != 0.0 && (reinterpret_cast<uintptr_t>(M.u_n) & 15u) == 0;
  if (bulk_n && tid == 0) {
    const uint32_t bytes = (uint32_t)ne * NV * ND * sizeof(double);
    mbar_init(&bar_n, 1);
    mbar_fence_init();
    mbar_arrive_expect_tx(&bar_n, bytes);
    if (!p.skip_tile_copy) bulk_copy_g2s(stage_n, M.u_n + (int64_t)e0 * NV * ND, bytes, &bar_n);
  }
  if (M.info) {
    for (int k = tid; k < ne * NI; k += NT) info[k] = __ldg(M.info + (int64_t)e0 * NI + k);
  } else {
    node_element_info<DIM, NI>(M, info, e0, ne, tid, NT);
  }
  if (!own_node) {
    tload.store(tile_src, us, ne, tid);
    __syncthreads();
  }
  if (active) {
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const int node = s ? nB : nA;
      if (own_node) {
#pragma unroll
        for (int q = 0; q < NV; ++q) us[(el * NV + q) * NDP + node] = u2[s][q];
      } else {
#pragma unroll
        for (int q = 0; q < NV; ++q) u2[s][q] = us[(el * NV + q) * NDP + node];
      }
      node_prepare<DIM, N, VF, NDP>(M, u2[s], gamma, info + el * NI, node,
                                    pr + el * NQ * NDP + node, own_node ? &mij_ab[s] : nullptr);
    }
  }
  __syncthreads();

  // ---- phase 2a: face fluxes ---------------------------------------------
  node_face_tasks<DIM, N, VF, SF, false, NDP, NT, NQ, NI>(p, M, us, pr, nullptr, info, sf, ne,
                                                          tid, gamma, t_stage, c0, c1, c2);

  // ---- phase 2b: volume term of both nodes -------------------------------
  // every lane runs it (lanes past the last element of a partial tile read
  // element 0 and discard the result), so the shuffles see full warps
  double accA[NV], accB[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) accA[q] = accB[q] = 0.0;
  {
    const int ev = active ? el : 0;
    const int* I = info + ev * NI;
    const double* U = us + ev * NV * NDP;
    const double* P = pr + ev * NQ * NDP;
    const double hgm1 = 0.5 * p.inv_gm1;
    const NodeFluxState<DIM> ownA = load_flux_state<DIM, VF>(U, P, NDP, nA);
    const NodeFluxState<DIM> ownB = load_flux_state<DIM, VF>(U, P, NDP, nB);
    node_volume_direction<0, DIM, N, VF, NDP, true, false>(p, M, U, P, I, nA, nA, ownA, hgm1,
                                                           accA);
    node_volume_direction<0, DIM, N, VF, NDP, true, false>(p, M, U, P, I, nB, nB, ownB, hgm1,
                                                           accB);
    node_volume_direction<1, DIM, N, VF, NDP, true, false>(p, M, U, P, I, nA, nA, ownA, hgm1,
                                                           accA);
    node_volume_direction<1, DIM, N, VF, NDP, true, false>(p, M, U, P, I, nB, nB, ownB, hgm1,
                                                           accB);
    node2_volume_z<N, VF>(p, M, U, P, I, nA, ownA, ownB, hgm1, accA, accB);
  }
  __syncthreads();
  // the block agrees on a timeout (vote) so that all of it leaves together
  if (bulk_n && __syncthreads_or(!mbar_wait_bounded(&bar_n, 0, p.wait_limit_ns))) {
    if (tid == 0) atomicOr(p.nonfinite, 2u);
    return;
  }
  // fused diagnostics need every thread of the block for the reduction
  const bool diag = p.diag != nullptr;
  if (!active && !diag) return;
  double dacc[3] = {0.0, 0.0, 0.0};

  // ---- phase 3: lifting, -1/J, SSPRK3 combination, store -----------------
  if (active) {
    bool bad = false;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const int node = s ? nB : nA;
      double* acc = s ? accB : accA;
      node_lift<DIM, N>(sf + el * NFACE * NF * NV, node, p.basis.lhat_l0, p.basis.lhat_rN, acc);
      const double mij = pr[(el * NQ + K::MIJ) * NDP + node];
      const int64_t gbase = (int64_t)(e0 + el) * NV * ND + node;
      double vals[NV];
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        const int64_t gi = gbase + (int64_t)q * ND;
        double val = M.c * (acc[q] * mij);
        if (p.b != 0.0) val = p.b * us[(el * NV + q) * NDP + node] + val;
        if (p.a != 0.0)
          val = p.a * (bulk_n ? stage_n[(el * NV + q) * ND + node] : M.u_n[gi]) + val;
        bad |= !isfinite(val);
        M.out[gi] = val;
        vals[q] = val;
      }
      if (diag) diag_add_node<DIM, N>(vals, p.basis, node, -mij, gamma, p.inv_gm1, dacc);
    }
    if (bad) atomicOr(p.nonfinite, 1u);
  }
  if (diag) {
    // the state tile is free after the epilogue (NV * NT >= 3 * NT doubles)
    __syncthreads();
    diag_block_store<NT>(dacc, us, p.diag + 3 * (int64_t)blockIdx.x);
  }
}

template <int N, int VF, int SF>
__global__ void __launch_bounds__(Node2Launch<N>::NT, 4) stage_node2_kernel(const StageArgs<N> p) {
  stage_node2_body<N, VF, SF>(p);
}

}  // namespace dgsem

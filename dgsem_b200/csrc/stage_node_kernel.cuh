// Node-parallel form of the fused stage kernel (split form without shock
// capturing or viscous terms): the same right-hand side and SSPRK3 epilogue
// as stage_kernel.cuh, organised for occupancy instead of minimal flux count.
//
// Per block: EPB elements, EPB * n^d threads.
//   0  element info and the coalesced u_in tile (padded shared memory);
//   1  per-node primitives and -1/J (as stage_kernel.cuh phase 1);
//   2a face tasks: every (face, face node) of the block's elements computes
//      its interface / boundary flux f* once into a shared face buffer
//      (faces of one direction are consecutive, so warps stay uniform);
//   2b one thread per node: for each direction, the two-point fluxes with the
//      n-1 other nodes of its line, sum_k Dsplit(m, k) f(u_m, u_k, (Ja_m +
//      Ja_k)/2), accumulated in registers (each pair is evaluated by both of
//      its nodes: twice the flux work of the symmetric line loop, but no
//      per-direction shared buffers and ~half the registers);
//   3  lifting of the node's face fluxes, -1/J, SSPRK3 combination, store.
// The two-point flux is symmetric in its states, so sum_k Dsplit(m,k) f(u_m,
// u_k) equals the reference's k > i pair loop (volume_flux.hpp:221-410)
// up to summation order.
#pragma once

#include "stage_kernel.cuh"

namespace dgsem {

template <int DIM, int N, int VF, int EPB>
struct NodeShape {
  static constexpr int NV = DIM + 2;
  static constexpr int ND = ipow(N, DIM);
  static constexpr int NDP = ND + ND / N;
  static constexpr int NF = ipow(N, DIM - 1);
  static constexpr int NFACE = 2 * DIM;
  static constexpr int NQ = NodeSlots<DIM, VF>::NQ;
  static constexpr int NI = 12;
  static constexpr int SM_U = EPB * NV * NDP;
  static constexpr int SM_P = EPB * NQ * NDP;
  static constexpr int SM_F = EPB * NFACE * NF * NV;  // f* [el][face][fn][var]
  static constexpr int NT = EPB * ND;
  static constexpr size_t smem_bytes = sizeof(double) * (SM_U + SM_P + SM_F) + sizeof(int) * EPB * NI;
};

template <int DIM, int VF>
__device__ __forceinline__ NodeState<DIM> load_node_state(const double* U, const double* P,
                                                          int NDP, int pn) {
  using Q = NodeSlots<DIM, VF>;
  NodeState<DIM> s;
  s.rho = U[pn];
#pragma unroll
  for (int d = 0; d < DIM; ++d) s.v[d] = P[d * NDP + pn];
  s.p = P[Q::P * NDP + pn];
  s.beta = VF == VF_RANOCHA ? 0.0 : P[Q::BETA * NDP + pn];
  s.kin = VF == VF_CHANDRASHEKAR ? P[Q::KIN * NDP + pn] : 0.0;
  return s;
}

// Volume contribution of direction DIR to node `node` (position m on its line).
template <int DIR, int DIM, int N, int VF, int NDP>
__device__ __forceinline__ void node_volume_direction(const StageArgs<N>& p, const MeshView& M,
                                                      const double* U, const double* P,
                                                      const int* I, int node,
                                                      const NodeState<DIM>& own, double* acc) {
  constexpr int NV = DIM + 2, ND = ipow(N, DIM);
  const int m = DIR == 0 ? node % N : DIR == 1 ? (node / N) % N : node / (N * N);
  const int line = DIR == 0 ? node / N
                   : DIR == 1 ? node % N + N * (node / (N * N))
                              : node % (N * N);
  double ja_own[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) ja_own[c] = __ldg(M.tab.ja[DIR][c] + (int64_t)I[3 + c] * ND + node);
#pragma unroll
  for (int o = 1; o < N; ++o) {
    int k = m + o;
    if (k >= N) k -= N;
    const int nk = line_node<DIM, N>(DIR, line, k);
    const NodeState<DIM> other = load_node_state<DIM, VF>(U, P, NDP, padn<N>(nk));
    double nrm[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c)
      nrm[c] = 0.5 * (ja_own[c] + __ldg(M.tab.ja[DIR][c] + (int64_t)I[3 + c] * ND + nk));
    double f[NV];
    volume_flux<DIM, VF>(own, other, nrm, p.inv_gm1, f);
    const double dmk = p.basis.Dsplit[m][k];
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] += dmk * f[q];
  }
}

template <int DIM, int N, int VF, int SF, int EPB, bool BATCH>
__device__ __forceinline__ void stage_node_body(const StageArgs<N>& p) {
  using S = NodeShape<DIM, N, VF, EPB>;
  using Q = NodeSlots<DIM, VF>;
  constexpr int NV = S::NV, ND = S::ND, NDP = S::NDP, NF = S::NF, NFACE = S::NFACE,
                NQ = S::NQ, NI = S::NI, NT = S::NT;
  extern __shared__ double smem[];
  double* us = smem;             // [el][var][pnode]
  double* pr = us + S::SM_U;     // [el][slot][pnode]
  double* sf = pr + S::SM_P;     // [el][face][fn][var]
  int* info = reinterpret_cast<int*>(sf + S::SM_F);

  const int tid = threadIdx.x;
  __shared__ MeshView mesh_s;
  int e0;
  if constexpr (BATCH) {
    e0 = p.tile_e0[blockIdx.x];
    if (tid == 0) mesh_s = p.meshes[p.tile_mesh[blockIdx.x]];
    __syncthreads();
  } else {
    e0 = (int)blockIdx.x * EPB;
  }
  const MeshView& M = BATCH ? mesh_s : p.mesh;
  const int nelem = M.nelem;
  if (e0 >= nelem) return;
  const int ne = min(EPB, nelem - e0);
  const double gamma = p.gamma;
  const double t_stage = p.t_dev ? (*p.t_dev + p.t) : p.t;
  const int c0 = M.cells[0], c1 = M.cells[1], c2 = M.cells[2];

  // ---- phase 0: element info and the u_in tile --------------------------
  for (int el = tid; el < ne; el += NT) {
    const int e = e0 + el;
    int ijk[3];
    ijk[0] = e % c0;
    ijk[1] = DIM == 2 ? e / c0 : (e / c0) % c1;
    ijk[2] = DIM == 2 ? 0 : e / (c0 * c1);
    int* I = info + el * NI;
    I[0] = ijk[0];
    I[1] = ijk[1];
    I[2] = ijk[2];
    if (DIM == 2) {
      I[3] = ijk[1];
      I[4] = ijk[0];
      I[5] = 0;
    } else {
      I[3] = ijk[1] + c1 * ijk[2];
      I[4] = ijk[0] + c0 * ijk[2];
      I[5] = ijk[0] + c0 * ijk[1];
    }
    const int cells[3] = {c0, c1, c2};
#pragma unroll
    for (int face = 0; face < NFACE; ++face) {
      const int dir = face >> 1, side = face & 1;
      int pos = ijk[dir] + (side ? 1 : -1);
      int nbr = -1;
      if (pos < 0 || pos >= cells[dir]) {
        if (M.periodic[dir]) pos = (pos + cells[dir]) % cells[dir];
        else pos = -1;
      }
      if (pos >= 0) {
        int q[3] = {ijk[0], ijk[1], ijk[2]};
        q[dir] = pos;
        nbr = DIM == 2 ? q[0] + c0 * q[1] : q[0] + c0 * (q[1] + c1 * q[2]);
      }
      I[6 + face] = nbr;
    }
  }
  {
    const double* src = M.u_in + (int64_t)e0 * NV * ND;
    for (int idx = tid; idx < ne * NV * ND; idx += NT) {
      const int row = idx / ND, node = idx % ND;
      us[row * NDP + padn<N>(node)] = __ldg(src + idx);
    }
  }
  __syncthreads();

  // ---- phase 1: node primitives and -1/J ---------------------------------
  for (int idx = tid; idx < ne * ND; idx += NT) {
    const int el = idx / ND, node = idx % ND;
    const int pn = padn<N>(node);
    double u[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) u[q] = us[(el * NV + q) * NDP + pn];
    const NodeState<DIM> s = prepare_node<DIM, VF>(u, gamma);
    double* P = pr + el * NQ * NDP + pn;
#pragma unroll
    for (int d = 0; d < DIM; ++d) P[d * NDP] = s.v[d];
    P[Q::P * NDP] = s.p;
    if (VF != VF_RANOCHA) P[Q::BETA * NDP] = s.beta;
    if (VF == VF_CHANDRASHEKAR) P[Q::KIN * NDP] = s.kin;
    const int* I = info + el * NI;
    const int in = node % N, jn = (node / N) % N, kn = DIM == 3 ? node / (N * N) : 0;
    double jdet = __ldg(M.tab.jdiag[0] + I[0] * N + in);
    if (DIM == 2) {
      jdet = jdet * __ldg(M.tab.jdiag[1] + I[1] * N + jn);
    } else {
      jdet = jdet * (__ldg(M.tab.jdiag[1] + I[1] * N + jn) * __ldg(M.tab.jdiag[2] + I[2] * N + kn));
    }
    P[Q::MIJ * NDP] = -(1.0 / jdet);
  }
  __syncthreads();

  // ---- phase 2a: face fluxes, one task per (element, face, face node) ------
  for (int idx = tid; idx < ne * NFACE * NF; idx += NT) {
    const int el = idx / (NFACE * NF);
    const int face = (idx / NF) % NFACE;
    const int fn = idx % NF;
    const int dir = face >> 1, side = face & 1;
    const int* I = info + el * NI;
    const double* U = us + el * NV * NDP;
    const double* P = pr + el * NQ * NDP;
    double f[NV];
    element_face_flux<DIM, N, VF, SF, false, NDP>(p, M, U, P, nullptr, I, dir, side, fn, gamma,
                                                  t_stage, c0, c1, c2, f);
    double* F = sf + ((el * NFACE + face) * NF + fn) * NV;
#pragma unroll
    for (int q = 0; q < NV; ++q) F[q] = f[q];
  }

  // ---- phase 2b: volume term, one thread per node --------------------------
  double acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q] = 0.0;
  const int el = tid / ND, node = tid % ND;
  const bool active = el < ne;
  if (active) {
    const int* I = info + el * NI;
    const double* U = us + el * NV * NDP;
    const double* P = pr + el * NQ * NDP;
    const NodeState<DIM> own = load_node_state<DIM, VF>(U, P, NDP, padn<N>(node));
    node_volume_direction<0, DIM, N, VF, NDP>(p, M, U, P, I, node, own, acc);
    node_volume_direction<1, DIM, N, VF, NDP>(p, M, U, P, I, node, own, acc);
    if constexpr (DIM == 3) node_volume_direction<2, DIM, N, VF, NDP>(p, M, U, P, I, node, own, acc);
  }
  __syncthreads();
  if (!active) return;

  // ---- phase 3: lifting (surface_integral.hpp:35-154), -1/J, SSPRK3 --------
  {
    const int pos[3] = {node % N, (node / N) % N, DIM == 3 ? node / (N * N) : 0};
#pragma unroll
    for (int dir = 0; dir < DIM; ++dir) {
      const int line = dir == 0 ? node / N
                       : dir == 1 ? node % N + N * (node / (N * N))
                                  : node % (N * N);
      if (pos[dir] == 0) {
        const double* F = sf + ((el * NFACE + 2 * dir) * NF + line) * NV;
#pragma unroll
        for (int q = 0; q < NV; ++q) acc[q] -= F[q] * p.basis.lhat_l0;
      }
      if (pos[dir] == N - 1) {
        const double* F = sf + ((el * NFACE + 2 * dir + 1) * NF + line) * NV;
#pragma unroll
        for (int q = 0; q < NV; ++q) acc[q] += F[q] * p.basis.lhat_rN;
      }
    }
  }
  const int pn = padn<N>(node);
  const double mij = pr[(el * NQ + Q::MIJ) * NDP + pn];
  const int64_t gbase = (int64_t)(e0 + el) * NV * ND + node;
  bool bad = false;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    const double du = acc[q] * mij;
    const int64_t gi = gbase + (int64_t)q * ND;
    double val = M.c * du;
    if (p.b != 0.0) val = p.b * us[(el * NV + q) * NDP + pn] + val;
    if (p.a != 0.0) val = p.a * M.u_n[gi] + val;
    bad |= !isfinite(val);
    M.out[gi] = val;
  }
  if (bad) atomicOr(p.nonfinite, 1u);
}

template <int DIM, int N, int VF, int SF, int EPB, bool BATCH>
__global__ void __launch_bounds__(EPB* ipow(N, DIM)) stage_node_kernel(const StageArgs<N> p) {
  stage_node_body<DIM, N, VF, SF, EPB, BATCH>(p);
}

}  // namespace dgsem

// Node-parallel form of the fused stage kernel (split form, optionally with
// Hennemann-Gassner shock capturing in 2D; no viscous terms): the same
// right-hand side and SSPRK3 epilogue as stage_kernel.cuh, organised for
// occupancy instead of minimal flux count.
//
// Per block: EPB elements, EPB * n^d threads.
//   0  element info and the coalesced u_in tile (unpadded shared memory);
//   1  per-node flux data (NodeKernelSlots), squared sound speed and -1/J;
//   2a face tasks: every (face, face node) of the block's elements computes
//      its interface / boundary flux f* once into a shared face buffer
//      (tasks grouped by side and direction, so a warp's lanes share both and
//      evaluate the flux in one argument order);
//   2b one thread per node: for each direction, the two-point fluxes with the
//      n-1 other nodes of its line, sum_k Dsplit(m, k) f(u_m, u_k, (Ja_m +
//      Ja_k)/2), accumulated in registers; the pair (m, m+o), o < n-o, is
//      evaluated by node m and handed to node m+o by warp shuffle (lines
//      inside one warp) or through a shared buffer (other x/y lines), z lines
//      evaluate each pair at both nodes (~60 % of the registers of the line
//      loop);
//   3  lifting of the node's face fluxes, -1/J, SSPRK3 combination, store;
//      the u_n tile of the combination is requested at kernel start as one
//      bulk (TMA) copy into shared memory (16-byte-aligned states with an
//      even number of doubles per element; otherwise read directly).
// The two-point flux is symmetric in its states, so sum_k Dsplit(m,k) f(u_m,
// u_k) equals the reference's k > i pair loop (volume_flux.hpp:221-410)
// up to summation order.
//
// Halved node data: the averages of the Kennedy-Gruber and Chandrashekar
// fluxes, 0.5 (a + b), and the pair normal 0.5 (Ja_m + Ja_k) are formed as
// a/2 + b/2 from values halved once per node.  Scaling by 1/2 is exact in
// binary floating point, so each average is bit for bit the same while the
// per-pair multiplications disappear.
#pragma once

#include "stage_kernel.cuh"
#include "tma.cuh"

namespace dgsem {

// Shared-memory slots per node (the conserved density comes from the tile).
//   KG / Chandrashekar: V (v/2, DIM), P (p/2), A (squared sound speed), MIJ (-1/J),
//                       H_RHO (rho/2), X (KG: e/2; Chandrashekar: beta),
//                       Y (Chandrashekar: |v|^2/4)
//   Ranocha:            V (v), P (p), A, MIJ
template <int DIM, int VF>
struct NodeKernelSlots {
  static constexpr bool HALF = VF != VF_RANOCHA;
  static constexpr int V = 0;
  static constexpr int P = DIM;
  static constexpr int A = DIM + 1;
  static constexpr int MIJ = DIM + 2;
  static constexpr int H_RHO = DIM + 3;
  static constexpr int X = DIM + 4;
  static constexpr int Y = DIM + 5;
  static constexpr int NQ = VF == VF_CHANDRASHEKAR ? DIM + 6
                            : VF == VF_KENNEDY_GRUBER ? DIM + 5 : DIM + 3;
};

template <int DIM, int N, int VF, int EPB, bool HG = false, bool NS = false>
struct NodeShape {
  static constexpr int NV = DIM + 2;
  static constexpr int ND = ipow(N, DIM);
  static constexpr bool PAD = false;  // unpadded node arrays (see padn)
  static constexpr int NDP = PAD ? ND + ND / N : ND;
  static constexpr int NF = ipow(N, DIM - 1);
  static constexpr int NFACE = 2 * DIM;
  static constexpr int NQ = NodeKernelSlots<DIM, VF>::NQ;
  static constexpr int NI = 12;
  static constexpr int SM_U = EPB * NV * NDP;
  static constexpr int SM_P = EPB * NQ * NDP;
  // f* [el][face][fn][var]; with shock capturing also the indicator scratch
  static constexpr int SM_F0 = EPB * NFACE * NF * NV;
  static constexpr int SM_F = HG && 2 * EPB * ND > SM_F0 ? 2 * EPB * ND : SM_F0;
  static constexpr int SM_A = HG ? EPB : 0;        // alpha per element
  static constexpr int SM_VINV = HG ? N * N : 0;   // inverse Legendre Vandermonde
  // volume-term exchange buffer [round][var][thread]: fluxes of the pairs
  // (m, m+o), o = 1..XR, on x and y lines that do not lie in one warp (see
  // node_volume_direction); lines inside a warp use shuffles instead, and z
  // lines (3D) evaluate each pair twice (at n = 4 the exchange cost as much
  // as it saved there and took shared memory from the persistent shape)
  static constexpr int XR = (N - 1) / 2;
  static constexpr bool WARP_ALL = (EPB * ND) % 32 == 0;
  static constexpr bool XCHG = XR > 0 && (!WARP_ALL || 32 % N != 0 || 32 % (N * N) != 0);
  static constexpr int SM_X = XCHG ? XR * NV * EPB * ND : 0;
  // staged u_n tile (one bulk copy) when a tile is a multiple of 16 bytes;
  // placed last so that launches without u_n (stage 1, RHS) can request
  // smem_bytes_base and leave the rest of the SM's storage to L1
  static constexpr int SM_N = (NV * ND) % 2 == 0 ? EPB * NV * ND : 0;
  static constexpr int NT = EPB * ND;
  // Navier-Stokes: -F_v per node [el][dim][var][node]
  static constexpr int SM_W = NS ? EPB * DIM * NV * ND : 0;
  static constexpr size_t smem_bytes_base =
      sizeof(double) * (SM_U + SM_P + SM_F + SM_A + SM_VINV + SM_X + SM_W) +
      sizeof(int) * EPB * NI;
  static constexpr size_t off_n_bytes = (smem_bytes_base + 15) / 16 * 16;
  static constexpr size_t smem_bytes = off_n_bytes + sizeof(double) * SM_N;
};

// Node data of one two-point flux evaluation (halved where NodeKernelSlots
// says so).
template <int DIM>
struct NodeFluxState {
  double rho;     // conserved density
  double hrho;    // rho / 2
  double v[DIM];  // v / 2 (KG, Chandrashekar) or v (Ranocha)
  double p;       // p / 2 (KG, Chandrashekar) or p (Ranocha)
  double x;       // KG: e / 2; Chandrashekar: beta
  double y;       // Chandrashekar: |v|^2 / 4
};

template <int DIM, int VF>
__device__ __forceinline__ NodeFluxState<DIM> load_flux_state(const double* U, const double* P,
                                                              int NDP, int pn) {
  using K = NodeKernelSlots<DIM, VF>;
  NodeFluxState<DIM> s;
  s.rho = U[pn];
#pragma unroll
  for (int d = 0; d < DIM; ++d) s.v[d] = P[(K::V + d) * NDP + pn];
  s.p = P[K::P * NDP + pn];
  // Chandrashekar loads rho anyway: rho / 2 is exact, so derive it instead
  // of a second shared-memory load (Kennedy-Gruber uses only rho / 2)
  s.hrho = !K::HALF ? 0.0 : VF == VF_CHANDRASHEKAR ? 0.5 * s.rho : P[K::H_RHO * NDP + pn];
  s.x = K::HALF ? P[K::X * NDP + pn] : 0.0;
  // |v|^2 / 4 = sum (v_d / 2)^2 from the halved velocity, in the summation
  // order of prepare_node: bit for bit the stored value, one load fewer
  s.y = 0.0;
  if constexpr (VF == VF_CHANDRASHEKAR) {
#pragma unroll
    for (int d = 0; d < DIM; ++d) s.y += s.v[d] * s.v[d];
  }
  return s;
}

// Two-point volume flux on node data; `n` is the full pair normal
// (Ja_m + Ja_k)/2, `hgm1` = 1 / (2 (gamma - 1)).  Same formulas as
// physics.cuh:volume_flux with the 1/2 factors moved into the node data.
template <int DIM, int VF>
__device__ __forceinline__ void node_volume_flux(const NodeFluxState<DIM>& L,
                                                 const NodeFluxState<DIM>& R, const double* n,
                                                 double inv_gm1, double hgm1, double* f) {
  if constexpr (VF == VF_KENNEDY_GRUBER) {
    const double rho_avg = L.hrho + R.hrho;
    const double e_avg = L.x + R.x;
    const double p_avg = L.p + R.p;
    double va[DIM], vn_avg = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      va[d] = L.v[d] + R.v[d];
      vn_avg += va[d] * n[d];
    }
    const double f1 = rho_avg * vn_avg;
    f[0] = f1;
#pragma unroll
    for (int d = 0; d < DIM; ++d) f[1 + d] = f1 * va[d] + p_avg * n[d];
    f[DIM + 1] = (rho_avg * e_avg + p_avg) * vn_avg;
  } else if constexpr (VF == VF_CHANDRASHEKAR) {
    double hvnL = 0.0, hvnR = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      hvnL += L.v[d] * n[d];
      hvnR += R.v[d] * n[d];
    }
    double rho_mean, inv_beta_mean, inv_beta_sum;
    chandrashekar_means(L.rho, R.rho, L.x, R.x, rho_mean, inv_beta_mean, inv_beta_sum);
    const double p_mean = (L.hrho + R.hrho) * inv_beta_sum;
    const double f1 = rho_mean * (hvnL + hvnR);
    f[0] = f1;
    double fe = f1 * (hgm1 * inv_beta_mean - (L.y + R.y));
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      const double va = L.v[d] + R.v[d];
      const double fm = f1 * va + p_mean * n[d];
      f[1 + d] = fm;
      fe += fm * va;
    }
    f[DIM + 1] = fe;
  } else {  // Ranocha on unhalved data
    NodeState<DIM> l, r;
    l.rho = L.rho;
    r.rho = R.rho;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      l.v[d] = L.v[d];
      r.v[d] = R.v[d];
    }
    l.p = L.p;
    r.p = R.p;
    l.beta = r.beta = l.kin = r.kin = 0.0;
    volume_flux<DIM, VF_RANOCHA>(l, r, n, inv_gm1, f);
  }
}

// Volume contribution of direction DIR to the node at shared-memory position
// `pn`, node index `node`, position m on its line.  WARP_ALL: every lane of
// the calling warp executes the call (thread = element * n^d + node, blocks
// a multiple of 32 threads); then, where a whole line of direction DIR lies
// in one warp, the partners' metric terms come from the partners' lanes by
// shuffle instead of a second global load (the same values, so the same
// normal bit for bit).  XB: the whole block executes the call and `xbuf`
// holds (n-1)/2 * NV * nth doubles; pairs on lines that do not lie in one
// warp are then shared through it (two block barriers per direction).
template <int DIR, int DIM, int N, int VF, int NDP, bool WARP_ALL = false, bool XB = false>
__device__ __forceinline__ void node_volume_direction(const StageArgs<N>& p, const MeshView& M,
                                                      const double* U, const double* P,
                                                      const int* I, int node, int pn,
                                                      const NodeFluxState<DIM>& own,
                                                      double hgm1, double* acc,
                                                      double* xbuf = nullptr, int tid = 0,
                                                      int nth = 0, bool in_range = true) {
  constexpr int NV = DIM + 2, ND = ipow(N, DIM);
  constexpr bool HALF = NodeKernelSlots<DIM, VF>::HALF;
  // node-index and shared-memory-index strides along DIR
  constexpr int SN = DIR == 0 ? 1 : DIR == 1 ? N : N * N;
  constexpr int SP = NDP == ND ? SN : DIR == 0 ? 1 : DIR == 1 ? N + 1 : N * N + N;
  const int m = DIR == 0 ? node % N : DIR == 1 ? (node / N) % N : node / (N * N);
  const double* jrow[DIM];
  double hja_own[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    jrow[c] = M.tab.ja[DIR][c] + (int64_t)I[3 + c] * ND + node;
    const double j = __ldg(jrow[c]);
    hja_own[c] = HALF ? 0.5 * j : j;
  }
  // lines of DIR inside one warp: N | 32 for DIR 0, N^2 | 32 for DIR 1
  constexpr bool SHFL = WARP_ALL && (DIR == 0 ? 32 % N == 0 : DIR == 1 ? 32 % (N * N) == 0 : false);
  constexpr int XR = (N - 1) / 2;
  constexpr bool XCHG = XB && !SHFL && XR > 0 && DIR < 2;
  const double* Dm = &p.basis.Dsplit[m][0];
  const int lane = (int)(threadIdx.x & 31u);
#pragma unroll
  for (int o = 1; o < N; ++o) {
    // The pair (m, m + o) for o < N - o is evaluated once, by node m, and
    // handed on to node m + o (by shuffle within a warp, else through xbuf):
    // the two-point flux and the pair normal are symmetric in the two nodes,
    // so the partners o > N - o arrive from round N - o instead of being
    // evaluated a second time.
    if ((SHFL || XCHG) && o > N - o) continue;
    const bool wrap = m + o >= N;
    const int delta = wrap ? o - N : o;  // k - m
    const NodeFluxState<DIM> other = load_flux_state<DIM, VF>(U, P, NDP, pn + delta * SP);
    double nrm[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      if constexpr (SHFL) {
        // the partner's own (halved when HALF) value: 0.5 * jk exactly
        const double hjk = __shfl_sync(0xffffffffu, hja_own[c], lane + delta * SN);
        nrm[c] = HALF ? hja_own[c] + hjk : 0.5 * (hja_own[c] + hjk);
      } else {
        const double jk = __ldg(jrow[c] + delta * SN);
        nrm[c] = HALF ? hja_own[c] + 0.5 * jk : 0.5 * (hja_own[c] + jk);
      }
    }
    double f[NV];
    node_volume_flux<DIM, VF>(own, other, nrm, p.inv_gm1, hgm1, f);
    const double dmk = Dm[m + delta];
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] += dmk * f[q];
    if (SHFL && o < N - o) {
      // f(m - o, m) from the node o back along the line (wrapping)
      const int back = m - o < 0 ? N - o : -o;  // (m - o) mod N - m
      const double dmb = Dm[m + back];
#pragma unroll
      for (int q = 0; q < NV; ++q)
        acc[q] += dmb * __shfl_sync(0xffffffffu, f[q], lane + back * SN);
    }
    if (XCHG && o < N - o && in_range) {
#pragma unroll
      for (int q = 0; q < NV; ++q) xbuf[((o - 1) * NV + q) * nth + tid] = f[q];
    }
  }
  if constexpr (XCHG) {
    __syncthreads();
    if (in_range) {
#pragma unroll
      for (int o = 1; o <= XR; ++o) {
        const int back = m - o < 0 ? N - o : -o;
        const double dmb = Dm[m + back];
#pragma unroll
        for (int q = 0; q < NV; ++q)
          acc[q] += dmb * xbuf[((o - 1) * NV + q) * nth + tid + back * SN];
      }
    }
    // direction 1 reuses the buffer; after direction 1 (the last one that
    // exchanges: z lines never do) the block passes another barrier before
    // anything writes it again
    if constexpr (DIR == 0) __syncthreads();
  }
}

// Hennemann-Gassner FV subcell contribution of direction DIR to the node
// (volume_flux.hpp:457-509 in 2D, :521-630 in 3D): LLF on the subcell normals
// at the node's two subcell interfaces, weighted by alpha / w_m (each
// interface flux is evaluated by both of its nodes).
template <int DIR, int DIM, int N, int VF, int NDP>
__device__ __forceinline__ void node_fv_direction(const StageArgs<N>& p, const MeshView& M,
                                                  const double* U, const double* P,
                                                  const int* I, int node, double alpha,
                                                  double* acc) {
  constexpr int NV = DIM + 2;
  constexpr int NF = ipow(N, DIM - 1);
  using K = NodeKernelSlots<DIM, VF>;
  const int m = DIR == 0 ? node % N : DIR == 1 ? (node / N) % N : node / (N * N);
  const int line = DIR == 0 ? node / N
                   : DIR == 1 ? node % N + N * (node / (N * N))
                              : node % (N * N);
  auto state = [&](int k) {
    const int pk = padn<N, (NDP != ipow(N, DIM))>(line_node<DIM, N>(DIR, line, k));
    FaceState<DIM> st;
#pragma unroll
    for (int q = 0; q < NV; ++q) st.u[q] = U[q * NDP + pk];
    const double g = K::HALF ? 2.0 : 1.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) st.v[d] = g * P[(K::V + d) * NDP + pk];
    st.p = g * P[K::P * NDP + pk];
    st.a2 = P[K::A * NDP + pk];
    return st;
  };
  auto normal = [&](int fi, double* nrm) {
#pragma unroll
    for (int c = 0; c < DIM; ++c)
      nrm[c] = __ldg(M.tab.fv[DIR][c] + (int64_t)I[3 + c] * (N - 1) * NF + (fi - 1) * NF + line);
  };
  const double w = alpha * p.basis.inv_w[m];
  const FaceState<DIM> own = state(m);
  // s = 0: interface fi = m, this node is its right node (-w f);
  // s = 1: interface fi = m + 1, this node is its left node (+w f).
  // One flux evaluation site keeps the kernel's code small.
#pragma unroll 1
  for (int s = 0; s < 2; ++s) {
    const int fi = m + s;
    if (fi < 1 || fi > N - 1) continue;
    double nrm[DIM], f[NV];
    normal(fi, nrm);
    const FaceState<DIM> other = state(s ? m + 1 : m - 1);
    FaceState<DIM> L, R;
    order_states<DIM>(s != 0, own, other, L, R);
    llf_flux<DIM>(L, R, nrm, f);
    const double ws = s ? w : -w;
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] += ws * f[q];
  }
}

// NTB: threads of the launch (>= EPB * n^d; the threads past EPB * n^d only
// take part in the block's barriers).  PERSIST: batched launches whose
// tiles come from a work list (`tile`), without the bulk copy of u_n.
// Element info of a tile, info[el * NI + entry]: 0-2 the element's indices,
// 3-5 its row in the metric tables of each axis (the indices of the other
// axes), 6.. the neighbour across each face (-1 at a boundary face; unused
// entries -1).  One entry per thread, so the whole tile's info is one pass
// of ne * NI threads instead of a serial loop per element.
template <int DIM, int NI>
__device__ __forceinline__ void node_element_info(const MeshView& M, int* info, int e0, int ne,
                                                  int tid, int nt) {
  const int c0 = M.cells[0], c1 = M.cells[1], c2 = M.cells[2];
  for (int k = tid; k < ne * NI; k += nt) {
    const int el = k / NI, entry = k - el * NI;
    const int e = e0 + el;
    const int i0 = e % c0;
    const int i1 = DIM == 2 ? e / c0 : (e / c0) % c1;
    const int i2 = DIM == 2 ? 0 : e / (c0 * c1);
    int v = -1;
    if (entry == 0) v = i0;
    else if (entry == 1) v = i1;
    else if (entry == 2) v = i2;
    else if (entry == 3) v = DIM == 2 ? i1 : i1 + c1 * i2;
    else if (entry == 4) v = DIM == 2 ? i0 : i0 + c0 * i2;
    else if (entry == 5) v = DIM == 2 ? 0 : i0 + c0 * i1;
    else if (entry < 6 + 2 * DIM) {
      const int face = entry - 6, dir = face >> 1;
      const int id = dir == 0 ? i0 : dir == 1 ? i1 : i2;
      const int cd = dir == 0 ? c0 : dir == 1 ? c1 : c2;
      const int stride = dir == 0 ? 1 : dir == 1 ? c0 : c0 * c1;
      int pos = id + ((face & 1) ? 1 : -1);
      if (pos < 0 || pos >= cd) pos = M.periodic[dir] ? (pos + cd) % cd : -1;
      v = pos < 0 ? -1 : e + (pos - id) * stride;
    }
    info[k] = v;
  }
}

// -1/J of a node from the separable tables: 1/J = 1/(J00 J11 [J22]) (the
// off-diagonal products do not change the rounded determinant).
template <int DIM, int N>
__device__ __forceinline__ double node_minus_inv_j(const DeviceTables& tab, int i0, int i1,
                                                   int i2, int in, int jn, int kn) {
  double jdet = __ldg(tab.jdiag[0] + i0 * N + in);
  if (DIM == 2) {
    jdet = jdet * __ldg(tab.jdiag[1] + i1 * N + jn);
  } else {
    jdet = jdet * (__ldg(tab.jdiag[1] + i1 * N + jn) * __ldg(tab.jdiag[2] + i2 * N + kn));
  }
  return -(1.0 / jdet);
}

// The per-mesh tables of the node-parallel kernels (MeshView::info, ::mij),
// once per context: every element's info entries (node_element_info) and
// -1/J of every node.  One thread per (element, node).
template <int DIM, int N, int NI>
__global__ void element_tables_kernel(const MeshView M, int* info, double* mij) {
  constexpr int ND = ipow(N, DIM);
  const int64_t total = (int64_t)M.nelem * ND;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += stride) {
    const int e = (int)(g / ND), node = (int)(g % ND);
    const int c0 = M.cells[0], c1 = M.cells[1];
    const int i0 = e % c0;
    const int i1 = DIM == 2 ? e / c0 : (e / c0) % c1;
    const int i2 = DIM == 2 ? 0 : e / (c0 * c1);
    const int in = node % N, jn = (node / N) % N, kn = DIM == 3 ? node / (N * N) : 0;
    mij[g] = node_minus_inv_j<DIM, N>(M.tab, i0, i1, i2, in, jn, kn);
  }
  // element info: the tile function over all elements as one tile
  node_element_info<DIM, NI>(M, info, 0, M.nelem, (int)(blockIdx.x * blockDim.x + threadIdx.x),
                             (int)(gridDim.x * blockDim.x));
}

// Per-node data of phase 1 (NodeKernelSlots) from the conserved state u:
// the (halved) primitive variables, the squared sound speed gamma p / rho and
// -1/J from the separable metric tables.
template <int DIM, int N, int VF, int NDP>
__device__ __forceinline__ void node_prepare(const MeshView& M, const double* u, double gamma,
                                             const int* I, int node, double* P,
                                             const double* mij_pre = nullptr) {
  using K = NodeKernelSlots<DIM, VF>;
  const NodeState<DIM> s = prepare_node<DIM, VF>(u, gamma);
  const double h = K::HALF ? 0.5 : 1.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) P[(K::V + d) * NDP] = h * s.v[d];
  P[K::P * NDP] = h * s.p;
  // used only by the wave-speed estimate of the surface flux: gamma p (1/rho)
  // is within an ulp of gamma p / rho
  P[K::A * NDP] = gamma * s.p * s.inv_rho;
  if constexpr (K::HALF) {
    P[K::H_RHO * NDP] = 0.5 * u[0];
    P[K::X * NDP] = VF == VF_KENNEDY_GRUBER ? 0.5 * s.beta : s.beta;
  }
  if constexpr (VF == VF_CHANDRASHEKAR) P[K::Y * NDP] = 0.5 * s.kin;
  if (mij_pre) {  // element_tables_kernel computed it with the expression below
    P[K::MIJ * NDP] = *mij_pre;
    return;
  }
  const int in = node % N, jn = (node / N) % N, kn = DIM == 3 ? node / (N * N) : 0;
  P[K::MIJ * NDP] = node_minus_inv_j<DIM, N>(M.tab, I[0], I[1], I[2], in, jn, kn);
}

// Surface lifting of one node (surface_integral.hpp:35-154): per direction,
// -lhat_l0 f* of the low face or +lhat_rN f* of the high face when the node
// lies on it.  Branch-free: every node reads one face flux per direction and
// interior nodes add it with the factor 0 (acc + 0 f = acc), so the lanes of
// a warp do not diverge over the faces.  sf_el = face buffer of the element.
template <int DIM, int N>
__device__ __forceinline__ void node_lift(const double* sf_el, int node, double lhat_l0,
                                          double lhat_rN, double* acc) {
  constexpr int NV = DIM + 2, NF = ipow(N, DIM - 1);
  const int pos[3] = {node % N, (node / N) % N, DIM == 3 ? node / (N * N) : 0};
#pragma unroll
  for (int dir = 0; dir < DIM; ++dir) {
    const int line = dir == 0   ? node / N
                     : dir == 1 ? node % N + N * (node / (N * N))
                                : node % (N * N);
    const bool hi = pos[dir] == N - 1;
    const double coef = pos[dir] == 0 ? -lhat_l0 : hi ? lhat_rN : 0.0;
    const double* F = sf_el + ((2 * dir + (hi ? 1 : 0)) * NF + line) * NV;
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] += coef * F[q];
  }
}

// Phase 2a of the node-parallel kernels: the interface / boundary flux f* of
// every (element, face, face node) of the tile, once, into the face buffer
// sf[el][face][fn][var].  The lanes of a warp share the face side, so they
// evaluate the flux in one argument order.
//   3D: tasks grouped by (side, direction), both compile-time constants in
//       the flux code (no runtime-indexed arrays); inside a group the order
//       is element-major, and a group fills whole warps where ne * NF is a
//       multiple of 32.  Task idx of the tile goes to thread idx % NT.
//   2D: one block-stride loop over the tasks in side-major order with the
//       direction at run time (measured faster there: the boundary branch
//       of the flux code then exists once).
template <int DIM, int N, int VF, int SF, bool NS, int NDP, int NT, int NQ, int NI>
__device__ __forceinline__ void node_face_tasks(const StageArgs<N>& p, const MeshView& M,
                                                const double* us, const double* pr,
                                                const double* wv, const int* info, double* sf,
                                                int ne, int tid, double gamma, double t_stage,
                                                int c0, int c1, int c2) {
  using K = NodeKernelSlots<DIM, VF>;
  constexpr int NV = DIM + 2, ND = ipow(N, DIM), NF = ipow(N, DIM - 1), NFACE = 2 * DIM;
  auto task = [&](int side, int dir, int fe, int fn) {
    const int face = 2 * dir + side;
    const int* I = info + fe * NI;
    const double* U = us + fe * NV * NDP;
    const double* P = pr + fe * NQ * NDP;
    const int opn = padn<N, NDP != ND>(line_node<DIM, N>(dir, fn, side ? N - 1 : 0));
    FaceState<DIM> so;
#pragma unroll
    for (int q = 0; q < NV; ++q) so.u[q] = U[q * NDP + opn];
    const double g = K::HALF ? 2.0 : 1.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) so.v[d] = g * P[(K::V + d) * NDP + opn];
    so.p = g * P[K::P * NDP + opn];
    so.a2 = P[K::A * NDP + opn];
    double f[NV];
    element_face_flux_state<DIM, N, VF, SF, NS, NDP>(p, M, so, U,
                                                     NS ? wv + fe * DIM * NV * ND : nullptr, I,
                                                     dir, side, fn, gamma, t_stage, c0, c1, c2,
                                                     f);
    double* F = sf + ((fe * NFACE + face) * NF + fn) * NV;
#pragma unroll
    for (int q = 0; q < NV; ++q) F[q] = f[q];
  };
  if constexpr (DIM == 3) {
    const int gsz = ne * NF;
#pragma unroll
    for (int side = 0; side < 2; ++side) {
#pragma unroll
      for (int dir = 0; dir < DIM; ++dir) {
        const int gbase = (side * DIM + dir) * gsz;
        int r = tid - gbase % NT;
        if (r < 0) r += NT;
        for (; r < gsz; r += NT) task(side, dir, r / NF, r - (r / NF) * NF);
      }
    }
  } else {
    for (int idx = tid; idx < ne * NFACE * NF; idx += NT) {
      const int side = idx >= ne * DIM * NF ? 1 : 0;
      const int r = idx - side * ne * DIM * NF;
      task(side, (r / NF) % DIM, r / (DIM * NF), r % NF);
    }
  }
}

template <int DIM, int N, int VF, int SF, int EPB, bool BATCH, bool HG, bool NS = false,
          int NTB = 0, bool PERSIST = false>
__device__ __forceinline__ void stage_node_body(const StageArgs<N>& p, int tile = 0) {
  static_assert(!NS || (!BATCH && (!HG || DIM == 2)),
                "Navier-Stokes: single mesh; with shock capturing in 2D");
  using S = NodeShape<DIM, N, VF, EPB, HG, NS>;
  using K = NodeKernelSlots<DIM, VF>;
  constexpr int NV = S::NV, ND = S::ND, NDP = S::NDP, NF = S::NF, NFACE = S::NFACE,
                NQ = S::NQ, NI = S::NI, NT = S::NT;
  extern __shared__ __align__(128) double smem_node[];
  double* us = smem_node;        // [el][var][pnode]
  double* pr = us + S::SM_U;     // [el][slot][pnode]
  double* sf = pr + S::SM_P;     // [el][face][fn][var]
  double* alpha_s = sf + S::SM_F;          // [el] (shock capturing)
  double* vinv_s = alpha_s + S::SM_A;      // [N][N] (shock capturing)
  double* xbuf = vinv_s + S::SM_VINV;      // volume-term exchange
  double* wv = xbuf + S::SM_X;             // Navier-Stokes -F_v [el][dim][var][node]
  int* info = reinterpret_cast<int*>(wv + S::SM_W);
  // [el][var][node] u_n tile (bulk-copy target; present when p.a != 0)
  double* stage_n = reinterpret_cast<double*>(reinterpret_cast<char*>(smem_node) + S::off_n_bytes);

  const int tid = threadIdx.x;
  __shared__ MeshView mesh_s;
  int e0;
  // threads past the element tile (wider persistent blocks) only join barriers
  const bool worker = NTB == 0 || tid < NT;
  // the tile list and the mesh views are written by host copies only, so
  // they are read before waiting for the previous kernel
  if constexpr (BATCH) {
    static_assert((NTB > 0 ? NTB : NT) >= int(sizeof(MeshView) / 8),
                  "block narrower than the mesh view");
    const int tl = PERSIST ? tile : (int)blockIdx.x;
    e0 = p.tile_e0[tl];
    copy_mesh_view(&mesh_s, p.meshes, p.tile_mesh[tl], tid);
  } else {
    e0 = (int)blockIdx.x * EPB;
  }
  stage_dependency_sync();
  if constexpr (BATCH) __syncthreads();
  const MeshView& M = BATCH ? mesh_s : p.mesh;
  const int nelem = M.nelem;
  if (e0 >= nelem) return;
  const int ne = min(EPB, nelem - e0);
  const double gamma = p.gamma;
  const double t_stage = p.t_dev ? (*p.t_dev + p.t) : p.t;
  const int c0 = M.cells[0], c1 = M.cells[1], c2 = M.cells[2];

  // ---- phases 0 and 1: the u_in tile, the epilogue's u_n tile, element
  // info, node data ----------------------------------------------------------
  // With the mesh's tables (single-mesh launches: -1/J and the element info
  // precomputed) every thread reads its own node's state, coalesced per
  // variable, and computes its node data without waiting for the rest of the
  // tile: one barrier for both phases.  Otherwise the tile's loads are issued
  // first, the element info is computed while they are in flight, and the
  // node data follow a barrier.  Either way the u_n tile is requested as one
  // bulk copy that arrives while the block computes (block-uniform decision).
  const int el = tid / ND, node = tid % ND;
  const bool active = el < ne;
  const int pn = padn<N, S::PAD>(node);
  const bool own_node = M.mij != nullptr && M.info != nullptr;
  const double* tile_src = M.u_in + (int64_t)e0 * NV * ND;
  ElementTileLoad<N, NV, ND, NDP, EPB, NT> tload;
  double u[NV];
  double mij_node = 0.0;
  if (own_node) {
    if (active) {
#pragma unroll
      for (int q = 0; q < NV; ++q)
        u[q] = __ldg(M.u_in + ((int64_t)(e0 + el) * NV + q) * ND + node);
      mij_node = __ldg(M.mij + (int64_t)(e0 + el) * ND + node);
    }
  } else if (worker) {
    tload.issue(tile_src, ne, tid);
  }
  __shared__ uint64_t bar_n;
  bool bulk_n = false;
  if constexpr (S::SM_N > 0 && !PERSIST)
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
  if constexpr (HG) {
    for (int k = tid; k < N * N; k += NT) vinv_s[k] = p.basis.Vinv[k / N][k % N];
  }
  // node data, squared sound speed and -1/J (and -F_v with viscous terms)
  auto node_data = [&](const double* u) {
    node_prepare<DIM, N, VF, NDP>(M, u, gamma, info + el * NI, node, pr + el * NQ * NDP + pn,
                                  own_node ? &mij_node : nullptr);
    if constexpr (NS && DIM == 3) {
      // -F_v at the node from the lifted gradient (parabolic_viscous.hpp:358-396)
      double q[5], g[3][4];
      ns_gradient_variables_3d(u, gamma, q);
      const double* G = p.grad + (int64_t)(e0 + el) * 4 * 3 * ND + node;
#pragma unroll
      for (int v = 0; v < 4; ++v)
#pragma unroll
        for (int d = 0; d < 3; ++d) g[d][v] = __ldg(G + (v * 3 + d) * ND);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        double f[5];
        ns_neg_viscous_flux_3d(q, g, p.mu, p.kappa, d, f);
#pragma unroll
        for (int v = 0; v < 5; ++v) wv[((el * 3 + d) * NV + v) * ND + node] = f[v];
      }
    } else if constexpr (NS) {
      // -F_v at the node from the lifted gradient (parabolic_viscous.hpp:358-396)
      double q[4], gx[4], gy[4];
      ns_gradient_variables(u, gamma, q);
      const double* G = p.grad + (int64_t)(e0 + el) * 4 * 2 * ND + node;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        gx[v] = __ldg(G + (v * 2 + 0) * ND);
        gy[v] = __ldg(G + (v * 2 + 1) * ND);
      }
#pragma unroll
      for (int d = 0; d < 2; ++d) {
        double f[4];
        ns_neg_viscous_flux(q, gx, gy, p.mu, p.kappa, d, f);
#pragma unroll
        for (int v = 0; v < 4; ++v) wv[((el * 2 + d) * NV + v) * ND + node] = f[v];
      }
    }
  };
  if (own_node) {
    if (active) {
#pragma unroll
      for (int q = 0; q < NV; ++q) us[(el * NV + q) * NDP + pn] = u[q];
      node_data(u);
    }
  } else {
    if (worker) tload.store(tile_src, us, ne, tid);
    __syncthreads();
    if (active) {
#pragma unroll
      for (int q = 0; q < NV; ++q) u[q] = us[(el * NV + q) * NDP + pn];
      node_data(u);
    }
  }
  __syncthreads();

  // ---- phase 1b: Hennemann-Gassner alpha per element (indicator.hpp:337-418),
  // node-parallel with the same explicitly rounded arithmetic as
  // stage_kernel.cuh (identical alpha and troubled-cell flags); scratch in the
  // face buffer, which is written only afterwards ------------------------------
  if constexpr (HG) {
    // two scratch arrays used in turn: node values (A) -> x pass (B) -> y
    // pass (A) [-> z pass (B) in 3D]; the last pass stores squared modes
    double* bufA = sf;             // [el][ND]
    double* bufB = sf + EPB * ND;  // [el][ND]
    const int i0 = node % N, j0 = (node / N) % N, k0 = DIM == 3 ? node / (N * N) : 0;
    if (active) {
      const double* Ue = us + el * NV * NDP;
      if constexpr (DIM == 2)
        bufA[el * ND + node] =
            hg_node_value(Ue[pn], Ue[NDP + pn], Ue[2 * NDP + pn], Ue[3 * NDP + pn]);
      else
        bufA[el * ND + node] = hg_node_value_3d(Ue[pn], Ue[NDP + pn], Ue[2 * NDP + pn],
                                                Ue[3 * NDP + pn], Ue[4 * NDP + pn]);
    }
    __syncthreads();
    if (active) {  // x: sum_ii V(i, ii) ind(.., ii)
      double r = 0.0;
#pragma unroll
      for (int ii = 0; ii < N; ++ii)
        r = __dadd_rn(r, __dmul_rn(vinv_s[i0 * N + ii], bufA[el * ND + node - i0 + ii]));
      bufB[el * ND + node] = r;
    }
    __syncthreads();
    if (active) {  // y: sum_jj V(j, jj) tmp(.., jj, i)
      double r = 0.0;
#pragma unroll
      for (int jj = 0; jj < N; ++jj)
        r = __dadd_rn(r, __dmul_rn(vinv_s[j0 * N + jj],
                                   bufB[el * ND + node + (jj - j0) * N]));
      bufA[el * ND + node] = DIM == 2 ? __dmul_rn(r, r) : r;
    }
    __syncthreads();
    if constexpr (DIM == 3) {
      if (active) {  // z: sum_kk V(k, kk) tmp(kk, j, i)
        double r = 0.0;
#pragma unroll
        for (int kk = 0; kk < N; ++kk)
          r = __dadd_rn(r, __dmul_rn(vinv_s[k0 * N + kk],
                                     bufA[el * ND + node + (kk - k0) * N * N]));
        bufB[el * ND + node] = __dmul_rn(r, r);
      }
      __syncthreads();
    }
    double* m2 = DIM == 2 ? bufA : bufB;
    if (tid < ne) {
      double total, c1e, c2e;
      if constexpr (DIM == 2)
        hg_energy_sums<N>(m2 + tid * ND, &total, &c1e, &c2e);
      else
        hg_energy_sums_3d<N>(m2 + tid * ND, &total, &c1e, &c2e);
      const double a = hg_alpha_from_energies(total, c1e, c2e, p.hg_threshold, p.hg_s,
                                              p.alpha_min, p.alpha_max);
      alpha_s[tid] = a;
      if (p.alpha_out) p.alpha_out[e0 + tid] = a;
    }
    __syncthreads();
  }

  // ---- phase 2a: face fluxes, one task per (element, face, face node) ------
  if (worker)
    node_face_tasks<DIM, N, VF, SF, NS, NDP, NT, NQ, NI>(p, M, us, pr, wv, info, sf, ne, tid,
                                                         gamma, t_stage, c0, c1, c2);

  // ---- phase 2b: volume term, one thread per node --------------------------
  double acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q] = 0.0;
  // blocks of whole warps run the volume term on every lane (lanes past the
  // last element read element 0 and discard the result), so that the metric
  // shuffles of node_volume_direction see full warps
  constexpr bool WARP_ALL = NT % 32 == 0;
  static_assert(WARP_ALL == S::WARP_ALL, "thread count");
  // with the exchange buffer every thread takes part (its barriers)
  if (active || WARP_ALL || S::XCHG) {
    const int ev = active ? el : 0;
    const int* I = info + ev * NI;
    const double* U = us + ev * NV * NDP;
    const double* P = pr + ev * NQ * NDP;
    const NodeFluxState<DIM> own = load_flux_state<DIM, VF>(U, P, NDP, pn);
    const double hgm1 = 0.5 * p.inv_gm1;
    node_volume_direction<0, DIM, N, VF, NDP, WARP_ALL, S::XCHG>(p, M, U, P, I, node, pn, own,
                                                                hgm1, acc, xbuf, tid, NT,
                                                                worker);
    node_volume_direction<1, DIM, N, VF, NDP, WARP_ALL, S::XCHG>(p, M, U, P, I, node, pn, own,
                                                                hgm1, acc, xbuf, tid, NT,
                                                                worker);
    if constexpr (DIM == 3)
      node_volume_direction<2, DIM, N, VF, NDP, WARP_ALL, S::XCHG>(p, M, U, P, I, node, pn, own,
                                                                  hgm1, acc, xbuf, tid, NT,
                                                                  worker);
  }
  if constexpr (HG) {
    if (active) {
      const int* I = info + el * NI;
      const double* U = us + el * NV * NDP;
      const double* P = pr + el * NQ * NDP;
      // volume_flux.hpp:817-842: (1 - alpha) DG + alpha FV for troubled elements
      const double alpha = alpha_s[el];
      if (fabs(alpha - 0.0) > p.atol) {
        const double one_m = 1.0 - alpha;
#pragma unroll
        for (int q = 0; q < NV; ++q) acc[q] *= one_m;
        node_fv_direction<0, DIM, N, VF, NDP>(p, M, U, P, I, node, alpha, acc);
        node_fv_direction<1, DIM, N, VF, NDP>(p, M, U, P, I, node, alpha, acc);
        if constexpr (DIM == 3)
          node_fv_direction<2, DIM, N, VF, NDP>(p, M, U, P, I, node, alpha, acc);
      }
    }
  }
  // viscous terms after the shock-capturing blend: the blend covers the
  // inviscid volume integral only (the reference adds the parabolic terms
  // separately, structured_solver.hpp:437-480)
  if constexpr (NS) {
    if (active) {
      const int ev = el;
      const int* I = info + el * NI;
      if constexpr (NS && DIM == 3) {
        // viscous weak-form volume term sum_k Dhat(m, k) Ja^dir(k) . (-F_v)(k)
        // along each line through the node (parabolic_viscous.hpp:398-469)
        const double* W = wv + ev * 3 * NV * ND;
#pragma unroll
        for (int dir = 0; dir < 3; ++dir) {
          const int m = dir == 0 ? node % N : dir == 1 ? (node / N) % N : node / (N * N);
          const int stride = dir == 0 ? 1 : dir == 1 ? N : N * N;
          const double* j0 = M.tab.ja[dir][0] + (int64_t)I[3] * ND;
          const double* j1 = M.tab.ja[dir][1] + (int64_t)I[4] * ND;
          const double* j2 = M.tab.ja[dir][2] + (int64_t)I[5] * ND;
#pragma unroll
          for (int k = 0; k < N; ++k) {
            const int nk = node + (k - m) * stride;
            const double a0 = __ldg(j0 + nk), a1 = __ldg(j1 + nk), a2 = __ldg(j2 + nk);
            const double dmk = p.basis.Dhat[m][k];
#pragma unroll
            for (int q = 0; q < NV; ++q)
              acc[q] += dmk * (a0 * W[(0 * NV + q) * ND + nk] + a1 * W[(1 * NV + q) * ND + nk] +
                               a2 * W[(2 * NV + q) * ND + nk]);
          }
        }
      } else if constexpr (NS) {
        // viscous weak-form volume term sum_k Dhat(m, k) Ja^dir(k) . (-F_v)(k)
        // along each line through the node (parabolic_viscous.hpp:418-466)
        const double* W = wv + ev * 2 * NV * ND;
#pragma unroll
        for (int dir = 0; dir < 2; ++dir) {
          const int m = dir == 0 ? node % N : node / N;
          const int stride = dir == 0 ? 1 : N;
          const double* j0 = M.tab.ja[dir][0] + (int64_t)I[3] * ND;
          const double* j1 = M.tab.ja[dir][1] + (int64_t)I[4] * ND;
#pragma unroll
          for (int k = 0; k < N; ++k) {
            const int nk = node + (k - m) * stride;
            const double a0 = __ldg(j0 + nk), a1 = __ldg(j1 + nk);
            const double dmk = p.basis.Dhat[m][k];
#pragma unroll
            for (int q = 0; q < NV; ++q)
              acc[q] += dmk * (a0 * W[(0 * NV + q) * ND + nk] + a1 * W[(1 * NV + q) * ND + nk]);
          }
        }
      }
    }
  }
  __syncthreads();
  // the block agrees on a timeout (vote) so that all of it leaves together
  if (bulk_n && __syncthreads_or(!mbar_wait_bounded(&bar_n, 0, p.wait_limit_ns))) {
    if (tid == 0) atomicOr(p.nonfinite, 2u);
    return;
  }
  // fused diagnostics need every thread of the block for the reduction
  const bool diag = !BATCH && p.diag != nullptr;
  if (!active && !diag) return;
  double dacc[3] = {0.0, 0.0, 0.0};
  if (active) {

  // ---- phase 3: lifting (surface_integral.hpp:35-154), -1/J, SSPRK3 --------
  node_lift<DIM, N>(sf + el * NFACE * NF * NV, node, p.basis.lhat_l0, p.basis.lhat_rN, acc);
  const double mij = pr[(el * NQ + K::MIJ) * NDP + pn];
  const int64_t gbase = (int64_t)(e0 + el) * NV * ND + node;
  bool bad = false;
  double vals[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    const double du = acc[q] * mij;
    const int64_t gi = gbase + (int64_t)q * ND;
    double val = M.c * du;
    if (p.b != 0.0) val = p.b * us[(el * NV + q) * NDP + pn] + val;
    if (p.a != 0.0)
      val = p.a * (bulk_n ? stage_n[(el * NV + q) * ND + node] : M.u_n[gi]) + val;
    bad |= !isfinite(val);
    M.out[gi] = val;
    vals[q] = val;
  }
  if (bad) atomicOr(p.nonfinite, 1u);
  if (diag) diag_add_node<DIM, N>(vals, p.basis, node, -mij, gamma, p.inv_gm1, dacc);
  }  // active
  // the state tile is free after the epilogue (it holds NV * NT >= 3 * NT doubles)
  if (diag) {
    __syncthreads();
    diag_block_store<NT>(dacc, us, p.diag + 3 * (int64_t)blockIdx.x);
  }
}

template <int DIM, int N, int VF, int SF, int EPB, bool BATCH, bool HG = false, bool NS = false>
__global__ void __launch_bounds__(EPB* ipow(N, DIM)) stage_node_kernel(const StageArgs<N> p) {
  stage_node_body<DIM, N, VF, SF, EPB, BATCH, HG, NS>(p);
}

// Same kernel with MINB resident blocks per SM requested from the register
// allocator.
template <int DIM, int N, int VF, int SF, int EPB, bool BATCH, int MINB, bool HG = false,
          bool NS = false>
__global__ void __launch_bounds__(EPB* ipow(N, DIM), MINB)
    stage_node_kernel_capped(const StageArgs<N> p) {
  stage_node_body<DIM, N, VF, SF, EPB, BATCH, HG, NS>(p);
}

}  // namespace dgsem

// dgsem_b200_kernels.cuh -- header-only device path with the reference's
// OPEN template plugin surface (RetrO598/DGSEM), for translation units that
// nvcc compiles (flags: -std=c++17 or later, --expt-relaxed-constexpr for
// std::array in device code, -gencode arch=compute_100a,code=sm_100a).
//
// The library's C ABI (dgsem_b200.h) compiles a closed set of equations,
// fluxes and boundary conditions.  This header lets user code plug its own
// in, exactly as the reference's templates do:
//   * a two-point volume flux or a surface flux is any struct template
//     F<Eq> with a static device-callable
//       std::array<T, NVARS> numerical_flux(const Eq&, const std::array<T, NVARS>& uL,
//                                           const std::array<T, NVARS>& uR,
//                                           const std::array<T, NDIMS>& normal)
//     (the reference's contract, base/numerical_flux.hpp:198-258; a plugin
//     written for the reference compiles unchanged: KOKKOS_INLINE_FUNCTION
//     is defined here as __host__ __device__ when Kokkos is absent);
//   * an equation provides NDIMS, NVARS, get_gamma(), flux(u, normal),
//     flux(u, dim), get_wave_speed(uL, uR, normal) (equations/
//     compressible_euler2D.hpp:25-112): CompressibleEuler2D/3D below;
//   * boundary conditions, one per face in the reference's face order left,
//     right, bottom, top(, back, front) (boundary_condition/boundary_set.hpp:
//     174-245): PeriodicBC, DirichletBC<Func> whose Func is a device-callable
//     f(x, t) -> conserved state or a constant std::array
//     (dirichlet_boundary.hpp:70-120), OutflowBC (outflow_boundary.hpp:57-110),
//     SlipWallBC and MixedDirichletSlipWallBC<Func, Pred> (dirichlet_boundary.hpp:
//     198-275).
// The fused kernel (plugin_stage_kernel) is the library's node-parallel stage
// kernel in generic form: one thread per node, the element tile in shared
// memory, face fluxes f* once per (face, face node) into a shared buffer, the
// split-form volume term sum_k Dsplit(m, k) f(u_lo, u_hi, (Ja_m + Ja_k)/2)
// with the reference's argument order (lower node index first, as its k > i
// pair loop, volume_flux.hpp:221-410) and its per-node summation order
// (partners in ascending index, directions x, y, z), lifting, -1/J and the
// fused SSPRK3 combination a*u_n + b*u_in + c*du.  Geometry is per node
// (contravariant vectors Ja^a_c, 1/J and node coordinates, in device
// arrays), so curvilinear meshes run through it unchanged.
//
// Host side: DGSEM::plugin::StructuredSolver<Eq, Polydeg, VolumeFlux,
// SurfaceFlux, BoundarySet> builds the LinearMapping geometry of a
// structured mesh through the library (dgsem_metrics_host,
// dgsem_coordinates_host, dgsem_basis_tables_host) or takes per-node geometry
// from the caller, and offers calc_rhs / stage / step on device arrays in
// the library's layout u[e][var][node].
#ifndef DGSEM_B200_KERNELS_CUH_
#define DGSEM_B200_KERNELS_CUH_

#include <cuda_runtime.h>

#include <array>
#include <cmath>
#include <cstddef>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "dgsem_b200.h"

#ifndef KOKKOS_INLINE_FUNCTION
#define KOKKOS_INLINE_FUNCTION __host__ __device__ inline
#endif

namespace DGSEM {
namespace plugin {

constexpr int ipow(int b, int e) { return e == 0 ? 1 : b * ipow(b, e - 1); }

// read-only global load (geometry, neighbour traces, u_n)
__device__ __forceinline__ double g_load(const double* p) { return __ldg(p); }

// ---- equations -------------------------------------------------------------
// Compressible Euler in DIM dimensions with the reference's member functions
// (equations/compressible_euler2D.hpp:25-112, compressible_euler3D.hpp:26-169).
template <class T, std::size_t DIM>
struct CompressibleEuler {
  static constexpr std::size_t NDIMS = DIM, NVARS = DIM + 2;
  using value_type = T;
  T gamma = T(1.4);
  CompressibleEuler() = default;
  KOKKOS_INLINE_FUNCTION explicit CompressibleEuler(T g) : gamma(g) {}
  KOKKOS_INLINE_FUNCTION T get_gamma() const { return gamma; }
  KOKKOS_INLINE_FUNCTION T pressure(const std::array<T, NVARS>& u) const {
    T sq = T(0);
    for (std::size_t d = 0; d < DIM; ++d) sq += u[1 + d] * u[1 + d];
    return (gamma - T(1)) * (u[DIM + 1] - T(0.5) * sq / u[0]);
  }
  // physical flux along the normal: F(u) . n
  KOKKOS_INLINE_FUNCTION std::array<T, NVARS> flux(const std::array<T, NVARS>& u,
                                                   const std::array<T, NDIMS>& n) const {
    const T p = pressure(u);
    T vn = T(0);
    for (std::size_t d = 0; d < DIM; ++d) vn += u[1 + d] / u[0] * n[d];
    std::array<T, NVARS> f{};
    f[0] = u[0] * vn;
    for (std::size_t d = 0; d < DIM; ++d) f[1 + d] = u[1 + d] * vn + p * n[d];
    f[DIM + 1] = (u[DIM + 1] + p) * vn;
    return f;
  }
  KOKKOS_INLINE_FUNCTION std::array<T, NVARS> flux(const std::array<T, NVARS>& u,
                                                   std::size_t dim) const {
    std::array<T, NDIMS> n{};
    n[dim] = T(1);
    return flux(u, n);
  }
  // LLF speed max(|v_L.n|, |v_R.n|) + max(c_L, c_R) |n|
  KOKKOS_INLINE_FUNCTION T get_wave_speed(const std::array<T, NVARS>& uL,
                                          const std::array<T, NVARS>& uR,
                                          const std::array<T, NDIMS>& n) const {
    T vnL = T(0), vnR = T(0), nn = T(0);
    for (std::size_t d = 0; d < DIM; ++d) {
      vnL += uL[1 + d] / uL[0] * n[d];
      vnR += uR[1 + d] / uR[0] * n[d];
      nn += n[d] * n[d];
    }
    const T cL = sqrt(gamma * pressure(uL) / uL[0]);
    const T cR = sqrt(gamma * pressure(uR) / uR[0]);
    return fmax(fabs(vnL), fabs(vnR)) + fmax(cL, cR) * sqrt(nn);
  }
};
template <class T>
using CompressibleEuler2D = CompressibleEuler<T, 2>;
template <class T>
using CompressibleEuler3D = CompressibleEuler<T, 3>;

// ---- a built-in surface flux written against the plugin contract ---------
// Local Lax-Friedrichs: 0.5 (F_L + F_R).n - 0.5 lambda (u_R - u_L)
// (numerical_flux.hpp:198-228, numerical_flux_detail.hpp:9-21).
template <class Eq>
struct LaxFriedrichsFlux {
  using T = typename Eq::value_type;
  static constexpr std::size_t NV = Eq::NVARS, ND = Eq::NDIMS;
  KOKKOS_INLINE_FUNCTION static std::array<T, NV> numerical_flux(const Eq& eq,
                                                                 const std::array<T, NV>& uL,
                                                                 const std::array<T, NV>& uR,
                                                                 const std::array<T, ND>& n) {
    const T lam = eq.get_wave_speed(uL, uR, n);
    const auto fL = eq.flux(uL, n);
    const auto fR = eq.flux(uR, n);
    std::array<T, NV> f{};
    for (std::size_t q = 0; q < NV; ++q)
      f[q] = T(0.5) * (fL[q] + fR[q]) - T(0.5) * lam * (uR[q] - uL[q]);
    return f;
  }
};

// ---- boundary conditions ---------------------------------------------------
struct PeriodicBC {};
struct OutflowBC {};
struct SlipWallBC {};
template <class Func>
struct DirichletBC {
  Func func;
  DirichletBC() = default;
  explicit DirichletBC(Func f) : func(f) {}
};
// Dirichlet state where use_dirichlet(x, t) holds, reflecting wall elsewhere.
template <class Func, class Pred>
struct MixedDirichletSlipWallBC {
  Func func;
  Pred use_dirichlet;
  MixedDirichletSlipWallBC() = default;
  MixedDirichletSlipWallBC(Func f, Pred p) : func(f), use_dirichlet(p) {}
};

// One boundary condition per face (2D: 4, 3D: 6), in the reference's face
// order left, right, bottom, top, back, front.
template <class B0, class B1, class B2, class B3, class B4 = PeriodicBC, class B5 = PeriodicBC>
struct BoundarySetT {
  B0 b0;
  B1 b1;
  B2 b2;
  B3 b3;
  B4 b4;
  B5 b5;
  template <int F>
  KOKKOS_INLINE_FUNCTION const auto& get() const {
    if constexpr (F == 0) return b0;
    else if constexpr (F == 1) return b1;
    else if constexpr (F == 2) return b2;
    else if constexpr (F == 3) return b3;
    else if constexpr (F == 4) return b4;
    else return b5;
  }
  template <int F>
  static constexpr bool periodic_face() {
    using B = std::decay_t<decltype(std::declval<BoundarySetT>().template get<F>())>;
    return std::is_same_v<B, PeriodicBC>;
  }
};
template <class B0, class B1, class B2, class B3>
BoundarySetT<B0, B1, B2, B3> BoundarySet(B0 b0, B1 b1, B2 b2, B3 b3) {
  return {b0, b1, b2, b3, PeriodicBC{}, PeriodicBC{}};
}
template <class B0, class B1, class B2, class B3, class B4, class B5>
BoundarySetT<B0, B1, B2, B3, B4, B5> BoundarySet(B0 b0, B1 b1, B2 b2, B3 b3, B4 b4, B5 b5) {
  return {b0, b1, b2, b3, b4, b5};
}

namespace detail {

template <class B, class = void>
struct is_mixed_bc : std::false_type {};
template <class B>
struct is_mixed_bc<B, std::void_t<decltype(std::declval<const B&>().use_dirichlet)>>
    : std::true_type {};

template <class Func, class T, std::size_t NV, std::size_t ND>
__device__ inline std::array<T, NV> outer_state(const Func& f, const std::array<T, ND>& x, T t) {
  if constexpr (std::is_invocable_v<const Func&, const std::array<T, ND>&, T>) {
    return f(x, t);
  } else {
    std::array<T, NV> u{};
    for (std::size_t q = 0; q < NV; ++q) u[q] = f[q];
    return u;
  }
}

// reflecting wall state: v - 2 (v.n / |n|^2) n, density and energy kept
// (MixedDirichletSlipWallBC::reflect_state, dirichlet_boundary.hpp:207-220)
template <class T, std::size_t NV, std::size_t ND>
__device__ inline std::array<T, NV> reflect(const std::array<T, NV>& ui,
                                            const std::array<T, ND>& n) {
  T vn = T(0), nn = T(0);
  for (std::size_t d = 0; d < ND; ++d) {
    vn += ui[1 + d] / ui[0] * n[d];
    nn += n[d] * n[d];
  }
  vn = vn / nn;
  std::array<T, NV> uw = ui;
  for (std::size_t d = 0; d < ND; ++d) uw[1 + d] = ui[0] * (ui[1 + d] / ui[0] - T(2) * vn * n[d]);
  return uw;
}

}  // namespace detail

// ---- kernel arguments --------------------------------------------------------
template <int N>
struct PluginNodes {
  double xi[N];  // Lobatto-Legendre nodes on [-1, 1]
};

template <int N>
struct PluginBasis {
  double Dsplit[N][N];
  double lhat_l0;  // l_0(-1) / w_0
  double lhat_rN;  // l_N(+1) / w_N
};

// Per-node geometry in device memory (element e in the library's order
// e = ie + nx*(je + ny*ke), node = in + n*(jn + n*kn)):
//   ja[((e * DIM + a) * DIM + c) * ND + node]  contravariant vector Ja^a_c
//   inv_j[e * ND + node]                       1/J
//   x[(e * DIM + d) * ND + node]               node coordinates
struct PluginGeometry {
  const double* ja;
  const double* inv_j;
  const double* x;
  int cells[3];
  int periodic[3];
  int nelem;
};

template <class Eq, int N, class Bcs>
struct PluginArgs {
  const double* u_n;
  const double* u_in;
  double* out;
  double a, b, c;  // out = a*u_n + b*u_in + c*du
  double t;
  Eq eq;
  Bcs bcs;
  PluginGeometry geo;
  PluginBasis<N> basis;
};

template <int DIM, int N>
__device__ inline int plugin_line_node(int dir, int line, int m) {
  if (DIM == 2) return dir == 0 ? m + N * line : line + N * m;
  if (dir == 0) return m + N * line;
  if (dir == 1) return (line % N) + N * m + N * N * (line / N);
  return line + N * N * m;
}

// Flux f* of face node `fn` on face (dir, side) of element e (own tile in
// shared memory): interface flux with the neighbour's trace, or the face's
// boundary condition (boundary_set.hpp:70-86, utils/boundary_helper.hpp:56-146).
template <class Eq, int N, template <class> class SF, class Bcs, int FACE>
__device__ inline void plugin_face_flux(const PluginArgs<Eq, N, Bcs>& p, const double* U, int e,
                                        const int* ijk, int fn, double* out) {
  using T = double;
  constexpr int DIM = (int)Eq::NDIMS, NV = (int)Eq::NVARS, ND = ipow(N, DIM);
  constexpr int dir = FACE / 2, side = FACE % 2;
  const PluginGeometry& g = p.geo;
  const int own = plugin_line_node<DIM, N>(dir, fn, side ? N - 1 : 0);
  std::array<T, NV> uo;
  for (int q = 0; q < NV; ++q) uo[q] = U[q * ND + own];
  int pos = ijk[dir] + (side ? 1 : -1);
  bool inside = pos >= 0 && pos < g.cells[dir];
  if (!inside && g.periodic[dir]) {
    pos = (pos + g.cells[dir]) % g.cells[dir];
    inside = true;
  }
  std::array<T, NV> f;
  std::array<T, DIM> nrm;
  if (inside) {
    int q3[3] = {ijk[0], ijk[1], ijk[2]};
    q3[dir] = pos;
    const int en = DIM == 2 ? q3[0] + g.cells[0] * q3[1]
                            : q3[0] + g.cells[0] * (q3[1] + g.cells[1] * q3[2]);
    const int nb = plugin_line_node<DIM, N>(dir, fn, side ? 0 : N - 1);
    std::array<T, NV> ux;
    for (int q = 0; q < NV; ++q) ux[q] = g_load(p.u_in + ((long long)en * NV + q) * ND + nb);
    // the normal is Ja^dir of the high-side element at its low-face node
    const int ehi = side ? en : e;
    const int nlo = side ? nb : own;
    for (int c = 0; c < DIM; ++c)
      nrm[c] = g_load(g.ja + (((long long)ehi * DIM + dir) * DIM + c) * ND + nlo);
    f = side ? SF<Eq>::numerical_flux(p.eq, uo, ux, nrm) : SF<Eq>::numerical_flux(p.eq, ux, uo, nrm);
  } else {
    for (int c = 0; c < DIM; ++c)
      nrm[c] = g_load(g.ja + (((long long)e * DIM + dir) * DIM + c) * ND + own);
    std::array<T, DIM> x;
    for (int d = 0; d < DIM; ++d) x[d] = g_load(g.x + ((long long)e * DIM + d) * ND + own);
    const auto& bc = p.bcs.template get<FACE>();
    using B = std::decay_t<decltype(bc)>;
    std::array<T, NV> ux = uo;
    if constexpr (std::is_same_v<B, OutflowBC>) {
      // outflow_boundary.hpp:79-104: the average along the line normal to the face
      for (int q = 0; q < NV; ++q) {
        T acc = T(0);
        for (int m = 0; m < N; ++m) acc += U[q * ND + plugin_line_node<DIM, N>(dir, fn, m)];
        ux[q] = acc / T(N);
      }
    } else if constexpr (std::is_same_v<B, SlipWallBC>) {
      ux = detail::reflect<T, NV, DIM>(uo, nrm);
    } else if constexpr (std::is_same_v<B, PeriodicBC>) {
      // a periodic face is never a boundary face
    } else if constexpr (detail::is_mixed_bc<B>::value) {
      ux = bc.use_dirichlet(x, p.t) ? detail::outer_state<decltype(bc.func), T, NV, DIM>(bc.func, x, p.t)
                                    : detail::reflect<T, NV, DIM>(uo, nrm);
    } else {
      ux = detail::outer_state<decltype(bc.func), T, NV, DIM>(bc.func, x, p.t);
    }
    // the inner state is the left state on high faces (left_state_inner)
    f = side ? SF<Eq>::numerical_flux(p.eq, uo, ux, nrm) : SF<Eq>::numerical_flux(p.eq, ux, uo, nrm);
  }
  for (int q = 0; q < NV; ++q) out[q] = f[q];
}

template <class Eq, int N, template <class> class VF, template <class> class SF, class Bcs,
          int EPB>
__global__ void __launch_bounds__(EPB* ipow(N, (int)Eq::NDIMS))
    plugin_stage_kernel(const PluginArgs<Eq, N, Bcs> p) {
  using T = double;
  constexpr int DIM = (int)Eq::NDIMS, NV = (int)Eq::NVARS, ND = ipow(N, DIM);
  constexpr int NF = ipow(N, DIM - 1), NFACE = 2 * DIM, NT = EPB * ND;
  extern __shared__ __align__(16) double plugin_smem[];
  double* us = plugin_smem;             // [el][var][node]
  double* sf = us + EPB * NV * ND;      // [el][face][fn][var]
  const PluginGeometry& g = p.geo;
  const int tid = threadIdx.x;
  const int e0 = (int)blockIdx.x * EPB;
  if (e0 >= g.nelem) return;
  const int ne = min(EPB, g.nelem - e0);
  for (int i = tid; i < ne * NV * ND; i += NT) us[i] = g_load(p.u_in + (long long)e0 * NV * ND + i);
  __syncthreads();
  // face fluxes, one task per (element, face, face node)
  for (int idx = tid; idx < ne * NFACE * NF; idx += NT) {
    const int el = idx / (NFACE * NF), face = (idx / NF) % NFACE, fn = idx % NF;
    const int e = e0 + el;
    const int ijk[3] = {e % g.cells[0], DIM == 2 ? e / g.cells[0] : (e / g.cells[0]) % g.cells[1],
                        DIM == 2 ? 0 : e / (g.cells[0] * g.cells[1])};
    const double* U = us + el * NV * ND;
    double* F = sf + ((el * NFACE + face) * NF + fn) * NV;
    switch (face) {
      case 0: plugin_face_flux<Eq, N, SF, Bcs, 0>(p, U, e, ijk, fn, F); break;
      case 1: plugin_face_flux<Eq, N, SF, Bcs, 1>(p, U, e, ijk, fn, F); break;
      case 2: plugin_face_flux<Eq, N, SF, Bcs, 2>(p, U, e, ijk, fn, F); break;
      case 3: plugin_face_flux<Eq, N, SF, Bcs, 3>(p, U, e, ijk, fn, F); break;
      case 4: if constexpr (DIM == 3) plugin_face_flux<Eq, N, SF, Bcs, 4>(p, U, e, ijk, fn, F); break;
      default: if constexpr (DIM == 3) plugin_face_flux<Eq, N, SF, Bcs, 5>(p, U, e, ijk, fn, F); break;
    }
  }
  // volume term: one thread per node
  const int el = tid / ND, node = tid % ND;
  const bool active = el < ne;
  std::array<T, NV> acc{};
  if (active) {
    const int e = e0 + el;
    const double* U = us + el * NV * ND;
    std::array<T, NV> um;
    for (int q = 0; q < NV; ++q) um[q] = U[q * ND + node];
    const int pos[3] = {node % N, (node / N) % N, node / (N * N)};
    for (int dir = 0; dir < DIM; ++dir) {
      const int m = pos[dir];
      const int stride = dir == 0 ? 1 : dir == 1 ? N : N * N;
      const double* jrow = g.ja + ((long long)e * DIM + dir) * DIM * ND;
      std::array<T, DIM> jm;
      for (int c = 0; c < DIM; ++c) jm[c] = g_load(jrow + c * ND + node);
      for (int k = 0; k < N; ++k) {
        if (k == m) continue;
        const int nk = node + (k - m) * stride;
        std::array<T, NV> uk;
        for (int q = 0; q < NV; ++q) uk[q] = U[q * ND + nk];
        std::array<T, DIM> nrm;
        for (int c = 0; c < DIM; ++c) nrm[c] = T(0.5) * (jm[c] + g_load(jrow + c * ND + nk));
        // the reference's pair (i, k), i < k, evaluates f(u_i, u_k)
        const std::array<T, NV> f = k > m ? VF<Eq>::numerical_flux(p.eq, um, uk, nrm)
                                          : VF<Eq>::numerical_flux(p.eq, uk, um, nrm);
        const T dmk = p.basis.Dsplit[m][k];
        for (int q = 0; q < NV; ++q) acc[q] += dmk * f[q];
      }
    }
  }
  __syncthreads();
  if (!active) return;
  const int e = e0 + el;
  // lifting (surface_integral.hpp:35-154), -1/J (jacobian.hpp:76-101), SSPRK3
  const int pos[3] = {node % N, (node / N) % N, node / (N * N)};
  for (int dir = 0; dir < DIM; ++dir) {
    const int line = dir == 0 ? node / N : dir == 1 ? node % N + N * (node / (N * N)) : node % (N * N);
    if (pos[dir] == 0) {
      const double* F = sf + ((el * NFACE + 2 * dir) * NF + line) * NV;
      for (int q = 0; q < NV; ++q) acc[q] -= F[q] * p.basis.lhat_l0;
    }
    if (pos[dir] == N - 1) {
      const double* F = sf + ((el * NFACE + 2 * dir + 1) * NF + line) * NV;
      for (int q = 0; q < NV; ++q) acc[q] += F[q] * p.basis.lhat_rN;
    }
  }
  const double mij = -g_load(g.inv_j + (long long)e * ND + node);
  for (int q = 0; q < NV; ++q) {
    const long long gi = ((long long)e * NV + q) * ND + node;
    double val = p.c * (acc[q] * mij);
    if (p.b != 0.0) val = p.b * us[(el * NV + q) * ND + node] + val;
    if (p.a != 0.0) val = p.a * g_load(p.u_n + gi) + val;
    p.out[gi] = val;
  }
}

// Node coordinates of a structured mesh as the image of the reference square
// or cube [-1, 1]^d under a mapping (StructuredContainerInitializer::
// calc_node_coordinates, containers/data_container.hpp:196-225): element ie
// covers [-1 + ie dx, -1 + (ie + 1) dx] with dx = 2 / n_cells, node i sits at
// its centre + (dx / 2) xi_i, and x = mapping.eval(reference point).  Mapping
// is any device-callable type with std::array<double, DIM> eval(const
// std::array<double, DIM>&) const (the reference's LinearMapping interface,
// base/mapping.hpp:31-50).  One thread per node; x[(e*DIM + c)*ND + node].
template <class Mapping, int DIM, int N>
__global__ void map_nodes_kernel(Mapping map, int c0, int c1, int c2, PluginNodes<N> gll,
                                 double* x) {
  constexpr int ND = ipow(N, DIM);
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nelem = (long long)c0 * c1 * (DIM == 3 ? c2 : 1);
  if (idx >= nelem * ND) return;
  const int e = (int)(idx / ND), node = (int)(idx % ND);
  const int ev[3] = {e % c0, (e / c0) % c1, DIM == 3 ? e / (c0 * c1) : 0};
  const int iv[3] = {node % N, (node / N) % N, node / (N * N)};
  const int cells[3] = {c0, c1, c2};
  std::array<double, DIM> ref;
  for (int a = 0; a < DIM; ++a) {
    const double dx = __ddiv_rn(2.0, (double)cells[a]);
    const double off = __dadd_rn(__dadd_rn(-1.0, __dmul_rn((double)ev[a], dx)), __dmul_rn(0.5, dx));
    ref[a] = __dadd_rn(off, __dmul_rn(__dmul_rn(0.5, dx), gll.xi[iv[a]]));
  }
  const std::array<double, DIM> p = map.eval(ref);
  for (int a = 0; a < DIM; ++a) x[((long long)e * DIM + a) * ND + node] = p[a];
}

// ---- host side -----------------------------------------------------------------
namespace detail {
inline void check(dgsem_status s, const char* where) {
  if (s != DGSEM_OK) throw std::runtime_error(std::string(where) + ": " + dgsem_status_string(s));
}
inline void check_cuda(cudaError_t e, const char* where) {
  if (e != cudaSuccess)
    throw std::runtime_error(std::string(where) + ": " + cudaGetErrorString(e));
}
}  // namespace detail

// Structured mesh solver over user plugins.  VolumeFlux and SurfaceFlux are
// plugin templates F<Eq>; Bcs is a BoundarySetT.  Arrays are device arrays
// in the library's layout u[e][var][node].
template <class Eq, std::size_t Polydeg, template <class> class VolumeFlux,
          template <class> class SurfaceFlux, class Bcs>
class StructuredSolver {
 public:
  static constexpr int DIM = (int)Eq::NDIMS, NV = (int)Eq::NVARS, N = (int)Polydeg + 1;
  static constexpr int ND = ipow(N, DIM);
  static constexpr int EPB = (128 / ND) > 0 ? (128 / ND) : 1;
  static constexpr int NT = EPB * ND;
  static constexpr size_t kSmem =
      sizeof(double) * (EPB * NV * ND + EPB * 2 * DIM * ipow(N, DIM - 1) * NV);

  // LinearMapping of [left, right] with `cells` elements per direction.
  StructuredSolver(const Eq& eq, const std::array<double, DIM>& left,
                   const std::array<double, DIM>& right, const std::array<int, DIM>& cells,
                   const Bcs& bcs, cudaStream_t stream = nullptr)
      : eq_(eq), bcs_(bcs), stream_(stream) {
    set_mesh(cells);
    dgsem_mesh_desc m{};
    m.ndims = DIM;
    m.polydeg = (int)Polydeg;
    for (int a = 0; a < 3; ++a) {
      m.n_cells[a] = a < DIM ? cells[a] : 1;
      m.domain_left[a] = a < DIM ? left[a] : 0.0;
      m.domain_right[a] = a < DIM ? right[a] : 1.0;
    }
    const size_t E = (size_t)nelem_;
    std::vector<double> ja_ref(E * ND * DIM * DIM), ij_ref(E * ND), x_ref(E * ND * DIM);
    detail::check(dgsem_metrics_host(&m, ja_ref.data(), ij_ref.data()), "dgsem_metrics_host");
    detail::check(dgsem_coordinates_host(&m, x_ref.data()), "dgsem_coordinates_host");
    // reference logical order (i slowest ... , dof, a, c) -> device order
    std::vector<double> ja(E * DIM * DIM * ND), ij(E * ND), x(E * DIM * ND);
    for (size_t e = 0; e < E; ++e) {
      const size_t ie = e % cells_[0], je = (e / cells_[0]) % cells_[1],
                   ke = DIM == 2 ? 0 : e / ((size_t)cells_[0] * cells_[1]);
      const size_t er = DIM == 2 ? ie * cells_[1] + je : (ie * cells_[1] + je) * cells_[2] + ke;
      for (int node = 0; node < ND; ++node) {
        ij[e * ND + node] = ij_ref[er * ND + node];
        for (int a = 0; a < DIM; ++a) {
          x[(e * DIM + a) * ND + node] = x_ref[(er * ND + node) * DIM + a];
          for (int c = 0; c < DIM; ++c)
            ja[((e * DIM + a) * DIM + c) * ND + node] = ja_ref[((er * ND + node) * DIM + a) * DIM + c];
        }
      }
    }
    upload_geometry(ja.data(), ij.data(), x.data());
  }

  // Geometry given per node by the caller (any mapping, e.g. curvilinear):
  // ja[((e*DIM + a)*DIM + c)*ND + node], inv_j[e*ND + node],
  // x[(e*DIM + d)*ND + node], DEVICE arrays, copied.
  StructuredSolver(const Eq& eq, const std::array<int, DIM>& cells, const double* ja_dev,
                   const double* inv_j_dev, const double* x_dev, const Bcs& bcs,
                   cudaStream_t stream = nullptr)
      : eq_(eq), bcs_(bcs), stream_(stream) {
    set_mesh(cells);
    alloc_geometry();
    const size_t E = (size_t)nelem_;
    detail::check_cuda(cudaMemcpy(ja_, ja_dev, E * DIM * DIM * ND * sizeof(double),
                                  cudaMemcpyDeviceToDevice), "cudaMemcpy");
    detail::check_cuda(cudaMemcpy(inv_j_, inv_j_dev, E * ND * sizeof(double),
                                  cudaMemcpyDeviceToDevice), "cudaMemcpy");
    detail::check_cuda(cudaMemcpy(x_, x_dev, E * DIM * ND * sizeof(double),
                                  cudaMemcpyDeviceToDevice), "cudaMemcpy");
  }

  // Any mapping of the reference square / cube (map_nodes_kernel): node
  // coordinates and per-node metrics are computed on the device
  // (dgsem_geometry_from_coordinates, the reference's metric formulas).
  template <class Mapping>
  StructuredSolver(const Eq& eq, const Mapping& map, const std::array<int, DIM>& cells,
                   const Bcs& bcs, cudaStream_t stream = nullptr)
      : eq_(eq), bcs_(bcs), stream_(stream) {
    set_mesh(cells);
    alloc_geometry();
    std::vector<double> tab(5 * N + 4 * N * N);
    detail::check(dgsem_basis_tables_host((int)Polydeg, tab.data()), "dgsem_basis_tables_host");
    PluginNodes<N> gll;
    for (int i = 0; i < N; ++i) gll.xi[i] = tab[i];
    const long long total = (long long)nelem_ * ND;
    map_nodes_kernel<Mapping, DIM, N><<<(unsigned)((total + 127) / 128), 128, 0, stream_>>>(
        map, cells_[0], cells_[1], cells_[2], gll, x_);
    detail::check_cuda(cudaGetLastError(), "map_nodes_kernel");
    const int64_t c64[3] = {cells_[0], cells_[1], cells_[2]};
    detail::check(dgsem_geometry_from_coordinates(DIM, (int)Polydeg, c64, x_, ja_, inv_j_,
                                                  stream_),
                  "dgsem_geometry_from_coordinates");
    detail::check_cuda(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
  }

  // device geometry (ja, inv_j, x) in the layout of PluginGeometry
  const double* geometry_ja() const { return ja_; }
  const double* geometry_inv_j() const { return inv_j_; }
  const double* geometry_x() const { return x_; }

  StructuredSolver(const StructuredSolver&) = delete;
  StructuredSolver& operator=(const StructuredSolver&) = delete;
  ~StructuredSolver() {
    for (double* q : {ja_, inv_j_, x_, tmp1_, tmp2_})
      if (q) cudaFree(q);
  }

  int64_t state_len() const { return (int64_t)nelem_ * NV * ND; }

  // out = a*u_n + b*u_in + c*RHS(u_in, t)
  void launch(const double* u_n, const double* u_in, double* out, double a, double b, double c,
              double t) {
    PluginArgs<Eq, N, Bcs> args;
    args.u_n = u_n;
    args.u_in = u_in;
    args.out = out;
    args.a = a;
    args.b = b;
    args.c = c;
    args.t = t;
    args.eq = eq_;
    args.bcs = bcs_;
    args.geo = geo_;
    args.basis = basis_;
    auto k = plugin_stage_kernel<Eq, N, VolumeFlux, SurfaceFlux, Bcs, EPB>;
    detail::check_cuda(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)kSmem), "cudaFuncSetAttribute");
    const unsigned blocks = (unsigned)((nelem_ + EPB - 1) / EPB);
    k<<<blocks, NT, kSmem, stream_>>>(args);
    detail::check_cuda(cudaGetLastError(), "plugin_stage_kernel");
  }

  // du = RHS(u, t) (StructuredSolver::calc_rhs, structured_solver.hpp:466-480)
  void calc_rhs(const double* u, double* du, double t) { launch(nullptr, u, du, 0.0, 0.0, 1.0, t); }

  // SSPRK3 stage 1..3 (SSPRK3.hpp:159-181)
  void stage(int s, const double* u_n, const double* u_in, double* out, double t, double dt) {
    if (s == 1) launch(nullptr, u_in, out, 0.0, 1.0, dt, t);
    else if (s == 2) launch(u_n, u_in, out, 0.75, 0.25, 0.25 * dt, t + dt);
    else launch(u_n, u_in, out, 1.0 / 3.0, 2.0 / 3.0, (2.0 / 3.0) * dt, t + 0.5 * dt);
  }

  // one SSPRK3 step in place
  void step(double* u, double t, double dt) {
    if (!tmp1_) {
      detail::check_cuda(cudaMalloc(&tmp1_, state_len() * sizeof(double)), "cudaMalloc");
      detail::check_cuda(cudaMalloc(&tmp2_, state_len() * sizeof(double)), "cudaMalloc");
    }
    stage(1, nullptr, u, tmp1_, t, dt);
    stage(2, u, tmp1_, tmp2_, t, dt);
    stage(3, u, tmp2_, u, t, dt);
  }

  cudaStream_t stream() const { return stream_; }

 private:
  void set_mesh(const std::array<int, DIM>& cells) {
    nelem_ = 1;
    for (int a = 0; a < 3; ++a) {
      cells_[a] = a < DIM ? cells[a] : 1;
      nelem_ *= cells_[a];
    }
    geo_.cells[0] = cells_[0];
    geo_.cells[1] = cells_[1];
    geo_.cells[2] = cells_[2];
    geo_.periodic[0] = Bcs::template periodic_face<0>() && Bcs::template periodic_face<1>();
    geo_.periodic[1] = Bcs::template periodic_face<2>() && Bcs::template periodic_face<3>();
    geo_.periodic[2] = DIM == 2 || (Bcs::template periodic_face<4>() && Bcs::template periodic_face<5>());
    geo_.nelem = nelem_;
    std::vector<double> tab(5 * N + 4 * N * N);
    detail::check(dgsem_basis_tables_host((int)Polydeg, tab.data()), "dgsem_basis_tables_host");
    // layout: nodes, weights, inv_weights, lhat(-1), lhat(+1), D, Dsplit, Dhat, Vinv
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j) basis_.Dsplit[i][j] = tab[5 * N + N * N + i * N + j];
    basis_.lhat_l0 = tab[3 * N + 0];
    basis_.lhat_rN = tab[4 * N + N - 1];
  }
  void alloc_geometry() {
    const size_t E = (size_t)nelem_;
    detail::check_cuda(cudaMalloc(&ja_, E * DIM * DIM * ND * sizeof(double)), "cudaMalloc");
    detail::check_cuda(cudaMalloc(&inv_j_, E * ND * sizeof(double)), "cudaMalloc");
    detail::check_cuda(cudaMalloc(&x_, E * DIM * ND * sizeof(double)), "cudaMalloc");
    geo_.ja = ja_;
    geo_.inv_j = inv_j_;
    geo_.x = x_;
  }
  void upload_geometry(const double* ja, const double* ij, const double* x) {
    alloc_geometry();
    const size_t E = (size_t)nelem_;
    detail::check_cuda(cudaMemcpy(ja_, ja, E * DIM * DIM * ND * sizeof(double),
                                  cudaMemcpyHostToDevice), "cudaMemcpy");
    detail::check_cuda(cudaMemcpy(inv_j_, ij, E * ND * sizeof(double), cudaMemcpyHostToDevice),
                       "cudaMemcpy");
    detail::check_cuda(cudaMemcpy(x_, x, E * DIM * ND * sizeof(double), cudaMemcpyHostToDevice),
                       "cudaMemcpy");
  }

  Eq eq_;
  Bcs bcs_;
  cudaStream_t stream_;
  int cells_[3] = {1, 1, 1};
  int nelem_ = 0;
  PluginGeometry geo_{};
  PluginBasis<N> basis_{};
  double *ja_ = nullptr, *inv_j_ = nullptr, *x_ = nullptr, *tmp1_ = nullptr, *tmp2_ = nullptr;
};

}  // namespace plugin
}  // namespace DGSEM

#endif  // DGSEM_B200_KERNELS_CUH_

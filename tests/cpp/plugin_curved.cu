// A user translation unit that runs the library's fused stage kernel on a
// curvilinear mesh through include/dgsem_b200_kernels.cuh: its own mapping
// of the reference square (the reference's Mapping interface, eval(xi),
// base/mapping.hpp:31-50) and its own central two-point flux (the
// reference's CentralFlux contract, base/numerical_flux.hpp:230-258); node
// coordinates and metrics are computed on the device.  Built by
// tests/test_geometry_curved.py into a shared object with C entry points.
#include <array>
#include <cmath>
#include <cstdint>
#include <memory>

#include "dgsem_b200_kernels.cuh"

namespace user {

// linear map onto [left, right] plus a displacement that vanishes on the
// boundary (the mesh stays periodic)
struct BumpMapping {
  std::array<double, 2> left, right;
  double amp = 0.05;
  KOKKOS_INLINE_FUNCTION std::array<double, 2> eval(const std::array<double, 2>& xi) const {
    const double pi = 3.14159265358979323846;
    std::array<double, 2> x;
    double bump = 1.0;
    for (int a = 0; a < 2; ++a) bump *= sin(pi * xi[a]);
    for (int a = 0; a < 2; ++a) {
      const double lin = 0.5 * ((1.0 - xi[a]) * left[a] + (1.0 + xi[a]) * right[a]);
      x[a] = lin + amp * (right[a] - left[a]) * bump * (a == 0 ? 1.0 : -0.5);
    }
    return x;
  }
};

template <class Equations>
struct CentralFlux {
  using T = typename Equations::value_type;
  static constexpr std::size_t NV = Equations::NVARS, ND = Equations::NDIMS;
  KOKKOS_INLINE_FUNCTION static std::array<T, NV> numerical_flux(
      const Equations& eq, const std::array<T, NV>& uL, const std::array<T, NV>& uR,
      const std::array<T, ND>& normal) {
    const auto fL = eq.flux(uL, normal);
    const auto fR = eq.flux(uR, normal);
    std::array<T, NV> f{};
    for (std::size_t q = 0; q < NV; ++q) f[q] = T(0.5) * (fL[q] + fR[q]);
    return f;
  }
};

}  // namespace user

namespace P = DGSEM::plugin;
using Eq = P::CompressibleEuler2D<double>;
using Bcs = P::BoundarySetT<P::PeriodicBC, P::PeriodicBC, P::PeriodicBC, P::PeriodicBC>;
using Solver = P::StructuredSolver<Eq, 3, user::CentralFlux, P::LaxFriedrichsFlux, Bcs>;

static std::unique_ptr<Solver> g_solver;
static int g_nelem = 0;

extern "C" int curved_create(int nx, int ny, double x0, double y0, double x1, double y1) {
  try {
    user::BumpMapping map{{x0, y0}, {x1, y1}, 0.05};
    P::PeriodicBC p;
    g_solver = std::make_unique<Solver>(Eq(1.4), map, std::array<int, 2>{nx, ny},
                                        P::BoundarySet(p, p, p, p));
    g_nelem = nx * ny;
    return 0;
  } catch (...) {
    return 1;
  }
}

// The same solver from given node coordinates (DEVICE array x[e][2][16]):
// metrics by the library's device geometry initializer.
extern "C" int curved_create_from_coordinates(int nx, int ny, const double* x) {
  try {
    const size_t E = (size_t)nx * ny, nd = 16;
    double *ja = nullptr, *ij = nullptr;
    if (cudaMalloc(&ja, E * 4 * nd * sizeof(double)) != cudaSuccess) return 1;
    if (cudaMalloc(&ij, E * nd * sizeof(double)) != cudaSuccess) return 1;
    const int64_t cells[3] = {nx, ny, 1};
    if (dgsem_geometry_from_coordinates(2, 3, cells, x, ja, ij, nullptr) != DGSEM_OK) return 1;
    P::PeriodicBC p;
    g_solver = std::make_unique<Solver>(Eq(1.4), std::array<int, 2>{nx, ny}, ja, ij, x,
                                        P::BoundarySet(p, p, p, p));
    cudaFree(ja);
    cudaFree(ij);
    g_nelem = nx * ny;
    return 0;
  } catch (...) {
    return 1;
  }
}

// du = RHS(u, t) on DEVICE arrays (library layout)
extern "C" int curved_rhs(const double* u, double* du, double t) {
  try {
    g_solver->calc_rhs(u, du, t);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
  } catch (...) {
    return 1;
  }
}

// copies the device geometry into DEVICE arrays x (E*2*16), ja (E*4*16), inv_j (E*16)
extern "C" int curved_geometry(double* x, double* ja, double* inv_j) {
  const size_t nd = 16, E = (size_t)g_nelem;
  cudaMemcpy(x, g_solver->geometry_x(), E * 2 * nd * sizeof(double), cudaMemcpyDeviceToDevice);
  cudaMemcpy(ja, g_solver->geometry_ja(), E * 4 * nd * sizeof(double), cudaMemcpyDeviceToDevice);
  cudaMemcpy(inv_j, g_solver->geometry_inv_j(), E * nd * sizeof(double), cudaMemcpyDeviceToDevice);
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

extern "C" void curved_destroy() { g_solver.reset(); }

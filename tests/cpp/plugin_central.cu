// A user translation unit outside the library: it plugs its own two-point
// volume flux and its own Dirichlet boundary function into the library's
// fused stage kernel through include/dgsem_b200_kernels.cuh, written only
// against the reference's plugin contract (base/numerical_flux.hpp:230-258
// for the central flux, boundary_condition/dirichlet_boundary.hpp:70-120 for
// DirichletBC<Func>).  Built by tests/test_plugin_surface.py into a shared
// object with C entry points for ctypes.
#include <array>
#include <cmath>
#include <cstdint>
#include <memory>

#include "dgsem_b200_kernels.cuh"

namespace user {

// central two-point flux 0.5 (F(u_L) + F(u_R)) . n, through the equation's
// physical flux, as a plugin for the reference's VolumeIntegralSplitForm
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

// time-dependent Dirichlet state f(x, t): a density and pressure wave
// travelling through a uniform flow, in conserved variables (gamma = 1.4)
struct TravellingWave {
  KOKKOS_INLINE_FUNCTION std::array<double, 4> operator()(const std::array<double, 2>& x,
                                                          double t) const {
    const double pi = 3.14159265358979323846;
    const double rho = 1.0 + 0.2 * sin(pi * (x[0] + x[1] - 0.4 * t));
    const double u = 0.3, v = -0.2;
    const double p = 1.0 + 0.1 * cos(pi * (x[0] - x[1]));
    return {rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)};
  }
};

}  // namespace user

namespace P = DGSEM::plugin;
using Eq = P::CompressibleEuler2D<double>;
using Bc = P::DirichletBC<user::TravellingWave>;
using Bcs = P::BoundarySetT<Bc, Bc, Bc, Bc>;
using Solver = P::StructuredSolver<Eq, 3, user::CentralFlux, P::LaxFriedrichsFlux, Bcs>;

static std::unique_ptr<Solver> g_solver;

extern "C" int plugin_create(int nx, int ny, double x0, double y0, double x1, double y1) {
  try {
    Bc bc{user::TravellingWave{}};
    g_solver = std::make_unique<Solver>(Eq(1.4), std::array<double, 2>{x0, y0},
                                        std::array<double, 2>{x1, y1}, std::array<int, 2>{nx, ny},
                                        P::BoundarySet(bc, bc, bc, bc));
    return 0;
  } catch (...) {
    return 1;
  }
}

extern "C" int64_t plugin_state_len() { return g_solver ? g_solver->state_len() : -1; }

// du = RHS(u, t); u and du are DEVICE arrays in the library layout
extern "C" int plugin_rhs(const double* u, double* du, double t) {
  try {
    g_solver->calc_rhs(u, du, t);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
  } catch (...) {
    return 1;
  }
}

// nsteps SSPRK3 steps in place on a DEVICE array
extern "C" int plugin_steps(double* u, double t0, double dt, int nsteps) {
  try {
    for (int s = 0; s < nsteps; ++s) g_solver->step(u, t0 + s * dt, dt);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
  } catch (...) {
    return 1;
  }
}

extern "C" void plugin_destroy() { g_solver.reset(); }

// dgsem_b200.hpp -- header-only C++ facade over the C ABI (dgsem_b200.h)
// with the reference's type names and call signatures (RetrO598/DGSEM
// src/), so code written against the reference's solver surface compiles
// against this library with an include-path change:
//
//   DGSEM::StructuredSolver<Eq, Basis, VolumeIntegral, SurfaceFlux, Mesh, BCs>
//     (eq, mesh, container, boundaries[, periodic])   structured_solver.hpp:36-58
//     ::calc_rhs(Solution&, T)                        structured_solver.hpp:466-480
//     ::initialize(const AbstractInitial&, Solution&) structured_solver.hpp:100-116
//     ::set_indicator_parameters(amax, amin, smooth)  structured_solver.hpp:118-123
//     ::get_ndofs()                                   structured_solver.hpp:125
//   DGSEM::Solution<Mesh, Basis, Eq>                  solution_container.hpp:157-234
//   DGSEM::SSPRK3<T, Solver, Mesh, Solution>          SSPRK3.hpp:145-187
//     ::step / ::solve / ::add_observer / ::get_time  integrator_base.hpp:15-47
//   plugins: equations::CompressibleEuler2D/3D, CompressibleNavierStokes2D/3D;
//     ChandrashekarFlux (+ RanochaFlux, KennedyGruberFlux), LaxFriedrichsFlux,
//     HLLCFlux (2D); VolumeIntegralSplitForm, VolumeIntegralShockCapturingHG
//     with HGIndicator; PeriodicBC, OutflowBC, SlipWallBC, DirichletBC,
//     MixedDirichletSlipWallBC, BoundarySet.
//
// Differences a caller sees:
//   * the plugin structs are tags: the fluxes are compiled into the library
//     (one instantiation per supported combination); an unsupported
//     combination throws from the solver constructor;
//   * user initial conditions (AbstractInitial subclasses with
//     operator()(std::array<T, NDIMS>)) are evaluated on the host at the
//     node coordinates and uploaded once;
//   * Solution holds device arrays (state(), rhs() return device pointers);
//     to_host() copies the state to the host in the reference's logical
//     layout u(i, j[, k], dof, var);
//   * errors throw DGSEM::Error (the reference has no runtime error path).
// Geometry is built by the library; StructuredElementContainer /
// StructuredElementInitializer / LinearMapping / KokkosSession / BasisGuard
// exist so that reference-style code compiles, and do nothing.
#ifndef DGSEM_B200_HPP_
#define DGSEM_B200_HPP_

#include <cuda_runtime.h>

#include <array>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "dgsem_b200.h"

namespace DGSEM {

class Error : public std::runtime_error {
 public:
  Error(const std::string& where, dgsem_status s)
      : std::runtime_error(where + ": " + dgsem_status_string(s)), status(s) {}
  dgsem_status status;
};

namespace detail {
inline void check(dgsem_status s, const char* where) {
  if (s != DGSEM_OK) throw Error(where, s);
}
inline void check_cuda(cudaError_t e, const char* where) {
  if (e != cudaSuccess) throw Error(std::string(where) + " (" + cudaGetErrorString(e) + ")",
                                    DGSEM_ERR_CUDA);
}

// Owning device array of doubles.
class DeviceArray {
 public:
  DeviceArray() = default;
  explicit DeviceArray(std::size_t n) : n_(n) {
    check_cuda(cudaMalloc(reinterpret_cast<void**>(&p_), n * sizeof(double)), "cudaMalloc");
    check_cuda(cudaMemset(p_, 0, n * sizeof(double)), "cudaMemset");
  }
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  DeviceArray(DeviceArray&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
  DeviceArray& operator=(DeviceArray&& o) noexcept {
    std::swap(p_, o.p_);
    std::swap(n_, o.n_);
    return *this;
  }
  ~DeviceArray() {
    if (p_) cudaFree(p_);
  }
  double* data() const { return p_; }
  std::size_t size() const { return n_; }

 private:
  double* p_ = nullptr;
  std::size_t n_ = 0;
};
}  // namespace detail

// ---- runtime guards (the reference's Kokkos session and basis tables) -----
struct KokkosSession {
  KokkosSession() = default;
  KokkosSession(int, char**) {}
};
template <class Basis>
struct BasisGuard {
  BasisGuard() { Basis::initialize(); }
  ~BasisGuard() { Basis::finalize(); }
};

// ---- equations (equations/*.hpp) --------------------------------------------
namespace equations {
template <class T>
struct CompressibleEuler2D {
  static constexpr std::size_t NDIMS = 2, NVARS = 4;
  static constexpr int dgsem_code = DGSEM_EULER_2D;
  T gamma = T(1.4);
  T get_gamma() const { return gamma; }
  T viscosity() const { return T(0); }
  T prandtl_number() const { return T(0.72); }
};
template <class T>
struct CompressibleEuler3D {
  static constexpr std::size_t NDIMS = 3, NVARS = 5;
  static constexpr int dgsem_code = DGSEM_EULER_3D;
  T gamma = T(1.4);
  T get_gamma() const { return gamma; }
  T viscosity() const { return T(0); }
  T prandtl_number() const { return T(0.72); }
};
template <class T>
struct CompressibleNavierStokes2D {
  static constexpr std::size_t NDIMS = 2, NVARS = 4;
  static constexpr int dgsem_code = DGSEM_NAVIER_STOKES_2D;
  T gamma = T(1.4);
  T mu = T(0);
  T prandtl = T(0.72);
  T get_gamma() const { return gamma; }
  T viscosity() const { return mu; }
  T prandtl_number() const { return prandtl; }
};
// equations/compressible_navier_stokes3D.hpp (periodic boxes)
template <class T>
struct CompressibleNavierStokes3D {
  static constexpr std::size_t NDIMS = 3, NVARS = 5;
  static constexpr int dgsem_code = DGSEM_NAVIER_STOKES_3D;
  T gamma = T(1.4);
  T mu = T(6.25e-4);
  T prandtl = T(0.72);
  T get_gamma() const { return gamma; }
  T viscosity() const { return mu; }
  T prandtl_number() const { return prandtl; }
};
}  // namespace equations

// ---- basis (polynomial_basis/basis.hpp) -------------------------------------
namespace Basis {
template <class T, std::size_t Polydeg>
struct LobattoLegendreBasis {
  using value_type = T;
  static constexpr std::size_t polydeg = Polydeg;
  static constexpr std::size_t NNodes = Polydeg + 1;
  static void initialize() {}
  static void finalize() {}
};
}  // namespace Basis

// ---- numerical fluxes (base/numerical_flux.hpp) -----------------------------
template <class Eq>
struct ChandrashekarFlux {
  static constexpr int dgsem_code = DGSEM_VF_CHANDRASHEKAR;
};
template <class Eq>
struct RanochaFlux {
  static constexpr int dgsem_code = DGSEM_VF_RANOCHA;
};
template <class Eq>
struct KennedyGruberFlux {
  static constexpr int dgsem_code = DGSEM_VF_KENNEDY_GRUBER;
};
template <class Eq>
struct LaxFriedrichsFlux {
  static constexpr int dgsem_code = DGSEM_SF_LAX_FRIEDRICHS;
};
template <class Eq>
struct HLLCFlux {
  static constexpr int dgsem_code = DGSEM_SF_HLLC;
};

// ---- volume integrals (space_integral/volume_flux.hpp) ----------------------
template <class Basis, class Eq>
struct HGIndicator {};

template <class Basis, class Eq, template <class> class VolumeFlux>
struct VolumeIntegralSplitForm {
  static constexpr int dgsem_code = DGSEM_VI_SPLIT_FORM;
  static constexpr int volume_flux = VolumeFlux<Eq>::dgsem_code;
};

template <class Basis, class Eq, template <class> class VolumeFlux,
          template <class> class FvFlux, class Indicator>
struct VolumeIntegralShockCapturingHG {
  static_assert(FvFlux<Eq>::dgsem_code == DGSEM_SF_LAX_FRIEDRICHS,
                "the FV subcell flux is LaxFriedrichsFlux (volume_flux.hpp:449-511)");
  static constexpr int dgsem_code = DGSEM_VI_SHOCK_CAPTURING_HG;
  static constexpr int volume_flux = VolumeFlux<Eq>::dgsem_code;
};

// ---- boundary conditions (boundary_condition/*.hpp) ------------------------
struct PeriodicBC {
  static constexpr int dgsem_kind = DGSEM_BC_PERIODIC;
};
struct OutflowBC {
  static constexpr int dgsem_kind = DGSEM_BC_OUTFLOW;
};
struct SlipWallBC {
  static constexpr int dgsem_kind = DGSEM_BC_SLIP_WALL;
};
// Outer state functors a DirichletBC can carry.
struct DoubleMachReflectionState {
  static constexpr int dgsem_kind = DGSEM_BC_DIRICHLET_DMR;
};
template <class T, std::size_t NVARS>
struct ConstantState {
  static constexpr int dgsem_kind = DGSEM_BC_DIRICHLET_CONST;
  std::array<T, NVARS> u{};
};
template <class Func>
struct DirichletBC {
  static constexpr int dgsem_kind = Func::dgsem_kind;
  Func func{};
  DirichletBC() = default;
  explicit DirichletBC(Func f) : func(f) {}
};
// MixedDirichletSlipWallBC with the double-Mach inflow state for x < 1/6 and
// a reflecting wall elsewhere (dirichlet_boundary.hpp:198-275).
template <class Func = DoubleMachReflectionState>
struct MixedDirichletSlipWallBC {
  static_assert(Func::dgsem_kind == DGSEM_BC_DIRICHLET_DMR,
                "the mixed wall is provided with the double-Mach inflow state");
  static constexpr int dgsem_kind = DGSEM_BC_MIXED_DMR_WALL;
};

template <std::size_t NFACES>
struct BoundarySetT {
  static constexpr std::size_t NFaces = NFACES;
  std::array<int, 6> kinds{};
  std::array<double, 4> state{};
};

namespace detail {
template <class B>
void bc_state(const B&, std::array<double, 4>&) {}
template <class T, std::size_t NV>
void bc_state(const DirichletBC<ConstantState<T, NV>>& b, std::array<double, 4>& s) {
  for (std::size_t q = 0; q < NV && q < 4; ++q) s[q] = static_cast<double>(b.func.u[q]);
}
}  // namespace detail

// BoundarySet(bc_left, bc_right, bc_bottom, bc_top[, bc_back, bc_front])
// (boundary_set.hpp, face order of doc/getting_started.md:42-47).
template <class... Bcs>
BoundarySetT<sizeof...(Bcs)> BoundarySet(const Bcs&... bcs) {
  static_assert(sizeof...(Bcs) == 4 || sizeof...(Bcs) == 6, "one BC per face (2D: 4, 3D: 6)");
  BoundarySetT<sizeof...(Bcs)> out;
  int f = 0;
  ((out.kinds[f++] = Bcs::dgsem_kind), ...);
  (detail::bc_state(bcs, out.state), ...);
  return out;
}

// ---- mesh and geometry (mesh/structured_mesh.hpp, containers/) -------------
template <class T, std::size_t D>
class StructuredMesh {
 public:
  StructuredMesh(const std::array<T, D>& left, const std::array<T, D>& right,
                 const std::array<std::size_t, D>& n_cells)
      : left_(left), right_(right), n_cells_(n_cells) {}
  std::size_t get_num_cells() const {
    std::size_t n = 1;
    for (auto c : n_cells_) n *= c;
    return n;
  }
  const std::array<T, D>& domain_left() const { return left_; }
  const std::array<T, D>& domain_right() const { return right_; }
  const std::array<std::size_t, D>& cells() const { return n_cells_; }

 private:
  std::array<T, D> left_, right_;
  std::array<std::size_t, D> n_cells_;
};

template <class T, std::size_t D>
struct StructuredElementContainer {};
template <class P>
struct LinearMapping {
  LinearMapping(const P&, const P&) {}
};
template <class T, class Basis, class Mapping, std::size_t D>
struct StructuredElementInitializer {
  StructuredElementInitializer(const Mapping&, const std::array<bool, D>&) {}
  template <class Container>
  void init_elements(const std::array<std::size_t, D>&, Container&) {}
};

// CRTP base of user initial conditions: Derived::operator()(std::array<T,
// NDIMS>) returns the conserved state std::array<T, NVARS>
// (boundary_condition/initial_functor.hpp:11-121).
template <class Derived, class Eq>
struct AbstractInitial {};

namespace utils {
// prim_to_cons (utils/state_conversion.hpp:9-24)
template <class T, std::size_t NV>
std::array<T, NV> prim_to_cons(const std::array<T, NV>& prim, T gamma) {
  std::array<T, NV> c{};
  c[0] = prim[0];
  T vsq = T(0);
  for (std::size_t d = 0; d + 2 < NV; ++d) {
    c[1 + d] = prim[0] * prim[1 + d];
    vsq = vsq + prim[1 + d] * prim[1 + d];
  }
  c[NV - 1] = prim[NV - 1] / (gamma - T(1)) + T(0.5) * prim[0] * vsq;
  return c;
}
}  // namespace utils

// ---- solution (containers/solution_container.hpp) ---------------------------
template <class Mesh, class Basis, class Eq>
class Solution {
 public:
  using value_type = typename Basis::value_type;
  static constexpr std::size_t NDIMS = Eq::NDIMS, NVARS = Eq::NVARS;

  explicit Solution(const Mesh& mesh)
      : mesh_(&mesh),
        n_(mesh.get_num_cells() * ipow(Basis::NNodes, NDIMS) * NVARS),
        u_(n_),
        du_(n_) {}

  double* state() const { return u_.data(); }
  double* rhs() const { return du_.data(); }
  std::size_t size() const { return n_; }
  Solution clone_shape() const { return Solution(*mesh_); }

 private:
  static constexpr std::size_t ipow(std::size_t b, std::size_t e) {
    return e == 0 ? 1 : b * ipow(b, e - 1);
  }
  const Mesh* mesh_;
  std::size_t n_;
  detail::DeviceArray u_, du_;
};

// ---- solver (solver/structured_solver.hpp) ----------------------------------
template <class Eq, class Basis, class VolumeIntegral, class SurfaceFlux, class Mesh,
          class BoundarySetType>
class StructuredSolver {
 public:
  using EquationType = Eq;
  using value_type = typename Basis::value_type;
  static constexpr std::size_t NDIMS = Eq::NDIMS;

  template <class Container>
  StructuredSolver(const Eq& eq, const Mesh& mesh, const Container&,
                   const BoundarySetType& bcs, cudaStream_t stream = nullptr)
      : StructuredSolver(eq, mesh, bcs, stream) {}

  template <class Container>
  StructuredSolver(const Eq& eq, const Mesh& mesh, Container&, const BoundarySetType& bcs,
                   const std::array<bool, NDIMS>&, cudaStream_t stream = nullptr)
      : StructuredSolver(eq, mesh, bcs, stream) {}

  StructuredSolver(const StructuredSolver&) = delete;
  StructuredSolver& operator=(const StructuredSolver&) = delete;
  ~StructuredSolver() {
    if (ctx_) dgsem_ctx_destroy(ctx_);
  }

  void calc_rhs(Solution<Mesh, Basis, Eq>& sol, value_type time) {
    detail::check(dgsem_rhs(ctx_, sol.state(), sol.rhs(), static_cast<double>(time)),
                  "dgsem_rhs");
  }

  template <class Initial>
  void initialize(const Initial& initial, Solution<Mesh, Basis, Eq>& sol) {
    const std::size_t nd = dofs_per_element_;
    std::vector<double> coords(mesh_.get_num_cells() * nd * NDIMS);
    detail::check(dgsem_coordinates_host(&mdesc_, coords.data()), "dgsem_coordinates_host");
    std::vector<double> u(sol.size());
    for (std::size_t k = 0; k < mesh_.get_num_cells() * nd; ++k) {
      std::array<value_type, NDIMS> x;
      for (std::size_t a = 0; a < NDIMS; ++a) x[a] = static_cast<value_type>(coords[k * NDIMS + a]);
      const auto s = initial(x);
      for (std::size_t q = 0; q < Eq::NVARS; ++q) u[k * Eq::NVARS + q] = static_cast<double>(s[q]);
    }
    detail::DeviceArray tmp(u.size());
    detail::check_cuda(cudaMemcpy(tmp.data(), u.data(), u.size() * sizeof(double),
                                  cudaMemcpyHostToDevice),
                       "cudaMemcpy");
    detail::check(dgsem_from_reference_layout(ctx_, tmp.data(), sol.state()),
                  "dgsem_from_reference_layout");
    detail::check_cuda(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
  }

  void set_indicator_parameters(value_type alpha_max, value_type alpha_min, bool smooth) {
    detail::check(dgsem_set_indicator_parameters(ctx_, alpha_max, alpha_min, smooth ? 1 : 0),
                  "dgsem_set_indicator_parameters");
  }

  std::size_t get_ndofs() const { return dofs_per_element_; }

  // State on the host in the reference's logical layout u(i, j[, k], dof, var).
  std::vector<double> to_host(const Solution<Mesh, Basis, Eq>& sol) const {
    detail::DeviceArray tmp(sol.size());
    detail::check(dgsem_to_reference_layout(ctx_, sol.state(), tmp.data()),
                  "dgsem_to_reference_layout");
    std::vector<double> out(sol.size());
    detail::check_cuda(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
    detail::check_cuda(cudaMemcpy(out.data(), tmp.data(), out.size() * sizeof(double),
                                  cudaMemcpyDeviceToHost),
                       "cudaMemcpy");
    return out;
  }

  dgsem_ctx* handle() const { return ctx_; }
  cudaStream_t stream() const { return stream_; }

 private:
  StructuredSolver(const Eq& eq, const Mesh& mesh, const BoundarySetType& bcs,
                   cudaStream_t stream)
      : mesh_(mesh), stream_(stream) {
    static_assert(BoundarySetType::NFaces == 2 * NDIMS, "one boundary condition per face");
    mdesc_ = dgsem_mesh_desc{};
    mdesc_.ndims = static_cast<int>(NDIMS);
    mdesc_.polydeg = static_cast<int>(Basis::polydeg);
    for (std::size_t a = 0; a < 3; ++a) {
      mdesc_.n_cells[a] = a < NDIMS ? static_cast<int64_t>(mesh.cells()[a]) : 1;
      mdesc_.domain_left[a] = a < NDIMS ? static_cast<double>(mesh.domain_left()[a]) : 0.0;
      mdesc_.domain_right[a] = a < NDIMS ? static_cast<double>(mesh.domain_right()[a]) : 1.0;
    }
    dgsem_scheme_desc s{};
    s.equation = Eq::dgsem_code;
    s.volume_flux = VolumeIntegral::volume_flux;
    s.surface_flux = SurfaceFlux::dgsem_code;
    s.volume_integral = VolumeIntegral::dgsem_code;
    for (std::size_t f = 0; f < 6; ++f) s.bc[f] = bcs.kinds[f];
    for (std::size_t q = 0; q < 4; ++q) s.bc_state[q] = bcs.state[q];
    s.gamma = static_cast<double>(eq.get_gamma());
    s.mu = static_cast<double>(eq.viscosity());
    s.prandtl = static_cast<double>(eq.prandtl_number());
    s.alpha_max = 0.5;
    s.alpha_min = 0.001;
    s.alpha_smooth = 0;
    detail::check(dgsem_ctx_create(&mdesc_, &s, stream, &ctx_), "dgsem_ctx_create");
    dofs_per_element_ = 1;
    for (std::size_t a = 0; a < NDIMS; ++a) dofs_per_element_ *= Basis::NNodes;
  }

  const Mesh& mesh_;
  cudaStream_t stream_;
  dgsem_mesh_desc mdesc_{};
  dgsem_ctx* ctx_ = nullptr;
  std::size_t dofs_per_element_ = 0;
};

// ---- observers (observer/observer_base.hpp) ---------------------------------
class SimulationObserver {
 public:
  virtual void on_step(int step, double time, bool& has_nan) { (void)step, (void)time, (void)has_nan; }
  virtual void on_finish(int step, double time) { (void)step, (void)time; }
  virtual ~SimulationObserver() = default;
};

class PrintObserver : public SimulationObserver {
 public:
  explicit PrintObserver(int interval = 100) : interval_(interval) {}
  void on_step(int step, double time, bool&) override {
    if (interval_ > 0 && step % interval_ == 0) std::printf("step %d  t = %.6e\n", step, time);
  }
  void on_finish(int step, double time) override {
    std::printf("finished: %d steps, t = %.6e\n", step, time);
  }

 private:
  int interval_;
};

// ---- time integration (time_integrator/SSPRK3.hpp, integrator_base.hpp) ----
template <class T, class Solver, class Mesh, class Sol>
class SSPRK3 {
 public:
  explicit SSPRK3(const Sol&, const Mesh&) {}
  SSPRK3(const Sol&, const Mesh&, T final_time) : final_time_(final_time) {}

  // One step at the integrator's clock (the clock itself advances in solve()).
  void step(Solver& solver, Sol& sol, T dt) {
    detail::check(dgsem_ssprk3_step(solver.handle(), sol.state(), static_cast<double>(time_),
                                    static_cast<double>(dt)),
                  "dgsem_ssprk3_step");
  }

  void add_observer(std::unique_ptr<SimulationObserver> obs) {
    observers_.push_back(std::move(obs));
  }

  // while (time < final_time) { observers; step; time += dt; stop on NaN }
  // (integrator_base.hpp:24-44); the non-finite check reads the device flag
  // set by the stage kernels.
  void solve(Solver& solver, Sol& sol, T dt) {
    while (time_ < final_time_) {
      for (auto& o : observers_) o->on_step(iter_, static_cast<double>(time_), has_nan_);
      step(solver, sol, dt);
      time_ += dt;
      ++iter_;
      if (!observers_.empty()) {
        const dgsem_status s = dgsem_check_finite(solver.handle());
        if (s == DGSEM_ERR_NONFINITE) has_nan_ = true;
        else detail::check(s, "dgsem_check_finite");
      }
      if (has_nan_) break;
    }
    for (auto& o : observers_) o->on_finish(iter_, static_cast<double>(time_));
  }

  T get_time() const { return time_; }
  void set_time(T t) { time_ = t; }
  bool has_nan() const { return has_nan_; }

 private:
  T time_ = T(0);
  T final_time_ = T(0);
  int iter_ = 0;
  bool has_nan_ = false;
  std::vector<std::unique_ptr<SimulationObserver>> observers_;
};

}  // namespace DGSEM

#endif  // DGSEM_B200_HPP_

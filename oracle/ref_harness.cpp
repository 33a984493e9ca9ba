// Oracle harness over the UNMODIFIED reference solver (test infrastructure).
//
// Compiled against the reference's own headers (src/ of RetrO598/DGSEM) and
// the project-written Kokkos-compatible shim in oracle/kokkos_shim.  Every
// numerical operation executed here is the reference's code:
//   StructuredSolver::calc_rhs          solver/structured_solver.hpp:466-480
//   SSPRK3::step                        time_integrator/SSPRK3.hpp:159-181
//   HGIndicator<.,.,2/3>::operator()    subcell_limiting/indicator.hpp:337,455
//   StructuredElementInitializer        containers/data_container.hpp:729-772
//   LobattoLegendreBasis::initialize    polynomial_basis/basis.hpp:69-153
// The only project-written numerics are the initial/boundary state functors
// of the benchmark cases (their formulas follow the reference examples
// Euler2D/double_mach_reflection/double_mach_reflection_structured.cpp:9-32,
// Euler2D/kelvin_helmholtz_hg/kelvin_helmholtz_hg.cpp IC and
// Euler3D/inviscid_tgv/inviscid_tgv.cpp:18-35).
//
// Arrays cross this C ABI in the reference's logical LayoutRight order:
//   u(i, j[, k], dof, var),  dof = local_dof(inode, jnode[, knode]).
#include <base/base.hpp>
#include <boundary_condition/boundary_condition.hpp>
#include <containers/containers.hpp>
#include <equations/equations.hpp>
#include <mesh/mesh.hpp>
#include <polynomial_basis/polynomial_basis.hpp>
#include <solver/solver.hpp>
#include <space_integral/space_integral.hpp>
#include <subcell_limiting/subcell_limiting.hpp>
#include <time_integrator/time_integrator.hpp>
#include <utils/utils.hpp>

#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <numbers>
#include <type_traits>

extern "C" {
// Case kinds understood by the harness.
enum {
  REF_EULER2D_PERIODIC_SPLIT = 0,  // KH-like plain split form
  REF_EULER2D_PERIODIC_HG = 1,     // periodic + HG shock capturing
  REF_EULER2D_DMR_HG = 2,          // double Mach reflection BCs + HG
  REF_EULER3D_PERIODIC_SPLIT = 3,  // TGV-like plain split form
  REF_EULER3D_PERIODIC_HG = 4,     // 3D periodic + HG
  REF_NS2D_PERIODIC_SPLIT = 5,     // Navier-Stokes BR1 + split form
  REF_EULER2D_CENTRAL_DIRICHLET = 6,  // the reference's CentralFlux + user DirichletBC
  REF_EULER2D_CURVED_CENTRAL = 7,     // curvilinear periodic mesh, CentralFlux + LLF
  REF_EULER3D_CURVED = 8,             // curvilinear periodic mesh, Chandrashekar + LLF
  REF_NS2D_CHANNEL_WALLS = 9,         // NS, x periodic, no-slip bottom / slip top walls
  REF_NS3D_PERIODIC_SPLIT = 10,       // 3D Navier-Stokes BR1 + split form, periodic box
  REF_NS2D_PERIODIC_HG = 11,          // 2D Navier-Stokes + HG shock capturing (viscous KHI)
};

typedef struct {
  int kind;
  int polydeg;
  int n_cells[3];
  double left[3];
  double right[3];
  double gamma;
  double mu;
  double prandtl;
  double alpha_max;
  double alpha_min;
  int volume_flux;   // 0 Chandrashekar (reference), 1 Ranocha, 2 Kennedy-Gruber
  int surface_flux;  // 0 LaxFriedrichs (reference), 1 HLLC (2D)
} dgsem_ref_case;
}

namespace {

using T = double;

// Double Mach reflection state; formula of the reference example
// double_mach_reflection_structured.cpp:9-32.
inline std::array<T, 4> dmr_state(const std::array<T, 2>& c, T time, T gamma) {
  constexpr T one_sixth = static_cast<T>(1.0 / 6.0);
  const T shock = one_sixth + (c[1] + static_cast<T>(20.0) * time) /
                                  std::sqrt(static_cast<T>(3.0));
  if (c[0] < shock) {
    constexpr T phi = static_cast<T>(std::numbers::pi / 6.0);
    const T s = std::sin(phi);
    const T co = std::cos(phi);
    return DGSEM::utils::prim_to_cons(
        std::array<T, 4>{static_cast<T>(8.0), static_cast<T>(8.25) * co,
                         -static_cast<T>(8.25) * s, static_cast<T>(116.5)},
        gamma);
  }
  return DGSEM::utils::prim_to_cons(
      std::array<T, 4>{static_cast<T>(1.4), T(0), T(0), static_cast<T>(1.0)},
      gamma);
}

struct DmrBoundaryState {
  T gamma;
  std::array<T, 4> operator()(const std::array<T, 2>& c, T t) const {
    return dmr_state(c, t, gamma);
  }
};
// The user Dirichlet state of the plugin-surface test (the same formula as
// tests/cpp/plugin_central.cu): a density and pressure wave travelling
// through a uniform flow, conserved variables, gamma = 1.4.
struct TravellingWave {
  std::array<T, 4> operator()(const std::array<T, 2>& x, T t) const {
    const T pi = static_cast<T>(3.14159265358979323846);
    const T rho = T(1) + T(0.2) * std::sin(pi * (x[0] + x[1] - T(0.4) * t));
    const T u = T(0.3), v = T(-0.2);
    const T p = T(1) + T(0.1) * std::cos(pi * (x[0] - x[1]));
    return {rho, rho * u, rho * v, p / T(0.4) + T(0.5) * rho * (u * u + v * v)};
  }
};

// A curvilinear mapping of the reference square / cube [-1, 1]^D with the
// reference's Mapping interface (eval, base/mapping.hpp:31-50): the linear
// map onto [left, right] plus a displacement that vanishes on the boundary,
// so the mesh stays periodic.  The same formula is the device mapping of the
// curvilinear tests (tests/cpp/plugin_curved.cu).
template <std::size_t D>
struct CurvedMapping {
  std::array<T, D> left{}, right{};
  T amp = T(0.05);
  std::array<T, D> eval(const std::array<T, D>& xi) const {
    const T pi = static_cast<T>(3.14159265358979323846);
    const std::array<T, D> lin = DGSEM::linear_interpolate(xi, left, right);
    T bump = T(1);
    for (std::size_t a = 0; a < D; ++a) bump *= std::sin(pi * xi[a]);
    std::array<T, D> x{};
    for (std::size_t a = 0; a < D; ++a)
      x[a] = lin[a] + amp * (right[a] - left[a]) * bump * (a == 0 ? T(1) : T(-0.5));
    return x;
  }
};

struct DmrBottomInflow {
  bool operator()(const std::array<T, 2>& c, T) const {
    return c[0] < static_cast<T>(1.0 / 6.0);
  }
};

// ---------------------------------------------------------------------------
// Two-point / surface fluxes the reference does not ship, written as plugins
// with the reference's flux signature numerical_flux(eq, uL, uR, normal)
// (base/numerical_flux.hpp:436-500) so they run inside the reference's own
// VolumeIntegralSplitForm / InterfaceHelper / boundary assembly.
//   Ranocha: J. Sci. Comput. 76 (2018) / (2020); Kennedy & Gruber: JCP 227
//   (2008); HLLC: the reference's 1D HLLC (numerical_flux.hpp:283-378) in the
//   face-normal frame with passive tangential momentum (Toro, ch. 10).
// ---------------------------------------------------------------------------
template <class Eq>
struct PluginTraits {
  static constexpr std::size_t D = Eq::NDIMS;
  static constexpr std::size_t V = Eq::NVARS;
};

template <class Eq>
void prim_of(const Eq& eq, const std::array<T, Eq::NVARS>& u, T& rho,
             std::array<T, Eq::NDIMS>& v, T& p) {
  constexpr std::size_t D = Eq::NDIMS;
  rho = u[0];
  T sq = 0;
  for (std::size_t d = 0; d < D; ++d) {
    v[d] = u[1 + d] / rho;
    sq += v[d] * v[d];
  }
  p = (eq.get_gamma() - T(1)) * (u[D + 1] - T(0.5) * rho * sq);
}

template <class Eq>
struct KennedyGruberPlugin {
  static std::array<T, Eq::NVARS> numerical_flux(
      const Eq& eq, const std::array<T, Eq::NVARS>& uL,
      const std::array<T, Eq::NVARS>& uR, const std::array<T, Eq::NDIMS>& n) {
    constexpr std::size_t D = Eq::NDIMS;
    T rL, rR, pL, pR;
    std::array<T, D> vL, vR;
    prim_of(eq, uL, rL, vL, pL);
    prim_of(eq, uR, rR, vR, pR);
    const T rho_avg = T(0.5) * (rL + rR);
    const T e_avg = T(0.5) * (uL[D + 1] / rL + uR[D + 1] / rR);
    const T p_avg = T(0.5) * (pL + pR);
    std::array<T, D> va;
    T vn = 0;
    for (std::size_t d = 0; d < D; ++d) {
      va[d] = T(0.5) * (vL[d] + vR[d]);
      vn += va[d] * n[d];
    }
    std::array<T, Eq::NVARS> f{};
    f[0] = rho_avg * vn;
    for (std::size_t d = 0; d < D; ++d) f[1 + d] = f[0] * va[d] + p_avg * n[d];
    f[D + 1] = (rho_avg * e_avg + p_avg) * vn;
    return f;
  }
};

template <class Eq>
struct RanochaPlugin {
  static T inv_ln_mean(T x, T y) {
    const T num = x * (x - T(2) * y) + y * y;
    const T den = x * (x + T(2) * y) + y * y;
    const T f2 = num / den;
    if (f2 < T(1.0e-4)) {
      const T poly = T(2) + f2 * (T(2.0 / 3.0) + f2 * (T(2.0 / 5.0) + f2 * T(2.0 / 7.0)));
      return poly / (x + y);
    }
    return std::log(y / x) / (y - x);
  }
  static std::array<T, Eq::NVARS> numerical_flux(
      const Eq& eq, const std::array<T, Eq::NVARS>& uL,
      const std::array<T, Eq::NVARS>& uR, const std::array<T, Eq::NDIMS>& n) {
    constexpr std::size_t D = Eq::NDIMS;
    T rL, rR, pL, pR;
    std::array<T, D> vL, vR;
    prim_of(eq, uL, rL, vL, pL);
    prim_of(eq, uR, rR, vR, pR);
    T vnL = 0, vnR = 0, vLvR = 0;
    for (std::size_t d = 0; d < D; ++d) {
      vnL += vL[d] * n[d];
      vnR += vR[d] * n[d];
      vLvR += vL[d] * vR[d];
    }
    const T rho_mean = DGSEM::ln_mean(rL, rR);
    const T inv_rho_p_mean = pL * pR * inv_ln_mean(rL * pR, rR * pL);
    const T p_avg = T(0.5) * (pL + pR);
    std::array<T, Eq::NVARS> f{};
    f[0] = rho_mean * T(0.5) * (vnL + vnR);
    for (std::size_t d = 0; d < D; ++d)
      f[1 + d] = f[0] * (T(0.5) * (vL[d] + vR[d])) + p_avg * n[d];
    f[D + 1] = f[0] * (T(0.5) * vLvR + inv_rho_p_mean / (eq.get_gamma() - T(1))) +
               T(0.5) * (pL * vnR + pR * vnL);
    return f;
  }
};

struct HLLC2DPlugin {
  using Eq = DGSEM::equations::CompressibleEuler2D<T>;
  static std::array<T, 4> numerical_flux(const Eq& eq, const std::array<T, 4>& uL,
                                         const std::array<T, 4>& uR,
                                         const std::array<T, 2>& n) {
    const T g = eq.get_gamma();
    const T nn = std::sqrt(n[0] * n[0] + n[1] * n[1]);
    const T nx = n[0] / nn, ny = n[1] / nn;
    const T rL = uL[0], rR = uR[0];
    const T mnL = uL[1] * nx + uL[2] * ny, mtL = -uL[1] * ny + uL[2] * nx;
    const T mnR = uR[1] * nx + uR[2] * ny, mtR = -uR[1] * ny + uR[2] * nx;
    const T EL = uL[3], ER = uR[3];
    const T vL = mnL / rL, vR = mnR / rR, wL = mtL / rL, wR = mtR / rR;
    const T pL = (g - T(1)) * (EL - T(0.5) * rL * (vL * vL + wL * wL));
    const T pR = (g - T(1)) * (ER - T(0.5) * rR * (vR * vR + wR * wR));
    const T cL = std::sqrt(g * pL / rL), cR = std::sqrt(g * pR / rR);
    const T srL = std::sqrt(rL), srR = std::sqrt(rR), ss = srL + srR;
    const T v_roe = (srL * vL + srR * vR) / ss;
    const T w_roe = (srL * wL + srR * wR) / ss;
    const T ek = T(0.5) * (v_roe * v_roe + w_roe * w_roe);
    const T H_roe = (srL * ((EL + pL) / rL) + srR * ((ER + pR) / rR)) / ss;
    const T c_roe = std::sqrt((g - T(1)) * (H_roe - ek));
    const T SL = std::min(vL - cL, v_roe - c_roe);
    const T SR = std::max(vR + cR, v_roe + c_roe);
    T q[4];
    if (SL >= 0) {
      q[0] = mnL; q[1] = mnL * vL + pL; q[2] = mnL * wL; q[3] = vL * (EL + pL);
    } else if (SR <= 0) {
      q[0] = mnR; q[1] = mnR * vR + pR; q[2] = mnR * wR; q[3] = vR * (ER + pR);
    } else {
      const T sMuL = SL - vL, sMuR = SR - vR;
      const T SS = (pR - pL + rL * vL * sMuL - rR * vR * sMuR) / (rL * sMuL - rR * sMuR);
      if (SS >= 0) {
        const T dS = rL * sMuL / (SL - SS);
        const T eS = EL / rL + (SS - vL) * (SS + pL / (rL * sMuL));
        q[0] = mnL + SL * (dS - rL);
        q[1] = (mnL * vL + pL) + SL * (dS * SS - mnL);
        q[2] = mnL * wL + SL * (dS * wL - mtL);
        q[3] = vL * (EL + pL) + SL * (dS * eS - EL);
      } else {
        const T dS = rR * sMuR / (SR - SS);
        const T eS = ER / rR + (SS - vR) * (SS + pR / (rR * sMuR));
        q[0] = mnR + SR * (dS - rR);
        q[1] = (mnR * vR + pR) + SR * (dS * SS - mnR);
        q[2] = mnR * wR + SR * (dS * wR - mtR);
        q[3] = vR * (ER + pR) + SR * (dS * eS - ER);
      }
    }
    return {q[0] * nn, (q[1] * nx - q[2] * ny) * nn, (q[1] * ny + q[2] * nx) * nn, q[3] * nn};
  }
};

class RefCaseBase {
 public:
  virtual ~RefCaseBase() = default;
  virtual void rhs(const T* u, T* du, T t) = 0;
  virtual void alpha(const T* u, T* a) = 0;
  virtual void steps(T* u, T t0, T dt, int n) = 0;
  virtual void geometry(T* coords, T* ja, T* inv_j) = 0;
  virtual std::size_t state_size() const = 0;
};

template <class Eq, std::size_t N, class VolumeFlux, class Boundaries,
          std::size_t D, class SurfaceFlux = DGSEM::LaxFriedrichsFlux<Eq>>
class RefCase final : public RefCaseBase {
 public:
  using Basis = DGSEM::Basis::LobattoLegendreBasis<T, N>;
  using Mesh = DGSEM::StructuredMesh<T, D>;
  using Solver = DGSEM::StructuredSolver<Eq, Basis, VolumeFlux, SurfaceFlux,
                                         Mesh, Boundaries>;
  using Sol = DGSEM::Solution<Mesh, Basis, Eq>;

  RefCase(const dgsem_ref_case& c, const Eq& eq, const Boundaries& bcs,
          bool periodic)
      : RefCase(c, eq, bcs, make_periodic(periodic)) {}

  RefCase(const dgsem_ref_case& c, const Eq& eq, const Boundaries& bcs,
          const std::array<bool, D>& periodic)
      : mesh_(make_left(c), make_right(c), make_cells(c)),
        solver_(eq, mesh_, container_, bcs, periodic),
        sol_(mesh_),
        c_(c) {
    solver_.set_indicator_parameters(c.alpha_max, c.alpha_min, false);
  }

  static std::array<T, D> make_left(const dgsem_ref_case& c) {
    std::array<T, D> a{};
    for (std::size_t i = 0; i < D; ++i) a[i] = c.left[i];
    return a;
  }
  static std::array<T, D> make_right(const dgsem_ref_case& c) {
    std::array<T, D> a{};
    for (std::size_t i = 0; i < D; ++i) a[i] = c.right[i];
    return a;
  }
  static std::array<std::size_t, D> make_cells(const dgsem_ref_case& c) {
    std::array<std::size_t, D> a{};
    for (std::size_t i = 0; i < D; ++i) a[i] = c.n_cells[i];
    return a;
  }
  static std::array<bool, D> make_periodic(bool p) {
    std::array<bool, D> a{};
    a.fill(p);
    return a;
  }

  std::size_t state_size() const override { return sol_.u_device.size(); }

  void rhs(const T* u, T* du, T t) override {
    std::memcpy(sol_.u_device.data(), u, state_size() * sizeof(T));
    solver_.calc_rhs(sol_, t);
    std::memcpy(du, sol_.du_device.data(), state_size() * sizeof(T));
  }

  void alpha(const T* u, T* a) override {
    // the reference defines no shock indicator for 3D Navier-Stokes
    if constexpr (!std::is_same_v<Eq, DGSEM::equations::CompressibleNavierStokes3D<T>>) {
    std::memcpy(sol_.u_device.data(), u, state_size() * sizeof(T));
    using ElementArray =
        typename DGSEM::solution_type_traits<T, D>::ElementArray;
    auto cells = make_cells(c_);
    ElementArray av;
    if constexpr (D == 2) {
      av = ElementArray("alpha", cells[0], cells[1]);
    } else {
      av = ElementArray("alpha", cells[0], cells[1], cells[2]);
    }
    DGSEM::HGIndicator<Basis, Eq> ind(c_.alpha_max, c_.alpha_min, false,
                                      Basis::device_data());
    ind(cells, sol_.u_device, av);
    std::memcpy(a, av.data(), av.size() * sizeof(T));
    }
  }

  void steps(T* u, T t0, T dt, int n) override {
    std::memcpy(sol_.u_device.data(), u, state_size() * sizeof(T));
    if (!integrator_) {
      integrator_ = std::make_unique<DGSEM::SSPRK3<T, Solver, Mesh, Sol>>(
          sol_, mesh_, t0 + n * dt);
    }
    // SSPRK3::step reads the integrator's own clock; drive it through the
    // public step() with the stage times t, t+dt, t+dt/2 of that clock.
    for (int s = 0; s < n; ++s) {
      StepAccess::set_time(*integrator_, t0 + s * dt);
      integrator_->step(solver_, sol_, dt);
    }
    std::memcpy(u, sol_.u_device.data(), state_size() * sizeof(T));
  }

  void geometry(T* coords, T* ja, T* inv_j) override {
    if (coords)
      std::memcpy(coords, container_.node_coordinates.data(),
                  container_.node_coordinates.size() * sizeof(T));
    if (ja)
      std::memcpy(ja, container_.contravariant_vectors.data(),
                  container_.contravariant_vectors.size() * sizeof(T));
    if (inv_j)
      std::memcpy(inv_j, container_.inverse_jacobian.data(),
                  container_.inverse_jacobian.size() * sizeof(T));
  }

 private:
  // TimeIntegrator keeps `time` protected; a derived accessor sets it.
  struct StepAccess : DGSEM::SSPRK3<T, Solver, Mesh, Sol> {
    static void set_time(DGSEM::SSPRK3<T, Solver, Mesh, Sol>& ig, T t) {
      static_cast<StepAccess&>(ig).time = t;
    }
  };

  Mesh mesh_;
  DGSEM::StructuredElementContainer<T, D> container_;
  Solver solver_;
  Sol sol_;
  dgsem_ref_case c_;
  std::unique_ptr<DGSEM::SSPRK3<T, Solver, Mesh, Sol>> integrator_;
};

// 2D shock capturing (VolumeIntegralShockCapturingHG with the reference's
// LaxFriedrichsFlux for the FV subcells) with the volume flux chosen by
// c.volume_flux and the surface flux by c.surface_flux.  The plugin volume
// fluxes are instantiated at polydeg 3 (the benchmark degree) only, to bound
// the build time.
template <std::size_t N, template <class> class VFlux, class Bcs>
RefCaseBase* make_hg_2d_vf(const dgsem_ref_case& c, const DGSEM::equations::CompressibleEuler2D<T>& eq,
                           const Bcs& b, bool periodic) {
  using Basis = DGSEM::Basis::LobattoLegendreBasis<T, N>;
  using E2 = DGSEM::equations::CompressibleEuler2D<T>;
  using VF = DGSEM::VolumeIntegralShockCapturingHG<Basis, E2, VFlux, DGSEM::LaxFriedrichsFlux,
                                                   DGSEM::HGIndicator<Basis, E2>>;
  if (c.surface_flux == 1) return new RefCase<E2, N, VF, Bcs, 2, HLLC2DPlugin>(c, eq, b, periodic);
  return new RefCase<E2, N, VF, Bcs, 2>(c, eq, b, periodic);
}

template <std::size_t N, class Bcs>
RefCaseBase* make_hg_2d(const dgsem_ref_case& c, const DGSEM::equations::CompressibleEuler2D<T>& eq,
                        const Bcs& b, bool periodic) {
  if constexpr (N == 3) {
    if (c.volume_flux == 1) return make_hg_2d_vf<N, RanochaPlugin>(c, eq, b, periodic);
    if (c.volume_flux == 2) return make_hg_2d_vf<N, KennedyGruberPlugin>(c, eq, b, periodic);
  }
  if (c.volume_flux != 0) return nullptr;
  return make_hg_2d_vf<N, DGSEM::ChandrashekarFlux>(c, eq, b, periodic);
}

// 3D periodic shock capturing with the volume flux chosen by c.volume_flux
// (the plugin fluxes at polydeg 3 only).
template <std::size_t N, template <class> class VFlux>
RefCaseBase* make_hg_3d_vf(const dgsem_ref_case& c) {
  using Basis = DGSEM::Basis::LobattoLegendreBasis<T, N>;
  using E3 = DGSEM::equations::CompressibleEuler3D<T>;
  using VF = DGSEM::VolumeIntegralShockCapturingHG<Basis, E3, VFlux, DGSEM::LaxFriedrichsFlux,
                                                   DGSEM::HGIndicator<Basis, E3>>;
  using P = DGSEM::PeriodicBC;
  auto b = DGSEM::BoundarySet(P{}, P{}, P{}, P{}, P{}, P{});
  return new RefCase<E3, N, VF, decltype(b), 3>(c, E3{c.gamma}, b, true);
}

template <std::size_t N>
RefCaseBase* make_hg_3d(const dgsem_ref_case& c) {
  if constexpr (N == 3) {
    if (c.volume_flux == 1) return make_hg_3d_vf<N, RanochaPlugin>(c);
    if (c.volume_flux == 2) return make_hg_3d_vf<N, KennedyGruberPlugin>(c);
  }
  if (c.volume_flux != 0) return nullptr;
  return make_hg_3d_vf<N, DGSEM::ChandrashekarFlux>(c);
}

// RefCase on a mesh given by an arbitrary Mapping: the reference's
// StructuredElementInitializer with that mapping fills the element container,
// which the solver's 4-argument constructor takes as is
// (solver/structured_solver.hpp:36-42).
template <class Eq, std::size_t N, class VolumeFlux, class Boundaries, std::size_t D,
          class Mapping, class SurfaceFlux = DGSEM::LaxFriedrichsFlux<Eq>>
class MappedRefCase final : public RefCaseBase {
 public:
  using Basis = DGSEM::Basis::LobattoLegendreBasis<T, N>;
  using Mesh = DGSEM::StructuredMesh<T, D>;
  using Container = DGSEM::StructuredElementContainer<T, D>;
  using Solver = DGSEM::StructuredSolver<Eq, Basis, VolumeFlux, SurfaceFlux, Mesh, Boundaries>;
  using Sol = DGSEM::Solution<Mesh, Basis, Eq>;

  MappedRefCase(const dgsem_ref_case& c, const Eq& eq, const Boundaries& bcs, const Mapping& map)
      : mesh_(RefCase<Eq, N, VolumeFlux, Boundaries, D>::make_left(c),
              RefCase<Eq, N, VolumeFlux, Boundaries, D>::make_right(c),
              RefCase<Eq, N, VolumeFlux, Boundaries, D>::make_cells(c)),
        container_(init_container(c, map)),
        solver_(eq, mesh_, container_, bcs),
        sol_(mesh_) {}

  static Container init_container(const dgsem_ref_case& c, const Mapping& map) {
    Container k;
    std::array<bool, D> per{};
    per.fill(true);
    DGSEM::StructuredElementInitializer<T, Basis, Mapping, D> init(map, per);
    init.init_elements(RefCase<Eq, N, VolumeFlux, Boundaries, D>::make_cells(c), k);
    return k;
  }

  std::size_t state_size() const override { return sol_.u_device.size(); }
  void rhs(const T* u, T* du, T t) override {
    std::memcpy(sol_.u_device.data(), u, state_size() * sizeof(T));
    solver_.calc_rhs(sol_, t);
    std::memcpy(du, sol_.du_device.data(), state_size() * sizeof(T));
  }
  void alpha(const T*, T*) override {}
  void steps(T*, T, T, int) override {}
  void geometry(T* coords, T* ja, T* inv_j) override {
    if (coords)
      std::memcpy(coords, container_.node_coordinates.data(),
                  container_.node_coordinates.size() * sizeof(T));
    if (ja)
      std::memcpy(ja, container_.contravariant_vectors.data(),
                  container_.contravariant_vectors.size() * sizeof(T));
    if (inv_j)
      std::memcpy(inv_j, container_.inverse_jacobian.data(),
                  container_.inverse_jacobian.size() * sizeof(T));
  }

 private:
  Mesh mesh_;
  Container container_;
  Solver solver_;
  Sol sol_;
};

template <std::size_t N>
RefCaseBase* make_case_n(const dgsem_ref_case& c) {
  using Basis = DGSEM::Basis::LobattoLegendreBasis<T, N>;
  Basis::initialize();
  using E2 = DGSEM::equations::CompressibleEuler2D<T>;
  using E3 = DGSEM::equations::CompressibleEuler3D<T>;
  using NS2 = DGSEM::equations::CompressibleNavierStokes2D<T>;
  using NS3 = DGSEM::equations::CompressibleNavierStokes3D<T>;
  using P = DGSEM::PeriodicBC;
  switch (c.kind) {
    case REF_EULER2D_PERIODIC_SPLIT: {
      auto b = DGSEM::BoundarySet(P{}, P{}, P{}, P{});
      if (c.volume_flux == 1) {
        using VF = DGSEM::VolumeIntegralSplitForm<Basis, E2, RanochaPlugin>;
        return new RefCase<E2, N, VF, decltype(b), 2>(c, E2{c.gamma}, b, true);
      }
      if (c.volume_flux == 2) {
        using VF = DGSEM::VolumeIntegralSplitForm<Basis, E2, KennedyGruberPlugin>;
        return new RefCase<E2, N, VF, decltype(b), 2>(c, E2{c.gamma}, b, true);
      }
      using VF = DGSEM::VolumeIntegralSplitForm<Basis, E2, DGSEM::ChandrashekarFlux>;
      return new RefCase<E2, N, VF, decltype(b), 2>(c, E2{c.gamma}, b, true);
    }
    case REF_EULER2D_PERIODIC_HG: {
      auto b = DGSEM::BoundarySet(P{}, P{}, P{}, P{});
      return make_hg_2d<N>(c, E2{c.gamma}, b, true);
    }
    case REF_EULER2D_DMR_HG: {
      DmrBoundaryState inflow{c.gamma};
      auto b = DGSEM::BoundarySet(
          DGSEM::DirichletBC(inflow), DGSEM::OutflowBC{},
          DGSEM::MixedDirichletSlipWallBC(inflow, DmrBottomInflow{}),
          DGSEM::DirichletBC(inflow));
      return make_hg_2d<N>(c, E2{c.gamma}, b, false);
    }
    case REF_EULER3D_PERIODIC_SPLIT: {
      auto b = DGSEM::BoundarySet(P{}, P{}, P{}, P{}, P{}, P{});
      if (c.volume_flux == 1) {
        using VF = DGSEM::VolumeIntegralSplitForm<Basis, E3, RanochaPlugin>;
        return new RefCase<E3, N, VF, decltype(b), 3>(c, E3{c.gamma}, b, true);
      }
      if (c.volume_flux == 2) {
        using VF = DGSEM::VolumeIntegralSplitForm<Basis, E3, KennedyGruberPlugin>;
        return new RefCase<E3, N, VF, decltype(b), 3>(c, E3{c.gamma}, b, true);
      }
      using VF = DGSEM::VolumeIntegralSplitForm<Basis, E3, DGSEM::ChandrashekarFlux>;
      return new RefCase<E3, N, VF, decltype(b), 3>(c, E3{c.gamma}, b, true);
    }
    case REF_EULER3D_PERIODIC_HG:
      return make_hg_3d<N>(c);
    case REF_EULER2D_CENTRAL_DIRICHLET: {
      if constexpr (N == 3) {
        TravellingWave w;
        auto b = DGSEM::BoundarySet(DGSEM::DirichletBC(w), DGSEM::DirichletBC(w),
                                    DGSEM::DirichletBC(w), DGSEM::DirichletBC(w));
        using VF = DGSEM::VolumeIntegralSplitForm<Basis, E2, DGSEM::CentralFlux>;
        return new RefCase<E2, N, VF, decltype(b), 2>(c, E2{c.gamma}, b, false);
      }
      return nullptr;
    }
    case REF_EULER2D_CURVED_CENTRAL: {
      if constexpr (N == 3) {
        CurvedMapping<2> map;
        for (int a = 0; a < 2; ++a) {
          map.left[a] = c.left[a];
          map.right[a] = c.right[a];
        }
        auto b = DGSEM::BoundarySet(P{}, P{}, P{}, P{});
        using VF = DGSEM::VolumeIntegralSplitForm<Basis, E2, DGSEM::CentralFlux>;
        return new MappedRefCase<E2, N, VF, decltype(b), 2, CurvedMapping<2>>(c, E2{c.gamma}, b,
                                                                              map);
      }
      return nullptr;
    }
    case REF_EULER3D_CURVED: {
      if constexpr (N <= 4) {
        CurvedMapping<3> map;
        for (int a = 0; a < 3; ++a) {
          map.left[a] = c.left[a];
          map.right[a] = c.right[a];
        }
        auto b = DGSEM::BoundarySet(P{}, P{}, P{}, P{}, P{}, P{});
        using VF = DGSEM::VolumeIntegralSplitForm<Basis, E3, DGSEM::ChandrashekarFlux>;
        return new MappedRefCase<E3, N, VF, decltype(b), 3, CurvedMapping<3>>(c, E3{c.gamma}, b,
                                                                              map);
      }
      return nullptr;
    }
    case REF_NS2D_CHANNEL_WALLS: {
      using VF = DGSEM::VolumeIntegralSplitForm<Basis, NS2, DGSEM::ChandrashekarFlux>;
      auto b = DGSEM::BoundarySet(P{}, P{}, DGSEM::NSNoSlipAdiabaticWallBC{},
                                  DGSEM::NSSlipAdiabaticWallBC{});
      return new RefCase<NS2, N, VF, decltype(b), 2>(c, NS2{c.gamma, c.mu, c.prandtl}, b,
                                                     std::array<bool, 2>{true, false});
    }
    case REF_NS2D_PERIODIC_SPLIT: {
      using VF = DGSEM::VolumeIntegralSplitForm<Basis, NS2, DGSEM::ChandrashekarFlux>;
      auto b = DGSEM::BoundarySet(P{}, P{}, P{}, P{});
      return new RefCase<NS2, N, VF, decltype(b), 2>(
          c, NS2{c.gamma, c.mu, c.prandtl}, b, true);
    }
    case REF_NS2D_PERIODIC_HG: {
      using VF = DGSEM::VolumeIntegralShockCapturingHG<Basis, NS2, DGSEM::ChandrashekarFlux,
                                                       DGSEM::LaxFriedrichsFlux,
                                                       DGSEM::HGIndicator<Basis, NS2>>;
      auto b = DGSEM::BoundarySet(P{}, P{}, P{}, P{});
      return new RefCase<NS2, N, VF, decltype(b), 2>(c, NS2{c.gamma, c.mu, c.prandtl}, b, true);
    }
    case REF_NS3D_PERIODIC_SPLIT: {
      if constexpr (N <= 4) {
        using VF = DGSEM::VolumeIntegralSplitForm<Basis, NS3, DGSEM::ChandrashekarFlux>;
        auto b = DGSEM::BoundarySet(P{}, P{}, P{}, P{}, P{}, P{});
        return new RefCase<NS3, N, VF, decltype(b), 3>(c, NS3{c.gamma, c.mu, c.prandtl}, b,
                                                       true);
      }
      return nullptr;
    }
    default:
      return nullptr;
  }
}

RefCaseBase* make_case(const dgsem_ref_case& c) {
  const bool is3d = c.kind == REF_EULER3D_PERIODIC_SPLIT || c.kind == REF_EULER3D_PERIODIC_HG ||
                    c.kind == REF_EULER3D_CURVED || c.kind == REF_NS3D_PERIODIC_SPLIT;
  if (is3d) {
    switch (c.polydeg) {
      case 1: return make_case_n<1>(c);
      case 2: return make_case_n<2>(c);
      case 3: return make_case_n<3>(c);
      case 4: return make_case_n<4>(c);
      default: return nullptr;
    }
  }
  switch (c.polydeg) {
    case 1: return make_case_n<1>(c);
    case 2: return make_case_n<2>(c);
    case 3: return make_case_n<3>(c);
    case 4: return make_case_n<4>(c);
    case 5: return make_case_n<5>(c);
    case 6: return make_case_n<6>(c);
    case 7: return make_case_n<7>(c);
    default: return nullptr;
  }
}

template <std::size_t N>
void basis_tables_n(double* out) {
  using Basis = DGSEM::Basis::LobattoLegendreBasis<T, N>;
  Basis::initialize();
  constexpr std::size_t n = N + 1;
  auto d = Basis::device_data();
  std::size_t o = 0;
  for (std::size_t i = 0; i < n; ++i) out[o++] = d.nodes(i);
  for (std::size_t i = 0; i < n; ++i) out[o++] = d.weights(i);
  for (std::size_t i = 0; i < n; ++i) out[o++] = d.inv_weights(i);
  for (std::size_t i = 0; i < n; ++i) out[o++] = d.boundary_interpolation_left(i);
  for (std::size_t i = 0; i < n; ++i) out[o++] = d.boundary_interpolation_right(i);
  for (std::size_t i = 0; i < n; ++i)
    for (std::size_t j = 0; j < n; ++j) out[o++] = d.derivative_matrix(i, j);
  for (std::size_t i = 0; i < n; ++i)
    for (std::size_t j = 0; j < n; ++j) out[o++] = d.derivative_split(i, j);
  for (std::size_t i = 0; i < n; ++i)
    for (std::size_t j = 0; j < n; ++j) out[o++] = d.derivative_dhat(i, j);
  for (std::size_t i = 0; i < n; ++i)
    for (std::size_t j = 0; j < n; ++j)
      out[o++] = d.inverse_vandermonde_legendre(i, j);
}

}  // namespace

extern "C" {

void* dgsem_ref_create(const dgsem_ref_case* c) {
  if (!c) return nullptr;
  if (!Kokkos::is_initialized()) Kokkos::initialize();
  return make_case(*c);
}

void dgsem_ref_destroy(void* h) { delete static_cast<RefCaseBase*>(h); }

long long dgsem_ref_state_size(void* h) {
  return h ? static_cast<long long>(static_cast<RefCaseBase*>(h)->state_size())
           : -1;
}

int dgsem_ref_rhs(void* h, const double* u, double* du, double t) {
  if (!h) return -1;
  static_cast<RefCaseBase*>(h)->rhs(u, du, t);
  return 0;
}

int dgsem_ref_alpha(void* h, const double* u, double* alpha) {
  if (!h) return -1;
  static_cast<RefCaseBase*>(h)->alpha(u, alpha);
  return 0;
}

int dgsem_ref_ssprk3(void* h, double* u, double t0, double dt, int nsteps) {
  if (!h) return -1;
  static_cast<RefCaseBase*>(h)->steps(u, t0, dt, nsteps);
  return 0;
}

int dgsem_ref_geometry(void* h, double* coords, double* ja, double* inv_j) {
  if (!h) return -1;
  static_cast<RefCaseBase*>(h)->geometry(coords, ja, inv_j);
  return 0;
}

// Basis tables in the order nodes, weights, inv_weights, lhat(-1), lhat(+1),
// D, Dsplit, Dhat, inverse Legendre Vandermonde (row-major n x n each).
int dgsem_ref_basis(int polydeg, double* out) {
  if (!Kokkos::is_initialized()) Kokkos::initialize();
  switch (polydeg) {
    case 1: basis_tables_n<1>(out); return 0;
    case 2: basis_tables_n<2>(out); return 0;
    case 3: basis_tables_n<3>(out); return 0;
    case 4: basis_tables_n<4>(out); return 0;
    case 5: basis_tables_n<5>(out); return 0;
    case 6: basis_tables_n<6>(out); return 0;
    case 7: basis_tables_n<7>(out); return 0;
    default: return -1;
  }
}

int dgsem_ref_omp_threads(void) {
#ifdef _OPENMP
  extern int omp_get_max_threads(void);
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"

// Tangent-linear oracle over the UNMODIFIED reference solver (test
// infrastructure only).
//
// The reference is generic in its scalar type (StructuredSolver<Eq<T>, ...>,
// LobattoLegendreBasis<T, N>, StructuredMesh<T, D>).  This harness
// instantiates it with a forward-mode dual number (value, tangent), so one
// run of the reference's own code yields R(u) together with the exact
// directional derivative dR/du . d, and one run of its SSPRK3 yields
// J(u(T)) with dJ/du0 . d0 -- the FP64 tangent-linear model the discrete
// adjoint is checked against.  The operations run are the reference's:
//   StructuredSolver::calc_rhs   solver/structured_solver.hpp:466-480
//   SSPRK3::step                 time_integrator/SSPRK3.hpp:159-181
// and the mean kinetic energy objective follows
// analyzer/volume_average_euler.hpp:9-69 (weights w/|1/J|,
// volume_weighted_analyzer_functor.hpp:80,104).
//
// Dual arithmetic: exact first-order derivative rules; comparisons, max, abs
// and branches act on the value (the derivative of the taken branch).
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <numeric>

struct Dual {
  double v = 0.0;  // value
  double d = 0.0;  // tangent
  constexpr Dual() = default;
  constexpr Dual(double x) : v(x), d(0.0) {}  // NOLINT: implicit by design
  constexpr Dual(double x, double y) : v(x), d(y) {}
  Dual& operator+=(const Dual& o) { v += o.v; d += o.d; return *this; }
  Dual& operator-=(const Dual& o) { v -= o.v; d -= o.d; return *this; }
  Dual& operator*=(const Dual& o) { d = d * o.v + v * o.d; v *= o.v; return *this; }
  Dual& operator/=(const Dual& o) {
    const double q = v / o.v;
    d = (d - q * o.d) / o.v;
    v = q;
    return *this;
  }
};

inline Dual operator+(Dual a, const Dual& b) { return a += b; }
inline Dual operator-(Dual a, const Dual& b) { return a -= b; }
inline Dual operator*(Dual a, const Dual& b) { return a *= b; }
inline Dual operator/(Dual a, const Dual& b) { return a /= b; }
inline Dual operator-(const Dual& a) { return Dual(-a.v, -a.d); }
inline Dual operator+(const Dual& a) { return a; }
inline bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
inline bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
inline bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
inline bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
inline bool operator==(const Dual& a, const Dual& b) { return a.v == b.v; }
inline bool operator!=(const Dual& a, const Dual& b) { return a.v != b.v; }

// The reference's ln_mean (base/math_utils.hpp:8-25) is constrained to
// floating-point types; this overload, found by argument-dependent lookup,
// evaluates the same formula (same f^2 expression, branch and series) on
// dual numbers.
inline Dual sqr_ratio_f2(const Dual& x, const Dual& y) {
  const Dual numerator = x * (x - Dual(2.0) * y) + y * y;
  const Dual denominator = x * (x + Dual(2.0) * y) + y * y;
  return numerator / denominator;
}
Dual ln_mean(Dual x, Dual y);

// Overloads the reference reaches through std:: qualified calls; they must be
// declared before its headers are included.
namespace std {
inline Dual sqrt(const Dual& a) {
  const double s = std::sqrt(a.v);
  return Dual(s, a.d / (2.0 * s));
}
inline Dual log(const Dual& a) { return Dual(std::log(a.v), a.d / a.v); }
inline Dual exp(const Dual& a) {
  const double e = std::exp(a.v);
  return Dual(e, e * a.d);
}
inline Dual abs(const Dual& a) { return a.v < 0.0 ? -a : a; }
inline Dual fabs(const Dual& a) { return a.v < 0.0 ? -a : a; }
inline Dual sin(const Dual& a) { return Dual(std::sin(a.v), std::cos(a.v) * a.d); }
inline Dual cos(const Dual& a) { return Dual(std::cos(a.v), -std::sin(a.v) * a.d); }
inline Dual tanh(const Dual& a) {
  const double t = std::tanh(a.v);
  return Dual(t, (1.0 - t * t) * a.d);
}
inline Dual pow(const Dual& a, double b) {
  const double p = std::pow(a.v, b);
  return Dual(p, b == 0.0 ? 0.0 : b * std::pow(a.v, b - 1.0) * a.d);
}
inline Dual pow(const Dual& a, int b) { return pow(a, static_cast<double>(b)); }
inline Dual pow(const Dual& a, const Dual& b) {
  const double p = std::pow(a.v, b.v);
  double d = b.v == 0.0 ? 0.0 : b.v * std::pow(a.v, b.v - 1.0) * a.d;
  if (b.d != 0.0) d += p * std::log(a.v) * b.d;
  return Dual(p, d);
}
inline Dual pow(double a, const Dual& b) { return pow(Dual(a), b); }
// The basis set-up sums Dual Lagrange polynomials with a double initial
// value (polynomial_basis/basis_detail.hpp:147); keep the sum in Dual.
inline Dual accumulate(Dual* first, Dual* last, double init) {
  Dual s(init);
  for (; first != last; ++first) s = s + *first;
  return s;
}
inline bool isnan(const Dual& a) { return std::isnan(a.v); }
inline bool isinf(const Dual& a) { return std::isinf(a.v); }
inline bool isfinite(const Dual& a) { return std::isfinite(a.v); }

template <>
class numeric_limits<Dual> {
 public:
  static constexpr bool is_specialized = true;
  static constexpr Dual epsilon() noexcept { return Dual(numeric_limits<double>::epsilon()); }
  static constexpr Dual min() noexcept { return Dual(numeric_limits<double>::min()); }
  static constexpr Dual max() noexcept { return Dual(numeric_limits<double>::max()); }
  static constexpr Dual lowest() noexcept { return Dual(numeric_limits<double>::lowest()); }
  static constexpr Dual infinity() noexcept { return Dual(numeric_limits<double>::infinity()); }
  static constexpr Dual quiet_NaN() noexcept { return Dual(numeric_limits<double>::quiet_NaN()); }
};
}  // namespace std

Dual ln_mean(Dual x, Dual y) {
  const Dual f2 = sqr_ratio_f2(x, y);
  if (f2 < Dual(1.0e-4)) {
    const Dual poly = Dual(2.0) + f2 * (Dual(2.0 / 3.0) + f2 * (Dual(2.0 / 5.0) + f2 * Dual(2.0 / 7.0)));
    return (x + y) / poly;
  }
  return (y - x) / std::log(y / x);
}

#include <base/base.hpp>
#include <boundary_condition/boundary_condition.hpp>
#include <containers/containers.hpp>
#include <equations/equations.hpp>
#include <mesh/mesh.hpp>
#include <polynomial_basis/polynomial_basis.hpp>
#include <solver/solver.hpp>
#include <space_integral/space_integral.hpp>
#include <time_integrator/time_integrator.hpp>
#include <utils/utils.hpp>

extern "C" {
// Cases: 0 = Euler 2D periodic split form, 5 = Navier-Stokes 2D periodic
// split form (BR1); Chandrashekar volume flux, LLF surface flux (the
// reference's own plugins).
typedef struct {
  int kind;
  int polydeg;
  int n_cells[2];
  double left[2];
  double right[2];
  double gamma;
  double mu;
  double prandtl;
} dgsem_tlm_case;
}

namespace {

using T = Dual;

class TlmBase {
 public:
  virtual ~TlmBase() = default;
  virtual std::size_t state_size() const = 0;
  virtual void rhs(const double* u, const double* du, double t, double* r, double* dr) = 0;
  virtual void objective(const double* u0, const double* du0, double t0, double dt, int nsteps,
                         double* J, double* dJ) = 0;
};

template <class Eq, std::size_t N>
class Tlm final : public TlmBase {
 public:
  using Basis = DGSEM::Basis::LobattoLegendreBasis<T, N>;
  using Mesh = DGSEM::StructuredMesh<T, 2>;
  using VF = DGSEM::VolumeIntegralSplitForm<Basis, Eq, DGSEM::ChandrashekarFlux>;
  using P = DGSEM::PeriodicBC;
  using Bcs = decltype(DGSEM::BoundarySet(P{}, P{}, P{}, P{}));
  using Solver = DGSEM::StructuredSolver<Eq, Basis, VF, DGSEM::LaxFriedrichsFlux<Eq>, Mesh, Bcs>;
  using Sol = DGSEM::Solution<Mesh, Basis, Eq>;

  Tlm(const dgsem_tlm_case& c, const Eq& eq)
      : mesh_(std::array<T, 2>{c.left[0], c.left[1]}, std::array<T, 2>{c.right[0], c.right[1]},
              std::array<std::size_t, 2>{(std::size_t)c.n_cells[0], (std::size_t)c.n_cells[1]}),
        solver_(eq, mesh_, container_, DGSEM::BoundarySet(P{}, P{}, P{}, P{}),
                std::array<bool, 2>{true, true}),
        sol_(mesh_),
        nx_(c.n_cells[0]),
        ny_(c.n_cells[1]) {}

  std::size_t state_size() const override { return sol_.u_device.size(); }

  void load(const double* u, const double* du) {
    T* p = sol_.u_device.data();
    for (std::size_t k = 0; k < state_size(); ++k) p[k] = Dual(u[k], du ? du[k] : 0.0);
  }

  void rhs(const double* u, const double* du, double t, double* r, double* dr) override {
    load(u, du);
    solver_.calc_rhs(sol_, T(t));
    const T* q = sol_.du_device.data();
    for (std::size_t k = 0; k < state_size(); ++k) {
      r[k] = q[k].v;
      if (dr) dr[k] = q[k].d;
    }
  }

  void objective(const double* u0, const double* du0, double t0, double dt, int nsteps,
                 double* J, double* dJ) override {
    load(u0, du0);
    DGSEM::SSPRK3<T, Solver, Mesh, Sol> ig(sol_, mesh_, T(t0 + nsteps * dt));
    for (int s = 0; s < nsteps; ++s) {
      StepAccess::set_time(ig, T(t0 + s * dt));
      ig.step(solver_, sol_, T(dt));
    }
    // mean kinetic energy with weights w_i w_j / |1/J|
    constexpr std::size_t n = N + 1;
    auto b = Basis::device_data();
    const std::size_t nx = nx_, ny = ny_;
    const T* u = sol_.u_device.data();
    const T* ij = container_.inverse_jacobian.data();
    T num(0.0), den(0.0);
    for (std::size_t ie = 0; ie < nx; ++ie)
      for (std::size_t je = 0; je < ny; ++je)
        for (std::size_t jn = 0; jn < n; ++jn)
          for (std::size_t in = 0; in < n; ++in) {
            const std::size_t dof = jn * n + in;
            const std::size_t base = ((ie * ny + je) * n * n + dof) * 4;
            const T w = b.weights(in) * b.weights(jn) / std::abs(ij[(ie * ny + je) * n * n + dof]);
            const T ke = T(0.5) * (u[base + 1] * u[base + 1] + u[base + 2] * u[base + 2]) / u[base];
            num += w * ke;
            den += w;
          }
    const T val = num / den;
    *J = val.v;
    if (dJ) *dJ = val.d;
  }

 private:
  struct StepAccess : DGSEM::SSPRK3<T, Solver, Mesh, Sol> {
    static void set_time(DGSEM::SSPRK3<T, Solver, Mesh, Sol>& ig, T t) {
      static_cast<StepAccess&>(ig).time = t;
    }
  };

  Mesh mesh_;
  DGSEM::StructuredElementContainer<T, 2> container_;
  Solver solver_;
  Sol sol_;
  std::size_t nx_, ny_;
};

template <std::size_t N>
TlmBase* make_n(const dgsem_tlm_case& c) {
  DGSEM::Basis::LobattoLegendreBasis<T, N>::initialize();
  using E2 = DGSEM::equations::CompressibleEuler2D<T>;
  using NS2 = DGSEM::equations::CompressibleNavierStokes2D<T>;
  if (c.kind == 0) return new Tlm<E2, N>(c, E2{T(c.gamma)});
  if (c.kind == 5) return new Tlm<NS2, N>(c, NS2{T(c.gamma), T(c.mu), T(c.prandtl)});
  return nullptr;
}

}  // namespace

extern "C" {

void* dgsem_tlm_create(const dgsem_tlm_case* c) {
  if (!c) return nullptr;
  if (!Kokkos::is_initialized()) Kokkos::initialize();
  switch (c->polydeg) {
    case 1: return make_n<1>(*c);
    case 2: return make_n<2>(*c);
    case 3: return make_n<3>(*c);
    case 4: return make_n<4>(*c);
    default: return nullptr;
  }
}

void dgsem_tlm_destroy(void* h) { delete static_cast<TlmBase*>(h); }

long long dgsem_tlm_state_size(void* h) {
  return h ? static_cast<long long>(static_cast<TlmBase*>(h)->state_size()) : -1;
}

// r = R(u), dr = dR/du . du (dr and du may be NULL)
int dgsem_tlm_rhs(void* h, const double* u, const double* du, double t, double* r, double* dr) {
  if (!h) return -1;
  static_cast<TlmBase*>(h)->rhs(u, du, t, r, dr);
  return 0;
}

// J(u(t0 + nsteps dt)) and dJ/du0 . du0
int dgsem_tlm_objective(void* h, const double* u0, const double* du0, double t0, double dt,
                        int nsteps, double* J, double* dJ) {
  if (!h) return -1;
  static_cast<TlmBase*>(h)->objective(u0, du0, t0, dt, nsteps, J, dJ);
  return 0;
}

}  // extern "C"

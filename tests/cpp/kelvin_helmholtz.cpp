// Kelvin-Helmholtz instability written against the reference's solver
// surface (the structure of examples/Euler2D/kelvin_helmholtz_hg/
// kelvin_helmholtz_hg.cpp: user initial condition as an AbstractInitial
// functor, StructuredSolver / Solution / SSPRK3 with observers), compiled
// against include/dgsem_b200.hpp.  Used by tests/test_cpp_facade.py.
//
//   kelvin_helmholtz <nx> <ny> <steps> <dt> <hg 0|1> <out_prefix>
// writes <out_prefix>_u0.bin and <out_prefix>_uT.bin (reference layout,
// float64) and prints the final time.
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <numbers>
#include <string>
#include <vector>

#include "dgsem_b200.hpp"

template <class T>
struct KelvinHelmholtzInitial
    : public DGSEM::AbstractInitial<KelvinHelmholtzInitial<T>,
                                    DGSEM::equations::CompressibleEuler2D<T>> {
  using Eq = DGSEM::equations::CompressibleEuler2D<T>;
  static constexpr std::size_t NDIMS = Eq::NDIMS;
  static constexpr std::size_t NVARS = Eq::NVARS;

  std::array<T, NVARS> operator()(std::array<T, NDIMS> coordinate) const {
    const T x = coordinate[0];
    const T y = coordinate[1];
    const T B = std::tanh(T(15.0) * y + T(7.5)) - std::tanh(T(15.0) * y - T(7.5));
    const T rho = T(0.5) + T(0.75) * B;
    const T v1 = T(0.5) * (B - T(1.0));
    const T v2 = T(0.1) * std::sin(T(2.0) * std::numbers::pi_v<T> * x);
    return DGSEM::utils::prim_to_cons(std::array<T, 4>{rho, v1, v2, T(1.0)}, T(1.4));
  }
};

template <class VolumeIntegral>
int run(std::size_t nx, std::size_t ny, int steps, double dt, const std::string& out) {
  using value_type = double;
  using Eq = DGSEM::equations::CompressibleEuler2D<value_type>;
  using MyBasis = DGSEM::Basis::LobattoLegendreBasis<value_type, 3>;
  using SurfaceFlux = DGSEM::LaxFriedrichsFlux<Eq>;
  using Mesh = DGSEM::StructuredMesh<value_type, 2>;
  DGSEM::BasisGuard<MyBasis> basis;
  auto boundaries = DGSEM::BoundarySet(DGSEM::PeriodicBC{}, DGSEM::PeriodicBC{},
                                       DGSEM::PeriodicBC{}, DGSEM::PeriodicBC{});
  using Solver = DGSEM::StructuredSolver<Eq, MyBasis, VolumeIntegral, SurfaceFlux, Mesh,
                                         decltype(boundaries)>;
  using Solution = DGSEM::Solution<Mesh, MyBasis, Eq>;

  std::array<value_type, 2> left = {-1.0, -1.0}, right = {1.0, 1.0};
  std::array<std::size_t, 2> n_cells = {nx, ny};
  Mesh mesh(left, right, n_cells);
  Eq eq{1.4};
  DGSEM::StructuredElementContainer<value_type, 2> container;
  DGSEM::StructuredElementInitializer<value_type, MyBasis,
                                      DGSEM::LinearMapping<std::array<value_type, 2>>, 2>
      initializer{DGSEM::LinearMapping<std::array<value_type, 2>>(left, right), {true, true}};
  initializer.init_elements(n_cells, container);
  Solver solver(eq, mesh, container, boundaries);
  Solution sol(mesh);
  solver.initialize(KelvinHelmholtzInitial<value_type>{}, sol);
  const std::vector<double> u0 = solver.to_host(sol);

  DGSEM::SSPRK3<value_type, Solver, Mesh, Solution> integrator(sol, mesh, steps * dt);
  integrator.add_observer(std::make_unique<DGSEM::PrintObserver>(100));
  integrator.solve(solver, sol, dt);
  const std::vector<double> uT = solver.to_host(sol);

  for (auto [name, v] : {std::pair{"_u0.bin", &u0}, std::pair{"_uT.bin", &uT}}) {
    FILE* f = std::fopen((out + name).c_str(), "wb");
    if (!f) return 2;
    std::fwrite(v->data(), sizeof(double), v->size(), f);
    std::fclose(f);
  }
  std::printf("final_time %.17g nan %d\n", integrator.get_time(), integrator.has_nan() ? 1 : 0);
  return 0;
}

int main(int argc, char* argv[]) {
  DGSEM::KokkosSession session(argc, argv);
  if (argc < 7) {
    std::fprintf(stderr, "usage: %s nx ny steps dt hg out_prefix\n", argv[0]);
    return 1;
  }
  const std::size_t nx = std::strtoull(argv[1], nullptr, 10);
  const std::size_t ny = std::strtoull(argv[2], nullptr, 10);
  const int steps = std::atoi(argv[3]);
  const double dt = std::strtod(argv[4], nullptr);
  const bool hg = std::atoi(argv[5]) != 0;
  const std::string out = argv[6];
  using Eq = DGSEM::equations::CompressibleEuler2D<double>;
  using MyBasis = DGSEM::Basis::LobattoLegendreBasis<double, 3>;
  try {
    if (hg) {
      using VI = DGSEM::VolumeIntegralShockCapturingHG<MyBasis, Eq, DGSEM::ChandrashekarFlux,
                                                       DGSEM::LaxFriedrichsFlux,
                                                       DGSEM::HGIndicator<MyBasis, Eq>>;
      return run<VI>(nx, ny, steps, dt, out);
    }
    using VI = DGSEM::VolumeIntegralSplitForm<MyBasis, Eq, DGSEM::ChandrashekarFlux>;
    return run<VI>(nx, ny, steps, dt, out);
  } catch (const DGSEM::Error& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 3;
  }
}

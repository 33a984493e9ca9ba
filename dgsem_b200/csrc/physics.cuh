// Device physics for the compressible Euler / Navier-Stokes DGSEM right-hand
// side: logarithmic mean, two-point volume fluxes and surface fluxes.
//
// Every flux works on per-node primitive data prepared once per node
// (`NodeState`), so the per-pair cost is only the two-point averages.  The
// formulas follow the reference's plugins:
//   ln_mean (ln_mean_rs)         base/math_utils.hpp:8-25
//   ChandrashekarFlux 2D/3D      base/numerical_flux.hpp:436-500, 520-594
//   LaxFriedrichsFlux 2D/3D      base/numerical_flux.hpp:198-228, 39-69
//   LLF wave speed |v.n|+a|n|    equations/compressible_euler2D.hpp:70-109
//   HLLC (1D, Roe/Einfeldt)      base/numerical_flux.hpp:283-378
// and, for fluxes the reference does not ship, the published formulas:
//   Ranocha (J. Sci. Comput. 2018 / 2020), Kennedy & Gruber (JCP 2008).
#pragma once

#include <cuda_runtime.h>

namespace dgsem {

enum VolumeFluxKind : int { VF_CHANDRASHEKAR = 0, VF_RANOCHA = 1, VF_KENNEDY_GRUBER = 2 };
enum SurfaceFluxKind : int { SF_LLF = 0, SF_HLLC = 1 };

// Per-node data shared by all two-point fluxes (SoA in shared memory).
template <int DIM>
struct NodeState {
  double rho;
  double v[DIM];
  double p;
  double beta;  // 0.5 rho / p  (Chandrashekar); e = E / rho (Kennedy-Gruber)
  double kin;   // 0.5 |v|^2
  double inv_rho;
};

// Reciprocals of two nonzero quantities with one division, 1/(a b) times the
// other factor.  The callers pass quantities of one pair of states (sums of
// densities, pressures, rho p products or rho / p ratios; face normal
// lengths; wave speed differences), far inside the normal range, so a b
// neither overflows nor underflows.
__device__ __forceinline__ void two_reciprocals(double a, double b, double& ra, double& rb) {
  const double r = 1.0 / (a * b);
  ra = r * b;
  rb = r * a;
}

// The logarithmic mean (series branch: (x+y)/2 times the reciprocal series
// of chandrashekar_means) and the inverse logarithmic mean, each given the
// reciprocal rs of s = x + y; the reference's branch rule.
__device__ __forceinline__ double ln_mean_rs(double x, double y, double s, double rs) {
  const double t = (x - y) * rs;
  const double f2 = t * t;
  if (f2 < 1.0e-4)
    return (0.5 * s) * (1.0 + f2 * (-1.0 / 3.0 + f2 * (-4.0 / 45.0 + f2 * (-44.0 / 945.0))));
  return (y - x) / log(y / x);
}
__device__ __forceinline__ double inv_ln_mean_rs(double x, double y, double rs) {
  const double t = (x - y) * rs;
  const double f2 = t * t;
  if (f2 < 1.0e-4) return (2.0 + f2 * (2.0 / 3.0 + f2 * (2.0 / 5.0 + f2 * (2.0 / 7.0)))) * rs;
  return log(y / x) / (y - x);
}

// The means of Chandrashekar's flux for one pair (numerical_flux.hpp:436-500):
// the logarithmic mean of rho, the inverse logarithmic mean of beta and
// 1 / (beta_L + beta_R), with the reference's branch rule for each logarithmic
// mean (series when f^2 = ((x-y)/(x+y))^2 < 1e-4, else (y-x)/log(y/x)).
// Series branches: the mean is (x+y)/2 / (1 + f^2/3 + f^4/5 + f^6/7), taken as
// (x+y)/2 times the reciprocal series 1 - f^2/3 - 4 f^4/45 - 44 f^6/945 (the
// next term, 1147 f^8/14175, is below 1e-17 relative for f^2 < 1e-4), and the
// inverse mean multiplies by 1/(x+y); the reciprocals of the rho and beta sums
// come from one division, so the series branches of a pair need one division
// instead of four.
__device__ __forceinline__ void chandrashekar_means(double rL, double rR, double bL, double bR,
                                                    double& rho_mean, double& inv_beta_mean,
                                                    double& inv_beta_sum) {
  const double s = rL + rR, sb = bL + bR;
  double rs, rb;
  two_reciprocals(s, sb, rs, rb);
  rho_mean = ln_mean_rs(rL, rR, s, rs);
  inv_beta_mean = inv_ln_mean_rs(bL, bR, rb);
  inv_beta_sum = rb;
}

// Node preparation from conserved variables (rho, m_1..m_DIM, E).
template <int DIM, int VF>
__device__ __forceinline__ NodeState<DIM> prepare_node(const double* u,
                                                       double gamma) {
  NodeState<DIM> s;
  s.rho = u[0];
  const double inv_rho = 1.0 / u[0];
  s.inv_rho = inv_rho;
  double sq = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    s.v[d] = u[1 + d] * inv_rho;
    sq += s.v[d] * s.v[d];
  }
  s.kin = 0.5 * sq;
  s.p = (gamma - 1.0) * (u[DIM + 1] - 0.5 * u[0] * sq);
  if (VF == VF_KENNEDY_GRUBER) {
    s.beta = u[DIM + 1] * inv_rho;
  } else {
    s.beta = 0.5 * u[0] / s.p;
  }
  return s;
}

// Two-point volume flux f(L, R; normal) -> f[DIM + 2].
template <int DIM, int VF>
__device__ __forceinline__ void volume_flux(const NodeState<DIM>& L,
                                            const NodeState<DIM>& R,
                                            const double* n, double inv_gm1,
                                            double* f) {
  double vnL = 0.0, vnR = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    vnL += L.v[d] * n[d];
    vnR += R.v[d] * n[d];
  }
  if (VF == VF_CHANDRASHEKAR) {
    // numerical_flux.hpp:436-500: rho_mean = ln(rho), beta_mean = ln(beta),
    // p_mean = 0.5 rho_avg / beta_avg = 0.5 (rhoL+rhoR) / (betaL+betaR).
    double rho_mean, inv_beta_mean, inv_beta_sum;
    chandrashekar_means(L.rho, R.rho, L.beta, R.beta, rho_mean, inv_beta_mean, inv_beta_sum);
    const double p_mean = 0.5 * (L.rho + R.rho) * inv_beta_sum;
    const double f1 = rho_mean * 0.5 * (vnL + vnR);
    f[0] = f1;
    double fe = f1 * 0.5 * (inv_gm1 * inv_beta_mean - (L.kin + R.kin));
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      const double va = 0.5 * (L.v[d] + R.v[d]);
      const double fm = f1 * va + p_mean * n[d];
      f[1 + d] = fm;
      fe += fm * va;
    }
    f[DIM + 1] = fe;
  } else if (VF == VF_RANOCHA) {
    // the reciprocals of the two sums of the logarithmic means from one division
    const double s1 = L.rho + R.rho;
    const double x2 = L.rho * R.p, y2 = R.rho * L.p, s2 = x2 + y2;
    double r1, r2;
    two_reciprocals(s1, s2, r1, r2);
    const double rho_mean = ln_mean_rs(L.rho, R.rho, s1, r1);
    const double inv_rho_p_mean = L.p * R.p * inv_ln_mean_rs(x2, y2, r2);
    const double p_avg = 0.5 * (L.p + R.p);
    double vLvR = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) vLvR += L.v[d] * R.v[d];
    const double f1 = rho_mean * 0.5 * (vnL + vnR);
    f[0] = f1;
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      f[1 + d] = f1 * (0.5 * (L.v[d] + R.v[d])) + p_avg * n[d];
    f[DIM + 1] = f1 * (0.5 * vLvR + inv_rho_p_mean * inv_gm1) +
                 0.5 * (L.p * vnR + R.p * vnL);
  } else {  // Kennedy-Gruber
    const double rho_avg = 0.5 * (L.rho + R.rho);
    const double e_avg = 0.5 * (L.beta + R.beta);
    const double p_avg = 0.5 * (L.p + R.p);
    double vn_avg = 0.0;
    double va[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      va[d] = 0.5 * (L.v[d] + R.v[d]);
      vn_avg += va[d] * n[d];
    }
    const double f1 = rho_avg * vn_avg;
    f[0] = f1;
#pragma unroll
    for (int d = 0; d < DIM; ++d) f[1 + d] = f1 * va[d] + p_avg * n[d];
    f[DIM + 1] = (rho_avg * e_avg + p_avg) * vn_avg;
  }
}

// Primitive data used by the surface fluxes.
template <int DIM>
struct FaceState {
  double u[DIM + 2];
  double v[DIM];
  double p;
  double a2;  // squared sound speed gamma p / rho
};

// (L, R) = first ? (a, b) : (b, a), field by field with selects, so that
// one flux evaluation serves both argument orders.
template <int DIM>
__device__ __forceinline__ void order_states(bool first, const FaceState<DIM>& a,
                                             const FaceState<DIM>& b, FaceState<DIM>& L,
                                             FaceState<DIM>& R) {
#pragma unroll
  for (int q = 0; q < DIM + 2; ++q) {
    L.u[q] = first ? a.u[q] : b.u[q];
    R.u[q] = first ? b.u[q] : a.u[q];
  }
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    L.v[d] = first ? a.v[d] : b.v[d];
    R.v[d] = first ? b.v[d] : a.v[d];
  }
  L.p = first ? a.p : b.p;
  R.p = first ? b.p : a.p;
  L.a2 = first ? a.a2 : b.a2;
  R.a2 = first ? b.a2 : a.a2;
}

template <int DIM>
__device__ __forceinline__ FaceState<DIM> prepare_face(const double* u,
                                                       double gamma) {
  FaceState<DIM> s;
#pragma unroll
  for (int q = 0; q < DIM + 2; ++q) s.u[q] = u[q];
  const double inv_rho = 1.0 / u[0];
  double sq = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    s.v[d] = u[1 + d] * inv_rho;
    sq += s.v[d] * s.v[d];
  }
  s.p = (gamma - 1.0) * (u[DIM + 1] - 0.5 * u[0] * sq);
  s.a2 = gamma * s.p * inv_rho;
  return s;
}

// Local Lax-Friedrichs flux (numerical_flux.hpp:198-228 with the wave speed
// of compressible_euler2D.hpp:70-109): 0.5 (F_L + F_R).n - 0.5 lambda (uR-uL),
// lambda = max|v.n| + max(a_L, a_R) |n|, evaluated as
// max|v.n| + sqrt(max(a_L^2, a_R^2) |n|^2): the same value (to rounding) with
// one square root per evaluation instead of three (two sound speeds, |n|).
template <int DIM>
__device__ __forceinline__ void llf_flux(const FaceState<DIM>& L,
                                         const FaceState<DIM>& R,
                                         const double* n, double* f) {
  double vnL = 0.0, vnR = 0.0, nn = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    vnL += L.v[d] * n[d];
    vnR += R.v[d] * n[d];
    nn += n[d] * n[d];
  }
  const double lam = fmax(fabs(vnL), fabs(vnR)) + sqrt(fmax(L.a2, R.a2) * nn);
  f[0] = 0.5 * (L.u[0] * vnL + R.u[0] * vnR) - 0.5 * lam * (R.u[0] - L.u[0]);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const double fl = L.u[1 + d] * vnL + L.p * n[d];
    const double fr = R.u[1 + d] * vnR + R.p * n[d];
    f[1 + d] = 0.5 * (fl + fr) - 0.5 * lam * (R.u[1 + d] - L.u[1 + d]);
  }
  f[DIM + 1] = 0.5 * (vnL * (L.u[DIM + 1] + L.p) + vnR * (R.u[DIM + 1] + R.p)) -
               0.5 * lam * (R.u[DIM + 1] - L.u[DIM + 1]);
}

// Normal-rotated HLLC for 2D Euler: the reference's 1D HLLC
// (numerical_flux.hpp:283-378) in the face frame, tangential momentum carried
// passively, rotated back and scaled by |n|.  Quotients by the same quantity
// share one reciprocal, and pairs of reciprocals one division
// (two_reciprocals): four divisions per call instead of sixteen.
__device__ __forceinline__ void hllc_flux_2d(const FaceState<2>& Ls,
                                             const FaceState<2>& Rs,
                                             const double* n, double gamma,
                                             double* f) {
  const double nn = sqrt(n[0] * n[0] + n[1] * n[1]);
  const double rL = Ls.u[0], rR = Rs.u[0];
  const double srL = sqrt(rL), srR = sqrt(rR);
  double inn, issum, irL, irR;
  two_reciprocals(nn, srL + srR, inn, issum);
  two_reciprocals(rL, rR, irL, irR);
  const double nx = n[0] * inn, ny = n[1] * inn;
  const double mnL = Ls.u[1] * nx + Ls.u[2] * ny;
  const double mtL = -Ls.u[1] * ny + Ls.u[2] * nx;
  const double mnR = Rs.u[1] * nx + Rs.u[2] * ny;
  const double mtR = -Rs.u[1] * ny + Rs.u[2] * nx;
  const double EL = Ls.u[3], ER = Rs.u[3];
  const double vL = mnL * irL, vR = mnR * irR;
  const double wL = mtL * irL, wR = mtR * irR;
  const double pL = (gamma - 1.0) * (EL - 0.5 * rL * (vL * vL + wL * wL));
  const double pR = (gamma - 1.0) * (ER - 0.5 * rR * (vR * vR + wR * wR));
  const double cL = sqrt(gamma * pL * irL);
  const double cR = sqrt(gamma * pR * irR);
  const double v_roe = (srL * vL + srR * vR) * issum;
  const double w_roe = (srL * wL + srR * wR) * issum;
  const double ekin_roe = 0.5 * (v_roe * v_roe + w_roe * w_roe);
  const double HL = (EL + pL) * irL;
  const double HR = (ER + pR) * irR;
  const double H_roe = (srL * HL + srR * HR) * issum;
  const double c_roe = sqrt((gamma - 1.0) * (H_roe - ekin_roe));
  const double SL = fmin(vL - cL, v_roe - c_roe);
  const double SR = fmax(vR + cR, v_roe + c_roe);
  double g[4];
  if (SL >= 0.0) {
    g[0] = mnL; g[1] = mnL * vL + pL; g[2] = mnL * wL; g[3] = vL * (EL + pL);
  } else if (SR <= 0.0) {
    g[0] = mnR; g[1] = mnR * vR + pR; g[2] = mnR * wR; g[3] = vR * (ER + pR);
  } else {
    const double sMuL = SL - vL, sMuR = SR - vR;
    const double SStar = (pR - pL + rL * vL * sMuL - rR * vR * sMuR) /
                         (rL * sMuL - rR * sMuR);
    // star state of the side that SStar selects: the same expressions for
    // both sides on selected operands, so the lanes of a warp that fall on
    // different sides still run one branch
    const bool l = SStar >= 0.0;
    const double r = l ? rL : rR, sMu = l ? sMuL : sMuR, S = l ? SL : SR;
    const double v = l ? vL : vR, w = l ? wL : wR, E = l ? EL : ER, p = l ? pL : pR;
    const double mn = l ? mnL : mnR, mt = l ? mtL : mtR, ir = l ? irL : irR;
    // S - SStar and S - v are nonzero in the star region (S_L < v_L, S_R > v_R)
    double idS, isMu;
    two_reciprocals(S - SStar, sMu, idS, isMu);
    const double dS = r * sMu * idS;
    const double eS = E * ir + (SStar - v) * (SStar + p * ir * isMu);
    g[0] = mn + S * (dS - r);
    g[1] = (mn * v + p) + S * (dS * SStar - mn);
    g[2] = mn * w + S * (dS * w - mt);
    g[3] = v * (E + p) + S * (dS * eS - E);
  }
  f[0] = g[0] * nn;
  f[1] = (g[1] * nx - g[2] * ny) * nn;
  f[2] = (g[1] * ny + g[2] * nx) * nn;
  f[3] = g[3] * nn;
}

template <int DIM, int SF>
__device__ __forceinline__ void surface_flux(const FaceState<DIM>& L,
                                             const FaceState<DIM>& R,
                                             const double* n, double gamma,
                                             double* f) {
  if constexpr (SF == SF_HLLC && DIM == 2) {
    hllc_flux_2d(L, R, n, gamma, f);
  } else {
    llf_flux<DIM>(L, R, n, f);
  }
}

}  // namespace dgsem

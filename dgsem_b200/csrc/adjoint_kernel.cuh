// Discrete adjoint of the 2D DGSEM right-hand side on periodic meshes:
// vector-Jacobian products  VJP(u; w) = (dR/du)^T w  for
//   R(u) = -1/J [ split-form volume (Chandrashekar) + LLF surface + lifting
//                 (+ Navier-Stokes BR1 viscous terms) ]
// i.e. the transpose of the linearisation of exactly the arithmetic of the
// forward kernels (stage_kernel.cuh, br1_kernel.cuh); the forward operators
// restate structured_solver.hpp:466-480, volume_flux.hpp:221-294,
// surface_flux.hpp:45-127, surface_integral.hpp:35-80, jacobian.hpp:76-101,
// parabolic_gradient.hpp:480-818 and parabolic_viscous.hpp:343-592.
//
// Notation: w_hat = -(1/J) w per node (the cotangent of the unscaled du).
//
// Two kernels, one thread per node, EPB elements per block:
//   adj_viscous_kernel (Navier-Stokes only): cotangent of the stored -F_v
//     (transposed Dhat volume term and one-sided interface flux), then of the
//     lifted gradient G; writes per node X~ = sum_d Ja^0_d G~_d / J and
//     Y~ = sum_d Ja^1_d G~_d / J (the cotangents of the reference-space
//     gradient) and the direct velocity cotangents of the energy row.
//   adj_main_kernel: transposed split-form pair loop (per node, every
//     partner on its two lines), transposed LLF interface fluxes on the
//     element's faces, transposed BR1 gradient (Dhat^T and face averages),
//     chain rule to conserved variables, and the linear epilogue
//       out = x0 X + x1 Y + b w + c VJP
//     used by the SSPRK3 adjoint stages.
// Every contribution is gathered by the node that owns it: no atomics, and
// the result is deterministic.
#pragma once

#include "br1_kernel.cuh"

namespace dgsem {

template <int N>
struct AdjArgs {
  const double* u;     // state at which the Jacobian is taken
  const double* w;     // cotangent input
  const double* grad;  // forward BR1 gradient of u [E][4][2][ND] (Navier-Stokes)
  double* xy;          // Navier-Stokes: X~, Y~ per node [E][4][2][ND]
  double* qdir;        // Navier-Stokes: direct velocity cotangents [E][2][ND]
  double* out;         // x0 X + x1 Y + b w + c VJP (may alias X)
  const double* X;
  const double* Y;
  double x0, x1, b, c;
  int cells[2];
  int nelem;
  double gamma, inv_gm1, mu, kappa;
  DeviceTables tab;
  BasisConst<N> basis;
};

// ---- geometry of 2D separable tables ---------------------------------------
template <int N>
__device__ __forceinline__ double adj_ja(const DeviceTables& t, int a, int c, int ie, int je,
                                         int node) {
  const int eo = c == 0 ? je : ie;  // element index over the axes other than c
  return __ldg(t.ja[a][c] + (int64_t)eo * (N * N) + node);
}

template <int N>
__device__ __forceinline__ double adj_inv_j(const DeviceTables& t, int ie, int je, int node) {
  return 1.0 / (__ldg(t.jdiag[0] + ie * N + node % N) * __ldg(t.jdiag[1] + je * N + node / N));
}

// ---- derivatives of the logarithmic mean (same branch rule as chandrashekar_means);
// rs = 1 / (x + y) is given.  Series branch: with P = 2 (1 + f^2/3 + f^4/5 +
// f^6/7), 1/P is the reciprocal series of chandrashekar_means; the log
// branch shares 1/x and 1/log(y/x) (or 1/(y-x)) between its quotients.
// mean(x, y) and d mean / dx
__device__ __forceinline__ void ln_mean_dx(double x, double y, double rs, double& m,
                                           double& dm) {
  const double s = x + y;
  const double t = (x - y) * rs;
  const double f2 = t * t;
  if (f2 < 1.0e-4) {
    const double iP =
        0.5 * (1.0 + f2 * (-1.0 / 3.0 + f2 * (-4.0 / 45.0 + f2 * (-44.0 / 945.0))));
    const double dP = 2.0 / 3.0 + f2 * (4.0 / 5.0 + f2 * (6.0 / 7.0));
    const double df2 = 4.0 * t * y * rs * rs;
    m = s * iP;
    dm = iP - s * dP * df2 * iP * iP;
  } else {
    double ix, ilg;
    const double lg = log(y / x);
    two_reciprocals(x, lg, ix, ilg);
    m = (y - x) * ilg;
    dm = (-lg + (y - x) * ix) * ilg * ilg;
  }
}

// 1 / mean(x, y) and its x-derivative
__device__ __forceinline__ void inv_ln_mean_dx(double x, double y, double rs, double& im,
                                               double& dim) {
  const double t = (x - y) * rs;
  const double f2 = t * t;
  if (f2 < 1.0e-4) {
    const double P = 2.0 + f2 * (2.0 / 3.0 + f2 * (2.0 / 5.0 + f2 * (2.0 / 7.0)));
    const double dP = 2.0 / 3.0 + f2 * (4.0 / 5.0 + f2 * (6.0 / 7.0));
    const double df2 = 4.0 * t * y * rs * rs;
    im = P * rs;
    dim = dP * df2 * rs - P * rs * rs;
  } else {
    const double lg = log(y / x);
    const double d = y - x;
    double ix, id;
    two_reciprocals(x, d, ix, id);
    im = lg * id;
    dim = (lg - d * ix) * id * id;
  }
}

// Cotangent of the Chandrashekar flux f(L, R; n) (numerical_flux.hpp:436-500)
// with respect to the LEFT node's primitives: accumulates into rb (rho),
// vb (velocity), bb (beta = rho / 2p) and kb (|v|^2 / 2).  The flux is
// symmetric in (L, R), so the right node's cotangent is this function with
// the roles swapped.
__device__ __forceinline__ void ec_flux_vjp_left(const NodeState<2>& L, const NodeState<2>& R,
                                                 const double* n, const double* c,
                                                 double igm1, double& rb, double* vb,
                                                 double& bb, double& kb) {
  const double vnL = L.v[0] * n[0] + L.v[1] * n[1];
  const double vnR = R.v[0] * n[0] + R.v[1] * n[1];
  double rho_m, drho_m, ib, dib, rrs, rbs;
  const double rsum = L.rho + R.rho, bsum = L.beta + R.beta;
  two_reciprocals(rsum, bsum, rrs, rbs);
  ln_mean_dx(L.rho, R.rho, rrs, rho_m, drho_m);
  inv_ln_mean_dx(L.beta, R.beta, rbs, ib, dib);
  const double pm = 0.5 * rsum * rbs;
  const double f1 = rho_m * 0.5 * (vnL + vnR);
  const double va[2] = {0.5 * (L.v[0] + R.v[0]), 0.5 * (L.v[1] + R.v[1])};
  const double fm[2] = {f1 * va[0] + pm * n[0], f1 * va[1] + pm * n[1]};
  const double A = 0.5 * (igm1 * ib - (L.kin + R.kin));
  const double fmb[2] = {c[1] + c[3] * va[0], c[2] + c[3] * va[1]};
  const double f1b = c[0] + c[3] * A + fmb[0] * va[0] + fmb[1] * va[1];
  const double pmb = fmb[0] * n[0] + fmb[1] * n[1];
  const double Ab = c[3] * f1;
  const double vnb = f1b * rho_m * 0.5;
#pragma unroll
  for (int d = 0; d < 2; ++d) vb[d] += 0.5 * (c[3] * fm[d] + fmb[d] * f1) + vnb * n[d];
  kb += -0.5 * Ab;
  rb += pmb * 0.5 * rbs + f1b * 0.5 * (vnL + vnR) * drho_m;
  bb += -pmb * pm * rbs + 0.5 * igm1 * Ab * dib;
}

// Chain rule from primitive cotangents (rho, v, p) to conserved ones, with
// v = m / rho and p = (gamma - 1)(E - |m|^2 / (2 rho)).
__device__ __forceinline__ void prim_to_cons_vjp(const double* u, double gm1, double rb,
                                                 const double* vb, double pb, double* ub,
                                                 double inv_rho) {
  const double v0 = u[1] * inv_rho, v1 = u[2] * inv_rho;
  ub[0] += rb + gm1 * pb * 0.5 * (v0 * v0 + v1 * v1) - (vb[0] * v0 + vb[1] * v1) * inv_rho;
  ub[1] += vb[0] * inv_rho - gm1 * pb * v0;
  ub[2] += vb[1] * inv_rho - gm1 * pb * v1;
  ub[3] += gm1 * pb;
}

// Cotangent of the LLF flux (numerical_flux.hpp:198-228) with respect to one
// side's conserved state (own_left selects L or R).  The max() of the wave
// speed passes its cotangent to the side that attains it (L on ties), so the
// two sides' cotangents partition the one-sided derivative consistently.
__device__ __forceinline__ void llf_vjp(const FaceState<2>& L, const FaceState<2>& R,
                                        const double* n, const double* c, bool own_left,
                                        double gamma, double* ub) {
  const double vnL = L.v[0] * n[0] + L.v[1] * n[1];
  const double vnR = R.v[0] * n[0] + R.v[1] * n[1];
  const double sn = sqrt(n[0] * n[0] + n[1] * n[1]);
  // sound speeds from the squared ones the forward stores; lambda is the
  // forward's max|v.n| + sqrt(max(a^2) |n|^2) = max|v.n| + max(a) |n|
  const double aL = sqrt(L.a2), aR = sqrt(R.a2);
  const double lam = fmax(fabs(vnL), fabs(vnR)) + fmax(aL, aR) * sn;
  const FaceState<2>& O = own_left ? L : R;
  const double vnO = own_left ? vnL : vnR;
  double uo[4] = {0.0, 0.0, 0.0, 0.0};
  // 0.5 G_own . c with G = (m.n, m_d vn + p n_d, vn (E + p))
  double vnb = 0.5 * (c[0] * O.u[0] + c[1] * O.u[1] + c[2] * O.u[2] + c[3] * (O.u[3] + O.p));
  double pb = 0.5 * (c[1] * n[0] + c[2] * n[1] + c[3] * vnO);
  uo[0] += 0.5 * c[0] * vnO;
  uo[1] += 0.5 * c[1] * vnO;
  uo[2] += 0.5 * c[2] * vnO;
  uo[3] += 0.5 * c[3] * vnO;
  // -0.5 lam (uR - uL)
  const double sgn = own_left ? 0.5 * lam : -0.5 * lam;
#pragma unroll
  for (int q = 0; q < 4; ++q) uo[q] += sgn * c[q];
  const double lamb = -0.5 * (c[0] * (R.u[0] - L.u[0]) + c[1] * (R.u[1] - L.u[1]) +
                              c[2] * (R.u[2] - L.u[2]) + c[3] * (R.u[3] - L.u[3]));
  const bool own_v = own_left ? (fabs(vnL) >= fabs(vnR)) : (fabs(vnR) > fabs(vnL));
  const bool own_a = own_left ? (aL >= aR) : (aR > aL);
  const double aO = own_left ? aL : aR;
  if (own_v) vnb += lamb * (vnO >= 0.0 ? 1.0 : -1.0);
  double rb = 0.0;
  double iaO, iuO;  // 1 / a and 1 / rho of the own side
  two_reciprocals(aO, O.u[0], iaO, iuO);
  if (own_a) {
    const double ab = lamb * sn;  // a = sqrt(gamma p / rho)
    pb += ab * gamma * 0.5 * iaO * iuO;
    rb += -ab * aO * 0.5 * iuO;
  }
  const double vb[2] = {vnb * n[0], vnb * n[1]};
  prim_to_cons_vjp(O.u, gamma - 1.0, rb, vb, pb, uo, iuO);
#pragma unroll
  for (int q = 0; q < 4; ++q) ub[q] += uo[q];
}

template <int N>
__device__ __forceinline__ void load_w_hat(const AdjArgs<N>& p, int ie, int je, int node,
                                           double* wh) {
  const int e = ie + p.cells[0] * je;
  const double s = -adj_inv_j<N>(p.tab, ie, je, node);
#pragma unroll
  for (int q = 0; q < 4; ++q) wh[q] = s * __ldg(p.w + ((int64_t)e * 4 + q) * (N * N) + node);
}

// ---- Navier-Stokes: cotangents of -F_v and of the lifted gradient ----------
template <int N, int EPB>
__global__ void __launch_bounds__(EPB* N* N) adj_viscous_kernel(const AdjArgs<N> p) {
  constexpr int ND = N * N;
  __shared__ double ws[EPB][4][ND];
  stage_dependency_sync();  // programmatic dependent launch (see launch_stage_kernel)
  const int tid = threadIdx.x;
  const int el = tid / ND, node = tid % ND;
  const int e = (int)blockIdx.x * EPB + el;
  const bool active = e < p.nelem;
  const int nx = p.cells[0], ny = p.cells[1];
  const int ie = active ? e % nx : 0, je = active ? e / nx : 0;
  if (active) {
    double wh[4];
    load_w_hat<N>(p, ie, je, node, wh);
#pragma unroll
    for (int q = 0; q < 4; ++q) ws[el][q][node] = wh[q];
  }
  __syncthreads();
  if (!active) return;
  const int i = node % N, j = node / N;
  const double lL = p.basis.lhat_l0, lR = p.basis.lhat_rN;
  double X[4], Y[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    double sx = 0.0, sy = 0.0;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      sx += p.basis.Dhat[k][i] * ws[el][q][j * N + k];
      sy += p.basis.Dhat[k][j] * ws[el][q][k * N + i];
    }
    X[q] = sx;
    Y[q] = sy;
  }
  if (i == 0) {  // one-sided interface flux of this element's x-low face
    double wn[4];
    load_w_hat<N>(p, (ie + nx - 1) % nx, je, (N - 1) + N * j, wn);
#pragma unroll
    for (int q = 0; q < 4; ++q) X[q] += -lL * ws[el][q][node] + lR * wn[q];
  }
  if (j == 0) {
    double wn[4];
    load_w_hat<N>(p, ie, (je + ny - 1) % ny, i + N * (N - 1), wn);
#pragma unroll
    for (int q = 0; q < 4; ++q) Y[q] += -lL * ws[el][q][node] + lR * wn[q];
  }
  const double ja00 = adj_ja<N>(p.tab, 0, 0, ie, je, node);
  const double ja01 = adj_ja<N>(p.tab, 0, 1, ie, je, node);
  const double ja10 = adj_ja<N>(p.tab, 1, 0, ie, je, node);
  const double ja11 = adj_ja<N>(p.tab, 1, 1, ie, je, node);
  // cotangent of the stored -F_v, times -mu:  s = -mu * (-F_v)bar
  double sx[4], sy[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    sx[q] = -p.mu * (ja00 * X[q] + ja10 * Y[q]);
    sy[q] = -p.mu * (ja01 * X[q] + ja11 * Y[q]);
  }
  double u[4], q[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) u[v] = __ldg(p.u + ((int64_t)e * 4 + v) * ND + node);
  ns_gradient_variables(u, p.gamma, q);
  double gx[4], gy[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    gx[v] = __ldg(p.grad + (((int64_t)e * 4 + v) * 2 + 0) * ND + node);
    gy[v] = __ldg(p.grad + (((int64_t)e * 4 + v) * 2 + 1) * ND + node);
  }
  const double tau11 = (4.0 * gx[1] - 2.0 * gy[2]) * (1.0 / 3.0);
  const double tau22 = (4.0 * gy[2] - 2.0 * gx[1]) * (1.0 / 3.0);
  const double tau12 = gy[1] + gx[2];
  const double t11b = sx[1] + sx[3] * q[1];
  const double t12b = sx[2] + sx[3] * q[2] + sy[1] + sy[3] * q[1];
  const double t22b = sy[2] + sy[3] * q[2];
  const double v1b = sx[3] * tau11 + sy[3] * tau12;
  const double v2b = sx[3] * tau12 + sy[3] * tau22;
  double Gb[4][2];
  Gb[0][0] = 0.0;
  Gb[0][1] = 0.0;
  Gb[1][0] = (4.0 * t11b - 2.0 * t22b) * (1.0 / 3.0);
  Gb[1][1] = t12b;
  Gb[2][0] = t12b;
  Gb[2][1] = (4.0 * t22b - 2.0 * t11b) * (1.0 / 3.0);
  Gb[3][0] = p.kappa * sx[3];
  Gb[3][1] = p.kappa * sy[3];
  const double ij = adj_inv_j<N>(p.tab, ie, je, node);
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    p.xy[(((int64_t)e * 4 + v) * 2 + 0) * ND + node] = (ja00 * Gb[v][0] + ja01 * Gb[v][1]) * ij;
    p.xy[(((int64_t)e * 4 + v) * 2 + 1) * ND + node] = (ja10 * Gb[v][0] + ja11 * Gb[v][1]) * ij;
  }
  p.qdir[((int64_t)e * 2 + 0) * ND + node] = v1b;
  p.qdir[((int64_t)e * 2 + 1) * ND + node] = v2b;
}

// ---- inviscid cotangents, transposed BR1, chain rule, epilogue -------------
template <int N, bool NS, int EPB>
__global__ void __launch_bounds__(EPB* N* N) adj_main_kernel(const AdjArgs<N> p) {
  constexpr int ND = N * N;
  constexpr int NXY = NS ? 8 : 1;
  __shared__ double ws[EPB][4][ND];
  __shared__ double ps[EPB][5][ND];  // rho, v1, v2, beta, kin
  __shared__ double xys[EPB][NXY][ND];
  stage_dependency_sync();  // programmatic dependent launch (see launch_stage_kernel)
  const int tid = threadIdx.x;
  const int el = tid / ND, node = tid % ND;
  const int e = (int)blockIdx.x * EPB + el;
  const bool active = e < p.nelem;
  const int nx = p.cells[0], ny = p.cells[1];
  const int ie = active ? e % nx : 0, je = active ? e / nx : 0;
  double u[4] = {1.0, 0.0, 0.0, 1.0};
  if (active) {
    double wh[4];
    load_w_hat<N>(p, ie, je, node, wh);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      ws[el][q][node] = wh[q];
      u[q] = __ldg(p.u + ((int64_t)e * 4 + q) * ND + node);
    }
    const NodeState<2> s = prepare_node<2, VF_CHANDRASHEKAR>(u, p.gamma);
    ps[el][0][node] = s.rho;
    ps[el][1][node] = s.v[0];
    ps[el][2][node] = s.v[1];
    ps[el][3][node] = s.beta;
    ps[el][4][node] = s.kin;
    if constexpr (NS) {
#pragma unroll
      for (int k = 0; k < 8; ++k) xys[el][k][node] = __ldg(p.xy + ((int64_t)e * 8 + k) * ND + node);
    }
  }
  __syncthreads();
  if (!active) return;
  const int i = node % N, j = node / N;
  const double lL = p.basis.lhat_l0, lR = p.basis.lhat_rN;
  const double gm1 = p.gamma - 1.0;

  auto node_state = [&](int m) {
    NodeState<2> s;
    s.rho = ps[el][0][m];
    s.v[0] = ps[el][1][m];
    s.v[1] = ps[el][2][m];
    s.beta = ps[el][3][m];
    s.kin = ps[el][4][m];
    s.p = 0.0;
    return s;
  };
  const NodeState<2> own = node_state(node);

  // -- split-form volume term: every partner on the node's x and y lines
  double rb = 0.0, vb[2] = {0.0, 0.0}, bb = 0.0, kb = 0.0;
#pragma unroll
  for (int dir = 0; dir < 2; ++dir) {
    const int pos = dir == 0 ? i : j;
    const double n0 = adj_ja<N>(p.tab, dir, 0, ie, je, node);
    const double n1 = adj_ja<N>(p.tab, dir, 1, ie, je, node);
#pragma unroll
    for (int k = 0; k < N; ++k) {
      if (k == pos) continue;
      const int mk = dir == 0 ? j * N + k : k * N + i;
      const double nrm[2] = {0.5 * (n0 + adj_ja<N>(p.tab, dir, 0, ie, je, mk)),
                             0.5 * (n1 + adj_ja<N>(p.tab, dir, 1, ie, je, mk))};
      const double dik = p.basis.Dsplit[pos][k], dki = p.basis.Dsplit[k][pos];
      double c[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) c[q] = dik * ws[el][q][node] + dki * ws[el][q][mk];
      ec_flux_vjp_left(own, node_state(mk), nrm, c, p.inv_gm1, rb, vb, bb, kb);
    }
  }
  double ub[4] = {0.0, 0.0, 0.0, 0.0};
  const FaceState<2> fo = prepare_face<2>(u, p.gamma);
  {
    // beta = rho / (2 p), kin = |v|^2 / 2
    double ip, iu;
    two_reciprocals(fo.p, u[0], ip, iu);
    const double rbt = rb + bb * 0.5 * ip;
    const double pb = -bb * own.beta * ip;
    const double vbt[2] = {vb[0] + kb * own.v[0], vb[1] + kb * own.v[1]};
    prim_to_cons_vjp(u, gm1, rbt, vbt, pb, ub, iu);
  }

  // -- LLF interface fluxes of the element's faces through this node
#pragma unroll
  for (int dir = 0; dir < 2; ++dir) {
    const int pos = dir == 0 ? i : j;
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      if ((side == 0 && pos != 0) || (side == 1 && pos != N - 1)) continue;
      const int nie = dir == 0 ? (side ? (ie + 1) % nx : (ie + nx - 1) % nx) : ie;
      const int nje = dir == 1 ? (side ? (je + 1) % ny : (je + ny - 1) % ny) : je;
      const int ne = nie + nx * nje;
      const int nb_node = dir == 0 ? ((side ? 0 : N - 1) + N * j) : (i + N * (side ? 0 : N - 1));
      double un[4], wn[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) un[q] = __ldg(p.u + ((int64_t)ne * 4 + q) * ND + nb_node);
      load_w_hat<N>(p, nie, nje, nb_node, wn);
      const FaceState<2> fn = prepare_face<2>(un, p.gamma);
      double nrm[2], c[4];
      if (side == 0) {  // face owned by this element (left state = neighbour)
        nrm[0] = adj_ja<N>(p.tab, dir, 0, ie, je, node);
        nrm[1] = adj_ja<N>(p.tab, dir, 1, ie, je, node);
#pragma unroll
        for (int q = 0; q < 4; ++q) c[q] = -lL * ws[el][q][node] + lR * wn[q];
        llf_vjp(fn, fo, nrm, c, false, p.gamma, ub);
      } else {  // face owned by the high-side neighbour (left state = this node)
        nrm[0] = adj_ja<N>(p.tab, dir, 0, nie, nje, nb_node);
        nrm[1] = adj_ja<N>(p.tab, dir, 1, nie, nje, nb_node);
#pragma unroll
        for (int q = 0; q < 4; ++q) c[q] = -lL * wn[q] + lR * ws[el][q][node];
        llf_vjp(fo, fn, nrm, c, true, p.gamma, ub);
      }
    }
  }

  // -- transposed BR1 gradient and the direct velocity cotangents
  if constexpr (NS) {
    double qb[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < N; ++k) {
        s += p.basis.Dhat[k][i] * xys[el][v * 2 + 0][j * N + k];
        s += p.basis.Dhat[k][j] * xys[el][v * 2 + 1][k * N + i];
      }
      qb[v] = s;
    }
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
      const int pos = dir == 0 ? i : j;
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        if ((side == 0 && pos != 0) || (side == 1 && pos != N - 1)) continue;
        const int nie = dir == 0 ? (side ? (ie + 1) % nx : (ie + nx - 1) % nx) : ie;
        const int nje = dir == 1 ? (side ? (je + 1) % ny : (je + ny - 1) % ny) : je;
        const int ne = nie + nx * nje;
        const int nb_node = dir == 0 ? ((side ? 0 : N - 1) + N * j) : (i + N * (side ? 0 : N - 1));
        // q^ = (q_low + q_high) / 2 lifted into both elements' face nodes
        const double own_f = side ? lR : -lL;
        const double nb_f = side ? -lL : lR;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const double xo = xys[el][v * 2 + dir][node];
          const double xn = __ldg(p.xy + (((int64_t)ne * 4 + v) * 2 + dir) * ND + nb_node);
          qb[v] += 0.5 * (own_f * xo + nb_f * xn);
        }
      }
    }
    qb[1] += __ldg(p.qdir + ((int64_t)e * 2 + 0) * ND + node);
    qb[2] += __ldg(p.qdir + ((int64_t)e * 2 + 1) * ND + node);
    // q = (rho, v1, v2, T = p / rho)
    double qv[4];
    ns_gradient_variables(u, p.gamma, qv);
    const double T = qv[3];
    const double iu = 1.0 / u[0];
    const double rbq = qb[0] - qb[3] * T * iu;
    const double vbq[2] = {qb[1], qb[2]};
    prim_to_cons_vjp(u, gm1, rbq, vbq, qb[3] * iu, ub, iu);
  }

  // -- epilogue
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int64_t gi = ((int64_t)e * 4 + q) * ND + node;
    double val = p.c * ub[q];
    if (p.b != 0.0) val += p.b * __ldg(p.w + gi);
    if (p.x1 != 0.0) val += p.x1 * p.Y[gi];
    if (p.x0 != 0.0) val += p.x0 * p.X[gi];
    p.out[gi] = val;
  }
}

}  // namespace dgsem

// BR1 lifted gradient of the Navier-Stokes gradient variables, one kernel,
// one thread per node: 2D q = (rho, v1, v2, T = p/rho) on periodic meshes or
// with wall faces, 3D q = (rho, v1, v2, v3, T) on periodic meshes (the
// reference's 3D Navier-Stokes runs periodic boxes only).
//   q at nodes                          compressible_navier_stokes2D.hpp:56-69
//   weak-form volume term with Dhat     parabolic_gradient.hpp:509-532
//   transform with Ja                   parabolic_gradient.hpp:573-585
//   interface average q^ = (q- + q+)/2  parabolic_gradient.hpp:620-686
//   lifting with the element's own face normals, then * 1/J
//                                       parabolic_gradient.hpp:712-818
// Output: grad[e][var][dim][node], read by the fused stage kernel for the
// viscous flux: 2D the four variables (rho, v1, v2, T) x 2 directions, 3D the
// four that the viscous flux uses (v1, v2, v3, T; the density gradient is not
// needed) x 3 directions.
#pragma once

#include "stage_kernel.cuh"

namespace dgsem {

__device__ __forceinline__ void ns_gradient_variables(const double* u, double gamma,
                                                      double* q) {
  const double rho = u[0];
  const double inv_rho = 1.0 / rho;
  const double v1 = u[1] * inv_rho;
  const double v2 = u[2] * inv_rho;
  const double p = (gamma - 1.0) * (u[3] - 0.5 * (u[1] * u[1] + u[2] * u[2]) * inv_rho);
  q[0] = rho;
  q[1] = v1;
  q[2] = v2;
  q[3] = p * inv_rho;
}

// Viscous flux -F_v in direction dim (compressible_navier_stokes2D.hpp:71-106;
// the solver stores -F_v, parabolic_viscous.hpp:383-387).  The 1/3 of the
// normal stresses is a multiplication by the rounded constant 1/3 (a
// division by 3 costs a full division sequence per stress).
__device__ __forceinline__ void ns_neg_viscous_flux(const double* q, const double* gx,
                                                    const double* gy, double mu,
                                                    double kappa, int dim, double* f) {
  const double tau11 = (4.0 * gx[1] - 2.0 * gy[2]) * (1.0 / 3.0);
  const double tau22 = (4.0 * gy[2] - 2.0 * gx[1]) * (1.0 / 3.0);
  const double tau12 = gy[1] + gx[2];
  f[0] = -0.0;
  if (dim == 0) {
    f[1] = -(mu * tau11);
    f[2] = -(mu * tau12);
    f[3] = -(mu * (q[1] * tau11 + q[2] * tau12 + kappa * gx[3]));
  } else {
    f[1] = -(mu * tau12);
    f[2] = -(mu * tau22);
    f[3] = -(mu * (q[1] * tau12 + q[2] * tau22 + kappa * gy[3]));
  }
}

// 3D: q = (rho, v1, v2, v3, T) (compressible_navier_stokes3D.hpp:55-70).
__device__ __forceinline__ void ns_gradient_variables_3d(const double* u, double gamma,
                                                         double* q) {
  const double rho = u[0];
  const double inv_rho = 1.0 / rho;
  const double p =
      (gamma - 1.0) * (u[4] - 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) * inv_rho);
  q[0] = rho;
  q[1] = u[1] * inv_rho;
  q[2] = u[2] * inv_rho;
  q[3] = u[3] * inv_rho;
  q[4] = p * inv_rho;
}

// 3D -F_v in direction dim (compressible_navier_stokes3D.hpp:72-124) from the
// stored gradient g[d][k] of (v1, v2, v3, T) in direction d.
__device__ __forceinline__ void ns_neg_viscous_flux_3d(const double* q, const double (*g)[4],
                                                       double mu, double kappa, int dim,
                                                       double* f) {
  const double dv1dx = g[0][0], dv2dx = g[0][1], dv3dx = g[0][2];
  const double dv1dy = g[1][0], dv2dy = g[1][1], dv3dy = g[1][2];
  const double dv1dz = g[2][0], dv2dz = g[2][1], dv3dz = g[2][2];
  const double tau11 = (4.0 * dv1dx - 2.0 * (dv2dy + dv3dz)) * (1.0 / 3.0);
  const double tau22 = (4.0 * dv2dy - 2.0 * (dv1dx + dv3dz)) * (1.0 / 3.0);
  const double tau33 = (4.0 * dv3dz - 2.0 * (dv1dx + dv2dy)) * (1.0 / 3.0);
  const double tau12 = dv1dy + dv2dx;
  const double tau13 = dv1dz + dv3dx;
  const double tau23 = dv2dz + dv3dy;
  const double t1 = dim == 0 ? tau11 : dim == 1 ? tau12 : tau13;
  const double t2 = dim == 0 ? tau12 : dim == 1 ? tau22 : tau23;
  const double t3 = dim == 0 ? tau13 : dim == 1 ? tau23 : tau33;
  f[0] = -0.0;
  f[1] = -(mu * t1);
  f[2] = -(mu * t2);
  f[3] = -(mu * t3);
  f[4] = -(mu * (q[1] * t1 + q[2] * t2 + q[3] * t3 + kappa * g[dim][3]));
}

template <int N>
struct GradArgs {
  const double* u;
  double* grad;
  int64_t cells[3];
  int64_t nelem;
  double gamma;
  DeviceTables tab;
  BasisConst<N> basis;
  int periodic[3];  // per direction; otherwise the faces carry wall BCs (2D)
  int bc_kind[6];   // BcKind per face (left, right, bottom, top, back, front)
};

template <int N, int EPB>
__global__ void __launch_bounds__(EPB* N* N) br1_gradient_kernel(const GradArgs<N> p) {
  constexpr int ND = N * N, NV = 4, NG = 4;
  __shared__ double qs[EPB][NG][ND];
  stage_dependency_sync();  // programmatic dependent launch (see launch_stage_kernel)
  const int tid = threadIdx.x;
  const int el = tid / ND;
  const int node = tid % ND;
  const int64_t e = (int64_t)blockIdx.x * EPB + el;
  const bool active = e < p.nelem;
  double q[NG] = {0, 0, 0, 0};
  if (active) {
    double u[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) u[v] = __ldg(p.u + (e * NV + v) * ND + node);
    ns_gradient_variables(u, p.gamma, q);
#pragma unroll
    for (int v = 0; v < NG; ++v) qs[el][v][node] = q[v];
  }
  __syncthreads();
  if (!active) return;
  const int i = node % N, j = node / N;
  const ElemIdx<2> ei = elem_coords<2>(e, p.cells);
  double ja[2][2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int c = 0; c < 2; ++c)
      ja[a][c] = __ldg(p.tab.ja[a][c] + eidx_other<2>(ei, c, p.cells) * ND + node);
  double g[NG][2];
#pragma unroll
  for (int v = 0; v < NG; ++v) {
    double gxi = 0.0, geta = 0.0;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      gxi += p.basis.Dhat[i][k] * qs[el][v][j * N + k];
      geta += p.basis.Dhat[j][k] * qs[el][v][k * N + i];
    }
    g[v][0] = ja[0][0] * gxi + ja[1][0] * geta;
    g[v][1] = ja[0][1] * gxi + ja[1][1] * geta;
  }
  // lifting: x faces first, then y faces (parabolic_gradient.hpp:722-744)
#pragma unroll
  for (int dir = 0; dir < 2; ++dir) {
    const int pos = dir == 0 ? i : j;
    if (pos != 0 && pos != N - 1) continue;
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      if ((side == 0 && pos != 0) || (side == 1 && pos != N - 1)) continue;
      ElemIdx<2> nb = ei;
      const int64_t nc = p.cells[dir];
      const int64_t npos = ei.i[dir] + (side ? 1 : -1);
      const double factor = side ? p.basis.lhat_rN : -p.basis.lhat_l0;
      if (!p.periodic[dir] && (npos < 0 || npos >= nc)) {
        // wall: q^ = q of the wall state (navier_stokes_wall_boundary.hpp:
        // 82-99 no-slip: velocity zero; :162-190 slip: the normal velocity
        // removed along the element's own face normal)
        double qw[NG];
#pragma unroll
        for (int v = 0; v < NG; ++v) qw[v] = q[v];
        if (p.bc_kind[2 * dir + side] == BC_NS_NOSLIP_ADIABATIC_WALL) {
          qw[1] = 0.0;
          qw[2] = 0.0;
        } else {
          const double n0 = ja[dir][0], n1 = ja[dir][1];
          const double vn = (qw[1] * n0 + qw[2] * n1) / (n0 * n0 + n1 * n1);
          qw[1] -= vn * n0;
          qw[2] -= vn * n1;
        }
#pragma unroll
        for (int v = 0; v < NG; ++v)
#pragma unroll
          for (int d = 0; d < 2; ++d) g[v][d] += factor * qw[v] * ja[dir][d];
        continue;
      }
      nb.i[dir] = (ei.i[dir] + (side ? 1 : nc - 1)) % nc;
      const int64_t en = elem_linear<2>(nb, p.cells);
      const int nb_node = dir == 0 ? ((side ? 0 : N - 1) + N * j) : (i + N * (side ? 0 : N - 1));
      double un[NV], qn[NG];
#pragma unroll
      for (int v = 0; v < NV; ++v) un[v] = __ldg(p.u + (en * NV + v) * ND + nb_node);
      ns_gradient_variables(un, p.gamma, qn);
#pragma unroll
      for (int v = 0; v < NG; ++v) {
        // q^ = 0.5 (q_left + q_right): the left state is the low-side element's
        const double qhat = side ? 0.5 * (q[v] + qn[v]) : 0.5 * (qn[v] + q[v]);
#pragma unroll
        for (int d = 0; d < 2; ++d) g[v][d] += factor * qhat * ja[dir][d];
      }
    }
  }
  const double inv_j =
      1.0 / (__ldg(p.tab.jdiag[0] + ei.i[0] * N + i) * __ldg(p.tab.jdiag[1] + ei.i[1] * N + j));
#pragma unroll
  for (int v = 0; v < NG; ++v)
#pragma unroll
    for (int d = 0; d < 2; ++d) p.grad[((e * NG + v) * 2 + d) * ND + node] = g[v][d] * inv_j;
}

// 3D periodic meshes: one thread per node; the gradients of (v1, v2, v3, T),
// weak-form volume term with Dhat along xi, eta, zeta
// (parabolic_gradient.hpp:17-95), transform with Ja (:100-154), interface
// averages and lifting on the six faces (:159-307, :312-437), times 1/J.
template <int N, int EPB>
__global__ void __launch_bounds__(EPB* N* N* N) br1_gradient_kernel_3d(const GradArgs<N> p) {
  constexpr int ND = N * N * N, NV = 5, NG = 4;  // stored: v1, v2, v3, T
  __shared__ double qs[EPB][NG][ND];
  stage_dependency_sync();  // programmatic dependent launch (see launch_stage_kernel)
  const int tid = threadIdx.x;
  const int el = tid / ND;
  const int node = tid % ND;
  const int64_t e = (int64_t)blockIdx.x * EPB + el;
  const bool active = e < p.nelem;
  double q[NV] = {0, 0, 0, 0, 0};
  if (active) {
    double u[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) u[v] = __ldg(p.u + (e * NV + v) * ND + node);
    ns_gradient_variables_3d(u, p.gamma, q);
#pragma unroll
    for (int v = 0; v < NG; ++v) qs[el][v][node] = q[1 + v];
  }
  __syncthreads();
  if (!active) return;
  const int pos[3] = {node % N, (node / N) % N, node / (N * N)};
  const int stride[3] = {1, N, N * N};
  const ElemIdx<3> ei = elem_coords<3>(e, p.cells);
  double ja[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      ja[a][c] = __ldg(p.tab.ja[a][c] + eidx_other<3>(ei, c, p.cells) * ND + node);
  double g[NG][3];
#pragma unroll
  for (int v = 0; v < NG; ++v) {
    double gr[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < N; ++k)
        s += p.basis.Dhat[pos[a]][k] * qs[el][v][node + (k - pos[a]) * stride[a]];
      gr[a] = s;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) g[v][d] = ja[0][d] * gr[0] + ja[1][d] * gr[1] + ja[2][d] * gr[2];
  }
  // lifting, direction by direction: q^ = (q_low + q_high) / 2 on each face
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      if (pos[dir] != (side ? N - 1 : 0)) continue;
      ElemIdx<3> nb = ei;
      const int64_t nc = p.cells[dir];
      nb.i[dir] = (ei.i[dir] + (side ? 1 : nc - 1)) % nc;
      const int64_t en = elem_linear<3>(nb, p.cells);
      const int nb_node = node + ((side ? 0 : N - 1) - pos[dir]) * stride[dir];
      double un[NV], qn[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) un[v] = __ldg(p.u + (en * NV + v) * ND + nb_node);
      ns_gradient_variables_3d(un, p.gamma, qn);
      const double factor = side ? p.basis.lhat_rN : -p.basis.lhat_l0;
#pragma unroll
      for (int v = 0; v < NG; ++v) {
        const double qhat = side ? 0.5 * (q[1 + v] + qn[1 + v]) : 0.5 * (qn[1 + v] + q[1 + v]);
#pragma unroll
        for (int d = 0; d < 3; ++d) g[v][d] += factor * qhat * ja[dir][d];
      }
    }
  }
  const double jdet = __ldg(p.tab.jdiag[0] + ei.i[0] * N + pos[0]) *
                      (__ldg(p.tab.jdiag[1] + ei.i[1] * N + pos[1]) *
                       __ldg(p.tab.jdiag[2] + ei.i[2] * N + pos[2]));
  const double inv_j = 1.0 / jdet;
#pragma unroll
  for (int v = 0; v < NG; ++v)
#pragma unroll
    for (int d = 0; d < 3; ++d) p.grad[((e * NG + v) * 3 + d) * ND + node] = g[v][d] * inv_j;
}

}  // namespace dgsem

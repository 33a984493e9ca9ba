// Device geometry initializer for arbitrary (e.g. curvilinear) structured
// meshes: per-node Jacobian matrix, contravariant vectors and inverse Jacobian
// from the node coordinates, with the reference's formulas and operation order
// (StructuredContainerInitializer, containers/data_container.hpp):
//   J(a, c) = sum_m D(i_a, m) x_c(.. m ..)       2D :230-264, 3D :420-478
//   Ja 2D: the adjugate of J                     :268-287
//   Ja 3D: the conservative curl form            :485-659
//   1/J = 1 / det J                              2D :289-312, 3D :661-692
// The reference evaluates these on the host, element by element
// (StructuredElementInitializer::init_elements, :729-772); here one block
// per element, one thread per node, every product and sum rounded explicitly
// (no contraction) so the result equals the reference's host arithmetic bit
// for bit.
#include <cuda_runtime.h>

#include "dgsem_b200.h"
#include "tables.hpp"

namespace {

constexpr int kMaxN = 8;

struct DerivTable {
  double D[kMaxN][kMaxN];
};

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// x[(e*2 + c)*ND + node], node = i + N j
template <int N>
__global__ void geometry_2d_kernel(const double* x, double* ja, double* inv_j, DerivTable T) {
  constexpr int ND = N * N;
  __shared__ double X[2][ND];
  const int e = blockIdx.x, node = threadIdx.x;
  const int i = node % N, j = node / N;
  for (int c = 0; c < 2; ++c) X[c][node] = x[((long long)e * 2 + c) * ND + node];
  __syncthreads();
  double dx_dxi = 0.0, dy_dxi = 0.0, dx_deta = 0.0, dy_deta = 0.0;
  for (int k = 0; k < N; ++k) {
    const int nx = k + N * j, ny = i + N * k;
    dx_dxi = add(dx_dxi, mul(T.D[i][k], X[0][nx]));
    dy_dxi = add(dy_dxi, mul(T.D[i][k], X[1][nx]));
    dx_deta = add(dx_deta, mul(T.D[j][k], X[0][ny]));
    dy_deta = add(dy_deta, mul(T.D[j][k], X[1][ny]));
  }
  // contravariant vectors Ja^a_c (a: reference direction, c: component)
  const long long base = (long long)e * 4 * ND + node;
  ja[base + 0 * ND] = dy_deta;   // (0, 0) =  J(1, 1)
  ja[base + 1 * ND] = -dx_deta;  // (0, 1) = -J(1, 0)
  ja[base + 2 * ND] = -dy_dxi;   // (1, 0) = -J(0, 1)
  ja[base + 3 * ND] = dx_dxi;    // (1, 1) =  J(0, 0)
  inv_j[(long long)e * ND + node] =
      __ddiv_rn(1.0, sub(mul(dx_dxi, dy_deta), mul(dx_deta, dy_dxi)));
}

// x[(e*3 + c)*ND + node], node = i + N (j + N k)
template <int N>
__global__ void geometry_3d_kernel(const double* x, double* ja, double* inv_j, DerivTable T) {
  constexpr int ND = N * N * N;
  __shared__ double X[3][ND];
  __shared__ double J[3][3][ND];  // J(a, c) = d x_c / d xi_a
  const int e = blockIdx.x, node = threadIdx.x;
  const int i = node % N, j = (node / N) % N, k = node / (N * N);
  auto id = [](int a, int b, int c) { return a + N * (b + N * c); };
  for (int c = 0; c < 3; ++c) X[c][node] = x[((long long)e * 3 + c) * ND + node];
  __syncthreads();
  {
    double acc[3][3];
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c) acc[a][c] = 0.0;
    for (int m = 0; m < N; ++m)
      for (int c = 0; c < 3; ++c) {
        acc[0][c] = add(acc[0][c], mul(T.D[i][m], X[c][id(m, j, k)]));
        acc[1][c] = add(acc[1][c], mul(T.D[j][m], X[c][id(i, m, k)]));
        acc[2][c] = add(acc[2][c], mul(T.D[k][m], X[c][id(i, j, m)]));
      }
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c) J[a][c][node] = acc[a][c];
  }
  __syncthreads();
  // curl form: Ja^a_n from 0.5 D (x_m J(b, l) - x_l J(b, m)) along the two
  // other reference directions, (n, m, l) cyclic
  auto term = [&](int q, int b, int mm, int ll) {
    return sub(mul(X[mm][q], J[b][ll][q]), mul(X[ll][q], J[b][mm][q]));
  };
  const long long base = (long long)e * 9 * ND + node;
  for (int n = 0; n < 3; ++n) {
    const int mm = (n + 1) % 3, ll = (n + 2) % 3;
    double r0 = 0.0, r1 = 0.0, r2 = 0.0;
    for (int ii = 0; ii < N; ++ii)
      r0 = add(r0, mul(mul(0.5, T.D[j][ii]), term(id(i, ii, k), 2, mm, ll)));
    for (int ii = 0; ii < N; ++ii)
      r0 = sub(r0, mul(mul(0.5, T.D[k][ii]), term(id(i, j, ii), 1, mm, ll)));
    for (int ii = 0; ii < N; ++ii)
      r1 = add(r1, mul(mul(0.5, T.D[k][ii]), term(id(i, j, ii), 0, mm, ll)));
    for (int ii = 0; ii < N; ++ii)
      r1 = sub(r1, mul(mul(0.5, T.D[i][ii]), term(id(ii, j, k), 2, mm, ll)));
    for (int ii = 0; ii < N; ++ii)
      r2 = add(r2, mul(mul(0.5, T.D[i][ii]), term(id(ii, j, k), 1, mm, ll)));
    for (int ii = 0; ii < N; ++ii)
      r2 = sub(r2, mul(mul(0.5, T.D[j][ii]), term(id(i, ii, k), 0, mm, ll)));
    ja[base + (0 * 3 + n) * ND] = r0;
    ja[base + (1 * 3 + n) * ND] = r1;
    ja[base + (2 * 3 + n) * ND] = r2;
  }
  const double j11 = J[0][0][node], j12 = J[0][1][node], j13 = J[0][2][node];
  const double j21 = J[1][0][node], j22 = J[1][1][node], j23 = J[1][2][node];
  const double j31 = J[2][0][node], j32 = J[2][1][node], j33 = J[2][2][node];
  const double det = add(sub(mul(j11, sub(mul(j22, j33), mul(j23, j32))),
                             mul(j12, sub(mul(j21, j33), mul(j23, j31)))),
                         mul(j13, sub(mul(j21, j32), mul(j22, j31))));
  inv_j[(long long)e * ND + node] = __ddiv_rn(1.0, det);
}

}  // namespace

extern "C" dgsem_status dgsem_geometry_from_coordinates(int ndims, int polydeg,
                                                        const int64_t* n_cells, const double* x,
                                                        double* ja, double* inv_j,
                                                        void* stream) {
  if (!n_cells || !x || !ja || !inv_j || (ndims != 2 && ndims != 3)) return DGSEM_ERR_INVALID_ARG;
  dgsem::BasisTables b;
  if (!dgsem::make_basis(polydeg, &b)) return DGSEM_ERR_INVALID_ARG;
  const int n = b.n;
  if (ndims == 3 && n > 5) return DGSEM_ERR_UNSUPPORTED;
  int64_t nelem = 1;
  for (int a = 0; a < ndims; ++a) {
    if (n_cells[a] < 1) return DGSEM_ERR_INVALID_ARG;
    nelem *= n_cells[a];
  }
  if (nelem > 0x7fffffff) return DGSEM_ERR_INVALID_ARG;
  DerivTable T{};
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) T.D[i][j] = b.D[i][j];
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const unsigned grid = (unsigned)nelem;
#define DGSEM_GEO2(NN) \
  case NN: geometry_2d_kernel<NN><<<grid, NN * NN, 0, s>>>(x, ja, inv_j, T); break;
#define DGSEM_GEO3(NN) \
  case NN: geometry_3d_kernel<NN><<<grid, NN * NN * NN, 0, s>>>(x, ja, inv_j, T); break;
  if (ndims == 2) {
    switch (n) {
      DGSEM_GEO2(2) DGSEM_GEO2(3) DGSEM_GEO2(4) DGSEM_GEO2(5) DGSEM_GEO2(6) DGSEM_GEO2(7)
      DGSEM_GEO2(8)
      default: return DGSEM_ERR_UNSUPPORTED;
    }
  } else {
    switch (n) {
      DGSEM_GEO3(2) DGSEM_GEO3(3) DGSEM_GEO3(4) DGSEM_GEO3(5)
      default: return DGSEM_ERR_UNSUPPORTED;
    }
  }
#undef DGSEM_GEO2
#undef DGSEM_GEO3
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? DGSEM_OK : DGSEM_ERR_CUDA;
}

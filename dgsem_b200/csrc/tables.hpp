// Host-side precompute for the device kernels: Lobatto-Legendre basis tables
// and the metric tables of uniform structured (LinearMapping) meshes.
//
// Basis: polynomial_basis/basis_detail.hpp:52-262 (GLL Newton iteration,
// barycentric weights, D, Dsplit, Dhat, l(+-1)/w, inverse Legendre
// Vandermonde by Gauss-Jordan, base/container_fixed.hpp:117-162).
//
// Geometry: containers/data_container.hpp:160-726.  On a LinearMapping mesh
// every coordinate component x_b depends only on (element index, node index)
// along axis b.  Hence the reference's per-node metrics -- including their
// round-off, which is what a 1e-12 parity bar sees -- factor exactly:
//   * contravariant Ja^a_c depends only on the element indices of the axes
//     other than c (and on the node indices): stored as table[a][c][eidx][node]
//     with eidx running over the axes != c;
//   * J(a,a) = d x_a / d xi_a depends on (element, node) along axis a only;
//     1/J = 1 / (J00 * J11 [* J22]) because the off-diagonal products of the
//     reference's determinant are ~eps^2 relative and never change the
//     rounded result;
//   * the FV subcell normals (base/global_def.hpp:174-252 in 2D, :296-440 in
//     3D) are cumulative sums of Ja along a line and factor the same way.
// The tables are computed by restating the reference's loops in the same
// accumulation order with no FP contraction, so they agree bitwise.
#pragma once

#include <cstdint>
#include <vector>

namespace dgsem {

constexpr int kMaxNodes = 8;

struct BasisTables {
  int n = 0;
  double nodes[kMaxNodes];
  double weights[kMaxNodes];
  double inv_weights[kMaxNodes];
  double lhat_left[kMaxNodes];
  double lhat_right[kMaxNodes];
  double D[kMaxNodes][kMaxNodes];
  double Dsplit[kMaxNodes][kMaxNodes];
  double Dhat[kMaxNodes][kMaxNodes];
  double Vinv[kMaxNodes][kMaxNodes];
};

// Computes the Lobatto-Legendre tables for n = polydeg + 1 nodes (n <= 8).
bool make_basis(int polydeg, BasisTables* out);

// Host copies of the separable metric tables of one mesh.
struct MetricTablesHost {
  int ndims = 0;
  int n = 0;
  int64_t cells[3] = {1, 1, 1};
  // coord[a][e_a * n + i]
  std::vector<double> coord[3];
  // jdiag[a][e_a * n + i] = J(a, a)
  std::vector<double> jdiag[3];
  // ja[a][c][eidx_c * n^d + node]
  std::vector<double> ja[3][3];
  // FV subcell normals: fv[dir][c][eidx_c * (n-1) * n^(d-1) + f * n^(d-1) + line]
  // (line = the node index over the axes != dir, first axis fastest)
  std::vector<double> fv[3][3];
};

// Element-index of the axes other than c (x fastest):
//   2D: c=0 -> je, c=1 -> ie;  3D: c=0 -> je + ny ke, c=1 -> ie + nx ke,
//   c=2 -> ie + nx je.
int64_t other_axes_count(int ndims, const int64_t* cells, int c);

bool make_metric_tables(const BasisTables& b, int ndims, const int64_t* cells,
                        const double* left, const double* right,
                        MetricTablesHost* out);

}  // namespace dgsem

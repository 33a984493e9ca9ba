// Host precompute of basis and metric tables (see tables.hpp).
// Must be compiled without floating-point contraction (-ffp-contract=off):
// the loops restate the reference's accumulation order so the results match
// the reference bitwise.
#include "tables.hpp"

#include <cmath>
#include <cstdlib>
#include <limits>

namespace dgsem {
namespace {

// basis_detail.hpp:34-50: Legendre recurrence for P_n and its derivative up
// to n = polydeg; q = (2n+1)/(n+1) (x P_n - P_{n-2}) and q' = (2n+1) P_n
// (same operations and order as the reference, for bitwise equal nodes).
void q_and_l(int polydeg, double x, double* q, double* qder, double* LN) {
  double p_prev2 = 1.0, p_prev = x, dp_prev2 = 0.0, dp_prev = 1.0;
  double p_cur = 0.0, dp_cur = 0.0;
  for (int i = 2; i <= polydeg; ++i) {
    p_cur = ((double)(2.0 * i - 1.0) * x * p_prev - (double)(i - 1.0) * p_prev2) /
            (double)i;
    dp_cur = dp_prev2 + (double)(2.0 * i - 1.0) * p_prev;
    p_prev2 = p_prev;
    p_prev = p_cur;
    dp_prev2 = dp_prev;
    dp_prev = dp_cur;
  }
  *q = (double)(2.0 * polydeg + 1.0) / (polydeg + 1.0) * (x * p_cur - p_prev2);
  *qder = (2.0 * polydeg + 1.0) * p_cur;
  *LN = p_cur;
}

void barycentric(int n, const double* nodes, double* wb) {
  for (int i = 0; i < n; ++i) wb[i] = 1.0;
  for (int j = 1; j < n; ++j)
    for (int k = 0; k < j; ++k) {
      wb[k] *= (nodes[k] - nodes[j]);
      wb[j] *= (nodes[j] - nodes[k]);
    }
  for (int i = 0; i < n; ++i) wb[i] = 1.0 / wb[i];
}

// Lagrange basis values at x divided by the weights (the lifting vector):
// barycentric form, exact 1 at a node.
void lhat(int n, double x, const double* nodes, const double* w, double* out) {
  double wb[kMaxNodes];
  barycentric(n, nodes, wb);
  double lag[kMaxNodes] = {0};
  bool at_node = false;
  for (int i = 0; i < n; ++i) {
    if (std::abs(x - nodes[i]) < std::numeric_limits<double>::epsilon()) {
      lag[i] = 1.0;
      at_node = true;
      break;
    }
  }
  if (!at_node) {
    for (int i = 0; i < n; ++i) lag[i] = wb[i] / (x - nodes[i]);
    double denom = 0.0;
    for (int i = 0; i < n; ++i) denom += lag[i];
    for (int i = 0; i < n; ++i) lag[i] /= denom;
  }
  for (int i = 0; i < n; ++i) out[i] = lag[i] / w[i];
}

// Normalised Legendre polynomial sqrt(n + 1/2) P_n(x) (the modal basis of the
// shock indicator's Vandermonde matrix).
double legendre(int nn, double x) {
  double p_n = 0.0;
  if (nn == 0) {
    p_n = 1.0;
  } else if (nn == 1) {
    p_n = x;
  } else {
    double p_prev2 = 1.0, p_prev = x;
    for (int i = 2; i <= nn; ++i) {
      p_n = ((double)(2.0 * i - 1.0) * x * p_prev - (double)(i - 1.0) * p_prev2) /
            (double)i;
      p_prev2 = p_prev;
      p_prev = p_n;
    }
  }
  return p_n * std::sqrt(nn + 0.5);
}

// base/container_fixed.hpp:117-162 (partial-pivot Gauss-Jordan)
void invert(int n, double A[kMaxNodes][kMaxNodes],
            double inv[kMaxNodes][kMaxNodes]) {
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) inv[i][j] = (i == j) ? 1.0 : 0.0;
  for (int col = 0; col < n; ++col) {
    int pivot = col;
    double max_val = A[col][col] < 0 ? -A[col][col] : A[col][col];
    for (int row = col + 1; row < n; ++row) {
      const double v = A[row][col] < 0 ? -A[row][col] : A[row][col];
      if (v > max_val) {
        max_val = v;
        pivot = row;
      }
    }
    if (pivot != col) {
      for (int k = 0; k < n; ++k) {
        std::swap(A[col][k], A[pivot][k]);
        std::swap(inv[col][k], inv[pivot][k]);
      }
    }
    const double diag = A[col][col];
    for (int k = 0; k < n; ++k) {
      A[col][k] /= diag;
      inv[col][k] /= diag;
    }
    for (int row = 0; row < n; ++row) {
      if (row == col) continue;
      const double f = A[row][col];
      for (int k = 0; k < n; ++k) {
        A[row][k] -= f * A[col][k];
        inv[row][k] -= f * inv[col][k];
      }
    }
  }
}

// data_container.hpp:208-241 cell offsets + base/mapping.hpp:8-31.
void axis_coords(const BasisTables& b, int64_t ncells, double left,
                 double right, std::vector<double>* out) {
  const int n = b.n;
  out->assign(ncells * n, 0.0);
  const double dx = 2.0 / (double)ncells;
  for (int64_t e = 0; e < ncells; ++e) {
    const double off = -1.0 + (double)e * dx + 0.5 * dx;
    for (int i = 0; i < n; ++i) {
      const double c = off + 0.5 * dx * b.nodes[i];
      (*out)[e * n + i] = 0.5 * ((1.0 - c) * left + (1.0 + c) * right);
    }
  }
}

// Per-element 3D metrics exactly as data_container.hpp:414-659 computes them.
// Node index = (k * n + j) * n + i; x[b](i, j, k) from the axis tables.
void element_metrics_3d(const BasisTables& b, const double* X, const double* Y,
                        const double* Z, std::vector<double>& jac,
                        std::vector<double>& ja) {
  const int n = b.n;
  const int nd = n * n * n;
  jac.assign(nd * 9, 0.0);
  ja.assign(nd * 9, 0.0);
  auto node = [n](int i, int j, int k) { return (k * n + j) * n + i; };
  auto coord = [&](int i, int j, int k, int c) -> double {
    return c == 0 ? X[i] : (c == 1 ? Y[j] : Z[k]);
  };
  auto J = [&](int nidx, int a, int c) -> double& { return jac[nidx * 9 + a * 3 + c]; };
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        double acc[3][3] = {{0}};
        for (int m = 0; m < n; ++m) {
          for (int c = 0; c < 3; ++c) {
            acc[0][c] += b.D[i][m] * coord(m, j, k, c);
            acc[1][c] += b.D[j][m] * coord(i, m, k, c);
            acc[2][c] += b.D[k][m] * coord(i, j, m, c);
          }
        }
        const int id = node(i, j, k);
        for (int a = 0; a < 3; ++a)
          for (int c = 0; c < 3; ++c) J(id, a, c) = acc[a][c];
      }
  for (int nn = 0; nn < 3; ++nn) {
    const int m_ = (nn + 1) % 3;
    const int l_ = (nn + 2) % 3;
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          double r = 0.0;
          for (int ii = 0; ii < n; ++ii) {
            const int q = node(i, ii, k);
            r += 0.5 * b.D[j][ii] *
                 (coord(i, ii, k, m_) * J(q, 2, l_) - coord(i, ii, k, l_) * J(q, 2, m_));
          }
          for (int ii = 0; ii < n; ++ii) {
            const int q = node(i, j, ii);
            r -= 0.5 * b.D[k][ii] *
                 (coord(i, j, ii, m_) * J(q, 1, l_) - coord(i, j, ii, l_) * J(q, 1, m_));
          }
          ja[node(i, j, k) * 9 + 0 * 3 + nn] = r;
        }
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          double r = 0.0;
          for (int ii = 0; ii < n; ++ii) {
            const int q = node(i, j, ii);
            r += 0.5 * b.D[k][ii] *
                 (coord(i, j, ii, m_) * J(q, 0, l_) - coord(i, j, ii, l_) * J(q, 0, m_));
          }
          for (int ii = 0; ii < n; ++ii) {
            const int q = node(ii, j, k);
            r -= 0.5 * b.D[i][ii] *
                 (coord(ii, j, k, m_) * J(q, 2, l_) - coord(ii, j, k, l_) * J(q, 2, m_));
          }
          ja[node(i, j, k) * 9 + 1 * 3 + nn] = r;
        }
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          double r = 0.0;
          for (int ii = 0; ii < n; ++ii) {
            const int q = node(ii, j, k);
            r += 0.5 * b.D[i][ii] *
                 (coord(ii, j, k, m_) * J(q, 1, l_) - coord(ii, j, k, l_) * J(q, 1, m_));
          }
          for (int ii = 0; ii < n; ++ii) {
            const int q = node(i, ii, k);
            r -= 0.5 * b.D[j][ii] *
                 (coord(i, ii, k, m_) * J(q, 0, l_) - coord(i, ii, k, l_) * J(q, 0, m_));
          }
          ja[node(i, j, k) * 9 + 2 * 3 + nn] = r;
        }
  }
}

}  // namespace

bool make_basis(int polydeg, BasisTables* out) {
  const int n = polydeg + 1;
  if (polydeg < 1 || n > kMaxNodes || !out) return false;
  BasisTables& b = *out;
  b = BasisTables{};
  b.n = n;
  // basis_detail.hpp:52-109
  const double tol = 2.0 * std::numeric_limits<double>::epsilon();
  b.nodes[0] = -1.0;
  b.nodes[n - 1] = 1.0;
  b.weights[0] = 2.0 / (polydeg * (polydeg + 1.0));
  b.weights[n - 1] = b.weights[0];
  const double cont1 = M_PI / polydeg;
  const double cont2 = 3.0 / (8.0 * polydeg * M_PI);
  for (int i = 0; i < n / 2 - 1; ++i) {
    double x = -std::cos(cont1 * ((i + 1) + 0.25) - cont2 / ((i + 1) + 0.25));
    double q, qder, LN;
    for (int it = 0; it < 20; ++it) {
      q_and_l(polydeg, x, &q, &qder, &LN);
      const double dx = -q / qder;
      x += dx;
      if (std::abs(dx) < tol * std::abs(x)) break;
    }
    b.nodes[i + 1] = x;
    q_and_l(polydeg, x, &q, &qder, &LN);
    b.weights[i + 1] = b.weights[0] / (LN * LN);
    b.nodes[n - 2 - i] = -x;
    b.weights[n - 2 - i] = b.weights[i + 1];
  }
  if (n % 2 == 1) {
    double q, qder, LN;
    b.nodes[n / 2] = 0.0;
    q_and_l(polydeg, 0.0, &q, &qder, &LN);
    b.weights[n / 2] = b.weights[0] / (LN * LN);
  }
  for (int i = 0; i < n; ++i) b.inv_weights[i] = 1.0 / b.weights[i];
  lhat(n, -1.0, b.nodes, b.weights, b.lhat_left);
  lhat(n, 1.0, b.nodes, b.weights, b.lhat_right);
  // basis_detail.hpp:170-188
  double wb[kMaxNodes];
  barycentric(n, b.nodes, wb);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) b.D[i][j] = 0.0;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      if (i != j) {
        b.D[i][j] = wb[j] / wb[i] * 1.0 / (b.nodes[i] - b.nodes[j]);
        b.D[i][i] -= b.D[i][j];
      }
  // basis_detail.hpp:190-215
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      b.Dsplit[i][j] = 2.0 * b.D[i][j];
      b.Dhat[i][j] = b.D[j][i];
    }
  b.Dsplit[0][0] += 1.0 / b.weights[0];
  b.Dsplit[n - 1][n - 1] -= 1.0 / b.weights[n - 1];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) b.Dhat[j][i] *= -b.weights[i] / b.weights[j];
  // basis_detail.hpp:247-262
  double V[kMaxNodes][kMaxNodes];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) V[i][j] = legendre(j, b.nodes[i]);
  invert(n, V, b.Vinv);
  return true;
}

int64_t other_axes_count(int ndims, const int64_t* cells, int c) {
  if (ndims == 2) return c == 0 ? cells[1] : cells[0];
  if (c == 0) return cells[1] * cells[2];
  if (c == 1) return cells[0] * cells[2];
  return cells[0] * cells[1];
}

bool make_metric_tables(const BasisTables& b, int ndims, const int64_t* cells,
                        const double* left, const double* right,
                        MetricTablesHost* out) {
  if (!out || (ndims != 2 && ndims != 3)) return false;
  const int n = b.n;
  MetricTablesHost& t = *out;
  t = MetricTablesHost{};
  t.ndims = ndims;
  t.n = n;
  for (int a = 0; a < ndims; ++a) {
    if (cells[a] < 1 || !(right[a] > left[a])) return false;
    t.cells[a] = cells[a];
    axis_coords(b, cells[a], left[a], right[a], &t.coord[a]);
    // J(a, a) along axis a: sum_k D(i, k) x_a(e, k), sequential.
    t.jdiag[a].assign(cells[a] * n, 0.0);
    for (int64_t e = 0; e < cells[a]; ++e)
      for (int i = 0; i < n; ++i) {
        double acc = 0.0;
        for (int k = 0; k < n; ++k) acc += b.D[i][k] * t.coord[a][e * n + k];
        t.jdiag[a][e * n + i] = acc;
      }
  }
  if (ndims == 2) {
    const int nd = n * n;
    const double* X = t.coord[0].data();
    const double* Y = t.coord[1].data();
    // data_container.hpp:247-304: J00 = sum D(i,k) x(k), J01 = sum D(i,k) y,
    // J10 = sum D(j,k) x, J11 = sum D(j,k) y(k); Ja = adjugate.
    for (int a = 0; a < 2; ++a)
      for (int c = 0; c < 2; ++c)
        t.ja[a][c].assign(other_axes_count(2, cells, c) * nd, 0.0);
    for (int64_t je = 0; je < cells[1]; ++je)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          double j01 = 0.0;
          for (int k = 0; k < n; ++k) j01 += b.D[i][k] * Y[je * n + j];
          t.ja[0][0][je * nd + j * n + i] = t.jdiag[1][je * n + j];  // J11
          t.ja[1][0][je * nd + j * n + i] = -j01;                     // -J01
        }
    for (int64_t ie = 0; ie < cells[0]; ++ie)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          double j10 = 0.0;
          for (int k = 0; k < n; ++k) j10 += b.D[j][k] * X[ie * n + i];
          t.ja[0][1][ie * nd + j * n + i] = -j10;                     // -J10
          t.ja[1][1][ie * nd + j * n + i] = t.jdiag[0][ie * n + i];   // J00
        }
    // global_def.hpp:174-252: cumulative subcell normals per line.
    for (int dir = 0; dir < 2; ++dir)
      for (int c = 0; c < 2; ++c) {
        const int64_t ne = other_axes_count(2, cells, c);
        std::vector<double>& fv = t.fv[dir][c];
        fv.assign(ne * (n - 1) * n, 0.0);
        const std::vector<double>& JA = t.ja[dir][c];
        for (int64_t e = 0; e < ne; ++e)
          for (int line = 0; line < n; ++line) {
            auto ja_at = [&](int pos) {
              const int node = dir == 0 ? line * n + pos : pos * n + line;
              return JA[e * nd + node];
            };
            double acc = ja_at(0);
            for (int m = 0; m < n; ++m) acc += b.weights[0] * b.D[0][m] * ja_at(m);
            fv[e * (n - 1) * n + 0 * n + line] = acc;
            for (int f = 1; f < n - 1; ++f) {
              acc = fv[e * (n - 1) * n + (f - 1) * n + line];
              for (int m = 0; m < n; ++m) acc += b.weights[f] * b.D[f][m] * ja_at(m);
              fv[e * (n - 1) * n + f * n + line] = acc;
            }
          }
      }
    return true;
  }
  // 3D: Ja^a_c depends on the element indices of the axes != c only.
  const int nd = n * n * n;
  for (int a = 0; a < 3; ++a)
    for (int c = 0; c < 3; ++c)
      t.ja[a][c].assign(other_axes_count(3, cells, c) * nd, 0.0);
  std::vector<double> jac, ja;
  const int64_t nx = cells[0], ny = cells[1], nz = cells[2];
  for (int c = 0; c < 3; ++c) {
    const int64_t n_outer = c == 0 ? ny : nx;
    const int64_t n_inner = c == 2 ? ny : nz;
    for (int64_t p = 0; p < n_outer; ++p)
      for (int64_t q = 0; q < n_inner; ++q) {
        int64_t ie = 0, je = 0, ke = 0;
        if (c == 0) { je = p; ke = q; }
        if (c == 1) { ie = p; ke = q; }
        if (c == 2) { ie = p; je = q; }
        element_metrics_3d(b, &t.coord[0][ie * n], &t.coord[1][je * n],
                           &t.coord[2][ke * n], jac, ja);
        const int64_t eidx = (c == 0) ? (je + ny * ke)
                             : (c == 1) ? (ie + nx * ke) : (ie + nx * je);
        for (int a = 0; a < 3; ++a)
          for (int node = 0; node < nd; ++node)
            t.ja[a][c][eidx * nd + node] = ja[node * 9 + a * 3 + c];
      }
  }
  // global_def.hpp:296-440: cumulative subcell normals along each line,
  // normal_dir(face f) = Ja^dir(node 0) + sum_{f' <= f} sum_m w_f' D(f', m) Ja^dir(node m)
  const int nf = n * n;
  for (int dir = 0; dir < 3; ++dir)
    for (int c = 0; c < 3; ++c) {
      const int64_t ne = other_axes_count(3, cells, c);
      std::vector<double>& fv = t.fv[dir][c];
      fv.assign(ne * (n - 1) * nf, 0.0);
      const std::vector<double>& JA = t.ja[dir][c];
      for (int64_t e = 0; e < ne; ++e)
        for (int line = 0; line < nf; ++line) {
          auto ja_at = [&](int pos) {
            const int a = line % n, b2 = line / n;  // the two other node indices
            const int node = dir == 0 ? pos + n * a + nf * b2
                             : dir == 1 ? a + n * pos + nf * b2 : a + n * b2 + nf * pos;
            return JA[e * nd + node];
          };
          double acc = ja_at(0);
          for (int m = 0; m < n; ++m) acc += b.weights[0] * b.D[0][m] * ja_at(m);
          fv[e * (n - 1) * nf + 0 * nf + line] = acc;
          for (int f = 1; f < n - 1; ++f) {
            acc = fv[e * (n - 1) * nf + (f - 1) * nf + line];
            for (int m = 0; m < n; ++m) acc += b.weights[f] * b.D[f][m] * ja_at(m);
            fv[e * (n - 1) * nf + f * nf + line] = acc;
          }
        }
    }
  return true;
}

}  // namespace dgsem

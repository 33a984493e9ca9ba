"""CPU restatement of the reference DGSEM right-hand side (TEST INFRASTRUCTURE).

This module is the oracle: a plain numpy restatement of the reference
algorithm (RetrO598/DGSEM, header-only C++ on Kokkos) for the hot path
  split-form flux differencing volume integral, LLF surface flux + lifting,
  Hennemann-Gassner subcell blending, BR1 viscous terms, SSPRK3 stages.
Each function cites the reference file:line it follows.  It is pinned against
the reference itself: ``oracle/_ref/libdgsem_ref.so`` (the unmodified
reference headers compiled against the project's Kokkos shim) and the golden
fixtures under ``tests/golden`` produced from it.

Only tests, ``__graft_entry__.smoke`` and the CPU-baseline leg of ``bench.py``
use this module; the product path never imports it.

Array layout is the reference's logical LayoutRight order
  2D: u[ie, je, dof, var]        dof = jn * n + in
  3D: u[ie, je, ke, dof, var]    dof = (kn * n + jn) * n + in
(``utils/local_dof.hpp:9-19``).  Internally the dof axis is reshaped to
[jn, in] / [kn, jn, in].

Where reference arithmetic is order-sensitive (basis tables, geometry), the
loops keep the reference's accumulation order so that results agree bitwise;
elsewhere vectorised numpy keeps each floating-point expression of the
reference but may sum contributions in a different order.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# ---------------------------------------------------------------------------
# Basis tables: polynomial_basis/basis_detail.hpp
# ---------------------------------------------------------------------------


def _q_and_l(polydeg: int, x: float):
    """basis_detail.hpp:34-50 evaluate_q_and_l (Legendre recursion)."""
    L_Nm2, L_Nm1 = 1.0, x
    Lder_Nm2, Lder_Nm1 = 0.0, 1.0
    L_N = Lder_N = 0.0
    for i in range(2, polydeg + 1):
        L_N = ((2.0 * i - 1.0) * x * L_Nm1 - (i - 1.0) * L_Nm2) / i
        Lder_N = Lder_Nm2 + (2.0 * i - 1.0) * L_Nm1
        L_Nm2, L_Nm1 = L_Nm1, L_N
        Lder_Nm2, Lder_Nm1 = Lder_Nm1, Lder_N
    q = (2.0 * polydeg + 1.0) / (polydeg + 1.0) * (x * L_N - L_Nm2)
    qder = (2.0 * polydeg + 1.0) * L_N
    return q, qder, L_N


def gll_nodes_weights(n: int):
    """basis_detail.hpp:52-109 gauss_lobatto_nodes_weights (Newton on q)."""
    polydeg = n - 1
    tol = 2.0 * np.finfo(np.float64).eps
    nodes = np.zeros(n)
    w = np.zeros(n)
    nodes[0], nodes[-1] = -1.0, 1.0
    w[0] = 2.0 / (polydeg * (polydeg + 1.0))
    w[-1] = w[0]
    cont1 = math.pi / polydeg
    cont2 = 3.0 / (8.0 * polydeg * math.pi)
    for i in range(n // 2 - 1):
        x = -math.cos(cont1 * ((i + 1) + 0.25) - cont2 / ((i + 1) + 0.25))
        for _ in range(20):
            q, qder, _ = _q_and_l(polydeg, x)
            dx = -q / qder
            x += dx
            if abs(dx) < tol * abs(x):
                break
        nodes[i + 1] = x
        _, _, L_N = _q_and_l(polydeg, x)
        w[i + 1] = w[0] / (L_N * L_N)
        nodes[n - 2 - i] = -x
        w[n - 2 - i] = w[i + 1]
    if n % 2 == 1:
        nodes[n // 2] = 0.0
        _, _, L_N = _q_and_l(polydeg, 0.0)
        w[n // 2] = w[0] / (L_N * L_N)
    return nodes, w


def _barycentric(nodes):
    """basis_detail.hpp:111-128."""
    n = len(nodes)
    wb = [1.0] * n
    for j in range(1, n):
        for k in range(j):
            wb[k] *= nodes[k] - nodes[j]
            wb[j] *= nodes[j] - nodes[k]
    return [1.0 / v for v in wb]


def _lhat(x, nodes, weights):
    """basis_detail.hpp:130-168 lagrange polynomials at x divided by w."""
    n = len(nodes)
    wb = _barycentric(nodes)
    poly = [0.0] * n
    hit = False
    for i in range(n):
        if abs(x - nodes[i]) < np.finfo(np.float64).eps:
            poly[i] = 1.0
            hit = True
            break
    if not hit:
        poly = [wb[i] / (x - nodes[i]) for i in range(n)]
        total = 0.0
        for p in poly:
            total += p
        poly = [p / total for p in poly]
    return np.array([poly[i] / weights[i] for i in range(n)])


def _derivative_matrix(nodes):
    """basis_detail.hpp:170-188 polynomial_derivative_matrix."""
    n = len(nodes)
    wb = _barycentric(nodes)
    D = [[0.0] * n for _ in range(n)]
    for i in range(n):
        for j in range(n):
            if i != j:
                D[i][j] = wb[j] / wb[i] * 1.0 / (nodes[i] - nodes[j])
                D[i][i] -= D[i][j]
    return np.array(D)


def _legendre(nn: int, x: float) -> float:
    """basis_detail.hpp:217-245 normalised Legendre polynomial value."""
    if nn == 0:
        poly = 1.0
    elif nn == 1:
        poly = x
    else:
        p2, p1 = 1.0, x
        poly = 0.0
        for i in range(2, nn + 1):
            poly = ((2.0 * i - 1.0) * x * p1 - (i - 1.0) * p2) / i
            p2, p1 = p1, poly
    return poly * math.sqrt(nn + 0.5)


def _inverse_gauss_jordan(A):
    """base/container_fixed.hpp:117-162 Mat::inverse (partial pivoting)."""
    n = len(A)
    A = [list(r) for r in A]
    inv = [[1.0 if i == j else 0.0 for j in range(n)] for i in range(n)]
    for col in range(n):
        pivot = col
        max_val = -A[col][col] if A[col][col] < 0 else A[col][col]
        for row in range(col + 1, n):
            v = -A[row][col] if A[row][col] < 0 else A[row][col]
            if v > max_val:
                max_val, pivot = v, row
        if pivot != col:
            A[col], A[pivot] = A[pivot], A[col]
            inv[col], inv[pivot] = inv[pivot], inv[col]
        diag = A[col][col]
        A[col] = [v / diag for v in A[col]]
        inv[col] = [v / diag for v in inv[col]]
        for row in range(n):
            if row == col:
                continue
            f = A[row][col]
            A[row] = [A[row][k] - f * A[col][k] for k in range(n)]
            inv[row] = [inv[row][k] - f * inv[col][k] for k in range(n)]
    return np.array(inv)


@dataclass
class Basis:
    """LobattoLegendreBasis<double, N> tables (polynomial_basis/basis.hpp:69-153)."""

    polydeg: int
    nodes: np.ndarray = field(init=False)
    weights: np.ndarray = field(init=False)
    inv_weights: np.ndarray = field(init=False)
    lhat_left: np.ndarray = field(init=False)
    lhat_right: np.ndarray = field(init=False)
    D: np.ndarray = field(init=False)
    Dsplit: np.ndarray = field(init=False)
    Dhat: np.ndarray = field(init=False)
    Vinv: np.ndarray = field(init=False)

    def __post_init__(self):
        n = self.polydeg + 1
        self.nodes, self.weights = gll_nodes_weights(n)
        self.inv_weights = np.array([1.0 / w for w in self.weights])
        self.lhat_left = _lhat(-1.0, self.nodes, self.weights)
        self.lhat_right = _lhat(1.0, self.nodes, self.weights)
        self.D = _derivative_matrix(self.nodes)
        # basis_detail.hpp:190-200 calc_dsplit
        Ds = 2.0 * self.D
        Ds[0, 0] += 1.0 / self.weights[0]
        Ds[n - 1, n - 1] -= 1.0 / self.weights[n - 1]
        self.Dsplit = Ds
        # basis_detail.hpp:202-215 calc_dhat
        Dh = self.D.T.copy()
        for i in range(n):
            for j in range(n):
                Dh[j, i] *= -self.weights[i] / self.weights[j]
        self.Dhat = Dh
        # basis_detail.hpp:247-262 inverse_vandermonde_legendre
        V = [[_legendre(j, self.nodes[i]) for j in range(n)] for i in range(n)]
        self.Vinv = _inverse_gauss_jordan(V)

    @property
    def n(self) -> int:
        return self.polydeg + 1


# ---------------------------------------------------------------------------
# Geometry: containers/data_container.hpp (uniform LinearMapping meshes)
# ---------------------------------------------------------------------------


def axis_coordinates(basis: Basis, ncells: int, left: float, right: float):
    """Node coordinates along one axis, x[e, node].

    data_container.hpp:208-241 / :367-408 (cell offsets) composed with
    base/mapping.hpp:8-31 linear_interpolate; the reference evaluates every
    physical coordinate component from its own axis only, so one table per
    axis reproduces them bitwise.
    """
    dx = 2.0 / ncells
    x = np.zeros((ncells, basis.n))
    for e in range(ncells):
        off = -1.0 + e * dx + 0.5 * dx
        for i in range(basis.n):
            c = off + 0.5 * dx * basis.nodes[i]
            x[e, i] = 0.5 * ((1.0 - c) * left + (1.0 + c) * right)
    return x


@dataclass
class Geometry:
    """Per-node metrics exactly as StructuredElementInitializer computes them."""

    coords: np.ndarray   # cells + (ndof, ndims)
    jac: np.ndarray      # cells + (ndof, ndims, ndims)   J(a, b) = d x_b / d xi_a
    ja: np.ndarray       # cells + (ndof, ndims, ndims)   contravariant Ja^a_b
    inv_j: np.ndarray    # cells + (ndof,)
    neighbors: np.ndarray  # cells + (ndims, ndims) (-1 = none)
    subcell: tuple = ()  # 2D only: (normal_1, normal_2)


def geometry_2d(basis: Basis, cells, left, right, periodic) -> Geometry:
    """data_container.hpp:160-331 (2D) + global_def.hpp:152-255 (subcell normals)."""
    n = basis.n
    nx, ny = cells
    D = basis.D
    X = axis_coordinates(basis, nx, left[0], right[0])
    Y = axis_coordinates(basis, ny, left[1], right[1])
    coords = np.zeros((nx, ny, n, n, 2))
    coords[..., 0] = X[:, None, None, :]
    coords[..., 1] = Y[None, :, :, None]
    jac = np.zeros((nx, ny, n, n, 2, 2))
    # data_container.hpp:247-282: sequential accumulation over k
    for jn in range(n):
        for i in range(n):
            dx_dxi = np.zeros((nx, ny)); dy_dxi = np.zeros((nx, ny))
            dx_deta = np.zeros((nx, ny)); dy_deta = np.zeros((nx, ny))
            for k in range(n):
                dx_dxi = dx_dxi + D[i, k] * coords[:, :, jn, k, 0]
                dy_dxi = dy_dxi + D[i, k] * coords[:, :, jn, k, 1]
                dx_deta = dx_deta + D[jn, k] * coords[:, :, k, i, 0]
                dy_deta = dy_deta + D[jn, k] * coords[:, :, k, i, 1]
            jac[:, :, jn, i, 0, 0] = dx_dxi
            jac[:, :, jn, i, 0, 1] = dy_dxi
            jac[:, :, jn, i, 1, 0] = dx_deta
            jac[:, :, jn, i, 1, 1] = dy_deta
    # data_container.hpp:284-304 contravariant vectors (adjugate)
    ja = np.zeros_like(jac)
    ja[..., 0, 0] = jac[..., 1, 1]
    ja[..., 0, 1] = -jac[..., 1, 0]
    ja[..., 1, 0] = -jac[..., 0, 1]
    ja[..., 1, 1] = jac[..., 0, 0]
    # data_container.hpp:306-312
    inv_j = 1.0 / (jac[..., 0, 0] * jac[..., 1, 1] - jac[..., 1, 0] * jac[..., 0, 1])
    # global_def.hpp:174-252 subcell normals by cumulative sums
    w = basis.weights
    n1 = np.zeros((nx, ny, n - 1, n, 2))
    n2 = np.zeros((nx, ny, n, n - 1, 2))
    for jn in range(n):
        acc = ja[:, :, jn, 0, 0, :].copy()
        for m in range(n):
            acc = acc + (w[0] * D[0, m]) * ja[:, :, jn, m, 0, :]
        n1[:, :, 0, jn, :] = acc
        for f in range(1, n - 1):
            acc = n1[:, :, f - 1, jn, :].copy()
            for m in range(n):
                acc = acc + (w[f] * D[f, m]) * ja[:, :, jn, m, 0, :]
            n1[:, :, f, jn, :] = acc
    for i in range(n):
        acc = ja[:, :, 0, i, 1, :].copy()
        for m in range(n):
            acc = acc + (w[0] * D[0, m]) * ja[:, :, m, i, 1, :]
        n2[:, :, i, 0, :] = acc
        for f in range(1, n - 1):
            acc = n2[:, :, i, f - 1, :].copy()
            for m in range(n):
                acc = acc + (w[f] * D[f, m]) * ja[:, :, m, i, 1, :]
            n2[:, :, i, f, :] = acc
    # data_container.hpp:314-331 left/bottom neighbours with periodic wrap
    nb = np.full((nx, ny, 2, 2), -1, dtype=np.int64)
    for ie in range(nx):
        for je in range(ny):
            nb[ie, je, 0, 0] = ie - 1 if ie > 0 else (nx - 1 if periodic[0] else -1)
            nb[ie, je, 0, 1] = je
            nb[ie, je, 1, 0] = ie
            nb[ie, je, 1, 1] = je - 1 if je > 0 else (ny - 1 if periodic[1] else -1)
    return Geometry(coords.reshape(nx, ny, n * n, 2), jac.reshape(nx, ny, n * n, 2, 2),
                    ja.reshape(nx, ny, n * n, 2, 2), inv_j.reshape(nx, ny, n * n), nb,
                    (n1, n2))


def geometry_3d(basis: Basis, cells, left, right, periodic) -> Geometry:
    """data_container.hpp:334-726 (3D, conservative curl-form metrics)."""
    n = basis.n
    nx, ny, nz = cells
    D = basis.D
    X = axis_coordinates(basis, nx, left[0], right[0])
    Y = axis_coordinates(basis, ny, left[1], right[1])
    Z = axis_coordinates(basis, nz, left[2], right[2])
    sh = (nx, ny, nz, n, n, n)  # [ie, je, ke, kn, jn, in]
    xs = [np.broadcast_to(X[:, None, None, None, None, :], sh),
          np.broadcast_to(Y[None, :, None, None, :, None], sh),
          np.broadcast_to(Z[None, None, :, :, None, None], sh)]
    coords = np.stack(xs, axis=-1).copy()
    # data_container.hpp:414-469: J(a, b) = sum_m D(node_a, m) x_b(node_a <- m)
    jac = np.zeros(sh + (3, 3))
    for kn in range(n):
        for jn in range(n):
            for i in range(n):
                acc = np.zeros((nx, ny, nz, 3, 3))
                for m in range(n):
                    for b in range(3):
                        acc[..., 0, b] = acc[..., 0, b] + D[i, m] * coords[:, :, :, kn, jn, m, b]
                        acc[..., 1, b] = acc[..., 1, b] + D[jn, m] * coords[:, :, :, kn, m, i, b]
                        acc[..., 2, b] = acc[..., 2, b] + D[kn, m] * coords[:, :, :, m, jn, i, b]
                jac[:, :, :, kn, jn, i] = acc
    ja = np.zeros_like(jac)
    x = coords
    # data_container.hpp:472-657 curl form, loop order n -> direction -> nodes
    for nn in range(3):
        m_ = (nn + 1) % 3
        l_ = (nn + 2) % 3
        for kn in range(n):
            for jn in range(n):
                for i in range(n):
                    # Ja^1_n: (A) eta term, (B) zeta term
                    r = np.zeros((nx, ny, nz))
                    for ii in range(n):
                        r = r + (0.5 * D[jn, ii]) * (x[:, :, :, kn, ii, i, m_] * jac[:, :, :, kn, ii, i, 2, l_]
                                                     - x[:, :, :, kn, ii, i, l_] * jac[:, :, :, kn, ii, i, 2, m_])
                    for ii in range(n):
                        r = r - (0.5 * D[kn, ii]) * (x[:, :, :, ii, jn, i, m_] * jac[:, :, :, ii, jn, i, 1, l_]
                                                     - x[:, :, :, ii, jn, i, l_] * jac[:, :, :, ii, jn, i, 1, m_])
                    ja[:, :, :, kn, jn, i, 0, nn] = r
        for kn in range(n):
            for jn in range(n):
                for i in range(n):
                    # Ja^2_n: (A) zeta term, (B) xi term
                    r = np.zeros((nx, ny, nz))
                    for ii in range(n):
                        r = r + (0.5 * D[kn, ii]) * (x[:, :, :, ii, jn, i, m_] * jac[:, :, :, ii, jn, i, 0, l_]
                                                     - x[:, :, :, ii, jn, i, l_] * jac[:, :, :, ii, jn, i, 0, m_])
                    for ii in range(n):
                        r = r - (0.5 * D[i, ii]) * (x[:, :, :, kn, jn, ii, m_] * jac[:, :, :, kn, jn, ii, 2, l_]
                                                    - x[:, :, :, kn, jn, ii, l_] * jac[:, :, :, kn, jn, ii, 2, m_])
                    ja[:, :, :, kn, jn, i, 1, nn] = r
        for kn in range(n):
            for jn in range(n):
                for i in range(n):
                    # Ja^3_n: (A) xi term, (B) eta term
                    r = np.zeros((nx, ny, nz))
                    for ii in range(n):
                        r = r + (0.5 * D[i, ii]) * (x[:, :, :, kn, jn, ii, m_] * jac[:, :, :, kn, jn, ii, 1, l_]
                                                    - x[:, :, :, kn, jn, ii, l_] * jac[:, :, :, kn, jn, ii, 1, m_])
                    for ii in range(n):
                        r = r - (0.5 * D[jn, ii]) * (x[:, :, :, kn, ii, i, m_] * jac[:, :, :, kn, ii, i, 0, l_]
                                                     - x[:, :, :, kn, ii, i, l_] * jac[:, :, :, kn, ii, i, 0, m_])
                    ja[:, :, :, kn, jn, i, 2, nn] = r
    j = jac
    det = (j[..., 0, 0] * (j[..., 1, 1] * j[..., 2, 2] - j[..., 1, 2] * j[..., 2, 1])
           - j[..., 0, 1] * (j[..., 1, 0] * j[..., 2, 2] - j[..., 1, 2] * j[..., 2, 0])
           + j[..., 0, 2] * (j[..., 1, 0] * j[..., 2, 1] - j[..., 1, 1] * j[..., 2, 0]))
    inv_j = 1.0 / det
    nb = np.full((nx, ny, nz, 3, 3), -1, dtype=np.int64)
    for ie in range(nx):
        for je in range(ny):
            for ke in range(nz):
                nb[ie, je, ke, 0] = (ie - 1 if ie > 0 else (nx - 1 if periodic[0] else -1), je, ke)
                nb[ie, je, ke, 1] = (ie, je - 1 if je > 0 else (ny - 1 if periodic[1] else -1), ke)
                nb[ie, je, ke, 2] = (ie, je, ke - 1 if ke > 0 else (nz - 1 if periodic[2] else -1))
    nd = n ** 3
    return Geometry(coords.reshape(nx, ny, nz, nd, 3), jac.reshape(nx, ny, nz, nd, 3, 3),
                    ja.reshape(nx, ny, nz, nd, 3, 3), inv_j.reshape(nx, ny, nz, nd), nb)


# ---------------------------------------------------------------------------
# Equations and two-point fluxes (vectorised over trailing "point" axes).
# States are arrays of shape (nvars, ...); normals (ndims, ...).
# ---------------------------------------------------------------------------


def ln_mean(x, y):
    """base/math_utils.hpp:8-25 logarithmic mean (Ismail-Roe series branch)."""
    num = x * (x - 2.0 * y) + y * y
    den = x * (x + 2.0 * y) + y * y
    f2 = num / den
    poly = 2.0 + f2 * (2.0 / 3.0 + f2 * (2.0 / 5.0 + f2 * (2.0 / 7.0)))
    with np.errstate(divide="ignore", invalid="ignore"):
        logv = (y - x) / np.log(y / x)
    return np.where(f2 < 1.0e-4, (x + y) / poly, logv)


def inv_ln_mean(x, y):
    """1 / ln_mean(x, y) evaluated with the same two branches (no extra division)."""
    num = x * (x - 2.0 * y) + y * y
    den = x * (x + 2.0 * y) + y * y
    f2 = num / den
    poly = 2.0 + f2 * (2.0 / 3.0 + f2 * (2.0 / 5.0 + f2 * (2.0 / 7.0)))
    with np.errstate(divide="ignore", invalid="ignore"):
        logv = np.log(y / x) / (y - x)
    return np.where(f2 < 1.0e-4, poly / (x + y), logv)


def _vel_p(u, gamma):
    nd = u.shape[0] - 2
    rho = u[0]
    v = [u[1 + d] / rho for d in range(nd)]
    v2 = v[0] * v[0]
    for d in range(1, nd):
        v2 = v2 + v[d] * v[d]
    p = (gamma - 1.0) * (u[nd + 1] - 0.5 * rho * v2)
    return rho, v, p, v2


def euler_flux_dim(u, dim, gamma):
    """compressible_euler2D.hpp:25-47 / compressible_euler3D.hpp:26-52."""
    nd = u.shape[0] - 2
    rho = u[0]
    vel = [u[1 + d] / rho for d in range(nd)]
    sq = vel[0] * vel[0]
    for d in range(1, nd):
        sq = sq + vel[d] * vel[d]
    kinetic = 0.5 * rho * sq
    p = (gamma - 1.0) * (u[nd + 1] - kinetic)
    mom = u[1 + dim]
    out = [mom]
    for d in range(nd):
        out.append(mom * vel[d] + (p if d == dim else 0.0))
    out.append(vel[dim] * (u[nd + 1] + p))
    return np.array(out)


def euler_flux_normal(u, normal, gamma):
    """compressible_euler2D.hpp:49-58 / 3D:54-67: sum_d n_d F_d."""
    nd = u.shape[0] - 2
    acc = normal[0] * euler_flux_dim(u, 0, gamma)
    for d in range(1, nd):
        acc = acc + normal[d] * euler_flux_dim(u, d, gamma)
    return acc


def wave_speed_normal(uL, uR, normal, gamma):
    """compressible_euler2D.hpp:70-109 / 3D:121-166 LLF speed with |n|."""
    nd = uL.shape[0] - 2
    rL, vL, pL, _ = _vel_p(uL, gamma)
    rR, vR, pR, _ = _vel_p(uR, gamma)
    aL = np.sqrt(gamma * pL / rL)
    aR = np.sqrt(gamma * pR / rR)
    nn = normal[0] * normal[0]
    for d in range(1, nd):
        nn = nn + normal[d] * normal[d]
    nnorm = np.sqrt(nn)
    vnL = vL[0] * normal[0]
    vnR = vR[0] * normal[0]
    for d in range(1, nd):
        vnL = vnL + vL[d] * normal[d]
        vnR = vnR + vR[d] * normal[d]
    return np.maximum(np.abs(vnL), np.abs(vnR)) + np.maximum(aL, aR) * nnorm


def flux_llf(uL, uR, normal, gamma):
    """numerical_flux.hpp:198-228 (2D) / :39-69 (3D) + numerical_flux_detail.hpp:9-21."""
    lam = wave_speed_normal(uL, uR, normal, gamma)
    fL = euler_flux_normal(uL, normal, gamma)
    fR = euler_flux_normal(uR, normal, gamma)
    return 0.5 * (fL + fR) - 0.5 * lam * (uR - uL)


def flux_chandrashekar(uL, uR, normal, gamma):
    """numerical_flux.hpp:436-500 (2D) / :520-594 (3D) EC/KEP two-point flux."""
    nd = uL.shape[0] - 2
    rL, vL, _, _ = _vel_p(uL, gamma)
    rR, vR, _, _ = _vel_p(uR, gamma)
    vnL = vL[0] * normal[0]
    vnR = vR[0] * normal[0]
    for d in range(1, nd):
        vnL = vnL + vL[d] * normal[d]
        vnR = vnR + vR[d] * normal[d]
    sqL = vL[0] * vL[0]
    sqR = vR[0] * vR[0]
    for d in range(1, nd):
        sqL = sqL + vL[d] * vL[d]
        sqR = sqR + vR[d] * vR[d]
    kinL = 0.5 * sqL
    kinR = 0.5 * sqR
    pL = (gamma - 1.0) * (uL[nd + 1] - 0.5 * rL * sqL)
    pR = (gamma - 1.0) * (uR[nd + 1] - 0.5 * rR * sqR)
    betaL = 0.5 * rL / pL
    betaR = 0.5 * rR / pR
    rho_avg = 0.5 * (rL + rR)
    rho_mean = ln_mean(rL, rR)
    beta_mean = ln_mean(betaL, betaR)
    beta_avg = 0.5 * (betaL + betaR)
    v_avg = [0.5 * (vL[d] + vR[d]) for d in range(nd)]
    p_mean = 0.5 * rho_avg / beta_avg
    vsq_avg = kinL + kinR
    f1 = rho_mean * 0.5 * (vnL + vnR)
    fm = [f1 * v_avg[d] + p_mean * normal[d] for d in range(nd)]
    fe = f1 * 0.5 * (1.0 / (gamma - 1.0) / beta_mean - vsq_avg)
    for d in range(nd):
        fe = fe + fm[d] * v_avg[d]
    return np.array([f1] + fm + [fe])


def flux_ranocha(uL, uR, normal, gamma):
    """Ranocha EC/KEP flux (absent in the reference; published formula).

    H. Ranocha, "Comparison of some entropy conservative numerical fluxes for
    the Euler equations", J. Sci. Comput. 76 (2018); Ranocha (2020) with the
    pressure-equilibrium energy term:
      f_rho = {{rho}}_log {{v.n}},  f_m = f_rho {{v}} + {{p}} n,
      f_E = f_rho (v_L.v_R / 2 + 1 / ((gamma-1) {{rho/p}}_log))
            + (p_L v_R.n + p_R v_L.n) / 2,
    with 1/{{rho/p}}_log = p_L p_R / {{rho_L p_R, rho_R p_L}}_log.
    """
    nd = uL.shape[0] - 2
    rL, vL, pL, _ = _vel_p(uL, gamma)
    rR, vR, pR, _ = _vel_p(uR, gamma)
    vnL = vL[0] * normal[0]
    vnR = vR[0] * normal[0]
    vLvR = vL[0] * vR[0]
    for d in range(1, nd):
        vnL = vnL + vL[d] * normal[d]
        vnR = vnR + vR[d] * normal[d]
        vLvR = vLvR + vL[d] * vR[d]
    rho_mean = ln_mean(rL, rR)
    inv_rho_p_mean = pL * pR * inv_ln_mean(rL * pR, rR * pL)
    p_avg = 0.5 * (pL + pR)
    f1 = rho_mean * 0.5 * (vnL + vnR)
    fm = [f1 * (0.5 * (vL[d] + vR[d])) + p_avg * normal[d] for d in range(nd)]
    fe = f1 * (0.5 * vLvR + inv_rho_p_mean / (gamma - 1.0)) + 0.5 * (pL * vnR + pR * vnL)
    return np.array([f1] + fm + [fe])


def flux_kennedy_gruber(uL, uR, normal, gamma):
    """Kennedy-Gruber split flux (absent in the reference; published formula).

    C. A. Kennedy, A. Gruber, J. Comput. Phys. 227 (2008):
      f_rho = {{rho}}{{v.n}}, f_m = {{rho}}{{v.n}}{{v}} + {{p}} n,
      f_E = ({{rho}}{{e}} + {{p}}) {{v.n}},  e = E / rho.
    """
    nd = uL.shape[0] - 2
    rL, vL, pL, _ = _vel_p(uL, gamma)
    rR, vR, pR, _ = _vel_p(uR, gamma)
    eL = uL[nd + 1] / rL
    eR = uR[nd + 1] / rR
    rho_avg = 0.5 * (rL + rR)
    e_avg = 0.5 * (eL + eR)
    p_avg = 0.5 * (pL + pR)
    v_avg = [0.5 * (vL[d] + vR[d]) for d in range(nd)]
    vn_avg = v_avg[0] * normal[0]
    for d in range(1, nd):
        vn_avg = vn_avg + v_avg[d] * normal[d]
    f1 = rho_avg * vn_avg
    fm = [f1 * v_avg[d] + p_avg * normal[d] for d in range(nd)]
    fe = (rho_avg * e_avg + p_avg) * vn_avg
    return np.array([f1] + fm + [fe])


def flux_hllc(uL, uR, normal, gamma):
    """Normal-rotated HLLC for 2D Euler (absent in the reference in 2D).

    Rotates to the face frame (n_hat, t_hat = (-n_y, n_x)), applies the
    reference's 1D HLLC with Roe-averaged Einfeldt speeds
    (numerical_flux.hpp:283-378) to (rho, rho v_n, rho E) with the tangential
    momentum carried passively (rho v_t)* = rho* v_t, rotates back and scales
    by |n| (Toro, Riemann Solvers, ch. 10).
    """
    assert uL.shape[0] == 4
    nn = np.sqrt(normal[0] * normal[0] + normal[1] * normal[1])
    nx_ = normal[0] / nn
    ny_ = normal[1] / nn

    def rot(u):
        rho = u[0]
        mn = u[1] * nx_ + u[2] * ny_
        mt = -u[1] * ny_ + u[2] * nx_
        return rho, mn, mt, u[3]

    rL, mnL, mtL, EL = rot(uL)
    rR, mnR, mtR, ER = rot(uR)
    vL = mnL / rL
    vR = mnR / rR
    wL = mtL / rL
    wR = mtR / rR
    pL = (gamma - 1.0) * (EL - 0.5 * rL * (vL * vL + wL * wL))
    pR = (gamma - 1.0) * (ER - 0.5 * rR * (vR * vR + wR * wR))
    cL = np.sqrt(gamma * pL / rL)
    cR = np.sqrt(gamma * pR / rR)
    fL = [mnL, mnL * vL + pL, mnL * wL, vL * (EL + pL)]
    fR = [mnR, mnR * vR + pR, mnR * wR, vR * (ER + pR)]
    srL = np.sqrt(rL)
    srR = np.sqrt(rR)
    ssum = srL + srR
    v_roe = (srL * vL + srR * vR) / ssum
    w_roe = (srL * wL + srR * wR) / ssum
    ekin_roe = 0.5 * (v_roe * v_roe + w_roe * w_roe)
    HL = (EL + pL) / rL
    HR = (ER + pR) / rR
    H_roe = (srL * HL + srR * HR) / ssum
    c_roe = np.sqrt((gamma - 1.0) * (H_roe - ekin_roe))
    SL = np.minimum(vL - cL, v_roe - c_roe)
    SR = np.maximum(vR + cR, v_roe + c_roe)
    sMuL = SL - vL
    sMuR = SR - vR
    with np.errstate(divide="ignore", invalid="ignore"):
        SStar = (pR - pL + rL * vL * sMuL - rR * vR * sMuR) / (rL * sMuL - rR * sMuR)
        dL = rL * sMuL / (SL - SStar)
        enL = EL / rL + (SStar - vL) * (SStar + pL / (rL * sMuL))
        dR = rR * sMuR / (SR - SStar)
        enR = ER / rR + (SStar - vR) * (SStar + pR / (rR * sMuR))
    starL = [fL[0] + SL * (dL - rL), fL[1] + SL * (dL * SStar - mnL),
             fL[2] + SL * (dL * wL - mtL), fL[3] + SL * (dL * enL - EL)]
    starR = [fR[0] + SR * (dR - rR), fR[1] + SR * (dR * SStar - mnR),
             fR[2] + SR * (dR * wR - mtR), fR[3] + SR * (dR * enR - ER)]
    out = []
    for q in range(4):
        v = np.where(SL >= 0, fL[q],
                     np.where(SR <= 0, fR[q],
                              np.where((SL <= 0) & (SStar >= 0), starL[q], starR[q])))
        out.append(v)
    fn, ft = out[1], out[2]
    return np.array([out[0] * nn, (fn * nx_ - ft * ny_) * nn, (fn * ny_ + ft * nx_) * nn, out[3] * nn])


VOLUME_FLUXES = {"chandrashekar": flux_chandrashekar, "ranocha": flux_ranocha,
                 "kennedy_gruber": flux_kennedy_gruber}
SURFACE_FLUXES = {"llf": flux_llf, "hllc": flux_hllc}


# ---------------------------------------------------------------------------
# Scheme description and RHS
# ---------------------------------------------------------------------------


@dataclass
class Scheme:
    ndims: int
    polydeg: int
    cells: tuple
    left: tuple
    right: tuple
    periodic: bool = True
    gamma: float = 1.4
    volume_flux: str = "chandrashekar"
    surface_flux: str = "llf"
    shock_capturing: bool = False
    alpha_max: float = 0.5
    alpha_min: float = 0.001
    bc: str = "periodic"            # "periodic" | "dmr"
    viscous: bool = False
    mu: float = 0.0
    prandtl: float = 0.72

    def __post_init__(self):
        self.basis = Basis(self.polydeg)
        per = (self.periodic,) * self.ndims
        if self.ndims == 2:
            self.geo = geometry_2d(self.basis, self.cells, self.left, self.right, per)
        else:
            self.geo = geometry_3d(self.basis, self.cells, self.left, self.right, per)

    @property
    def nvars(self):
        return self.ndims + 2

    @property
    def n(self):
        return self.polydeg + 1


def _grid(s: Scheme, a):
    """View cells+(dof, ...) as cells+(n,)*d+(...) with [.., kn, jn, in, ..]."""
    nd = s.ndims
    cells = a.shape[:nd]
    return a.reshape(cells + (s.n,) * nd + a.shape[nd + 1:])


def hg_alpha(s: Scheme, u, raw: bool = False):
    """subcell_limiting/indicator.hpp:313-428 (2D) / :430-585 (3D).

    Indicator rho*p with gamma fixed to 1.4 (indicator.hpp:137-210).  With
    raw=True the logistic alpha before the alpha_min / alpha_max clipping
    (indicator.hpp:409-416) is returned: the troubled-cell decision is
    raw >= alpha_min, so |raw - alpha_min| is its margin.
    """
    n = s.n
    nd = s.ndims
    U = _grid(s, u)
    rho = U[..., 0]
    vel = [U[..., 1 + d] / rho for d in range(nd)]
    sq = vel[0] * vel[0]
    for d in range(1, nd):
        sq = sq + vel[d] * vel[d]
    p = (1.4 - 1.0) * (U[..., nd + 1] - 0.5 * rho * sq)
    ind = p * rho  # [cells..., (kn,) jn, in]
    V = s.basis.Vinv
    if nd == 2:
        # indicator.hpp:32-67 dimension-wise transform, sequential sums
        tmp = np.zeros_like(ind)
        for i in range(n):
            r = np.zeros(ind.shape[:-1])
            for ii in range(n):
                r = r + V[i, ii] * ind[..., ii]
            tmp[..., i] = r
        modal = np.zeros_like(ind)
        for j in range(n):
            r = np.zeros(ind.shape[:-2] + (n,))
            for jj in range(n):
                r = r + V[j, jj] * tmp[..., jj, :]
            modal[..., j, :] = r
        m2 = modal * modal
        total = np.zeros(ind.shape[:-2]); c1 = np.zeros_like(total); c2 = np.zeros_like(total)
        for j in range(n):
            for i in range(n):
                total = total + m2[..., j, i]
        for j in range(n - 1):
            for i in range(n - 1):
                c1 = c1 + m2[..., j, i]
        for j in range(n - 2):
            for i in range(n - 2):
                c2 = c2 + m2[..., j, i]
    else:
        t1 = np.zeros_like(ind)
        for i in range(n):
            r = np.zeros(ind.shape[:-1])
            for ii in range(n):
                r = r + V[i, ii] * ind[..., ii]
            t1[..., i] = r
        t2 = np.zeros_like(ind)
        for j in range(n):
            r = np.zeros(ind.shape[:-2] + (n,))
            for jj in range(n):
                r = r + V[j, jj] * t1[..., jj, :]
            t2[..., j, :] = r
        modal = np.zeros_like(ind)
        for k in range(n):
            r = np.zeros(ind.shape[:-3] + (n, n))
            for kk in range(n):
                r = r + V[k, kk] * t2[..., kk, :, :]
            modal[..., k, :, :] = r
        m2 = modal * modal
        c2 = np.zeros(ind.shape[:-3])
        for k in range(n - 2):
            for j in range(n - 2):
                for i in range(n - 2):
                    c2 = c2 + m2[..., k, j, i]
        c1 = c2.copy()
        for j in range(n - 1):
            for i in range(n - 1):
                c1 = c1 + m2[..., n - 2, j, i]
        for k in range(n - 2):
            for i in range(n - 1):
                c1 = c1 + m2[..., k, n - 2, i]
        for k in range(n - 2):
            for j in range(n - 2):
                c1 = c1 + m2[..., k, j, n - 2]
        total = c1.copy()
        for j in range(n):
            for i in range(n):
                total = total + m2[..., n - 1, j, i]
        for k in range(n - 1):
            for i in range(n):
                total = total + m2[..., k, n - 1, i]
    with np.errstate(divide="ignore", invalid="ignore"):
        e1 = np.where(total != 0, (total - c1) / total, 0.0)
        e2 = np.where(c1 != 0, (c1 - c2) / c1, 0.0)
    energy = np.maximum(e1, e2)
    threshold = 0.5 * 10.0 ** (-1.8 * float(n) ** 0.25)
    sfac = math.log((1.0 - 0.0001) / 0.0001)
    # libm exp per element (numpy's vectorised exp may differ by an ulp from
    # the C library the reference calls, indicator.hpp:409)
    arg = -sfac / threshold * (energy - threshold)
    ex = np.vectorize(math.exp, otypes=[np.float64])(arg)
    alpha = 1.0 / (1.0 + ex)
    if raw:
        return alpha
    alpha = np.where(alpha < s.alpha_min, 0.0, alpha)
    alpha = np.where(alpha > 1.0 - s.alpha_min, 1.0, alpha)
    return np.minimum(s.alpha_max, alpha)


def hg_atol():
    """volume_flux.hpp:772-773."""
    eps = np.finfo(np.float64).eps
    return max(100.0 * eps, eps ** 0.75)


def _volume_split(s: Scheme, U, JA, scale):
    """volume_flux.hpp:221-294 (2D) / :296-410 (3D): symmetric pair loop.

    Returns sum_k Dsplit(i,k) f(u_i, u_k, (Ja_i+Ja_k)/2) per node, each term
    multiplied by `scale` (the HG (1 - alpha) factor) like the reference.
    """
    n = s.n
    nd = s.ndims
    g = s.gamma
    f = VOLUME_FLUXES[s.volume_flux]
    Ds = s.basis.Dsplit
    du = np.zeros_like(U)
    ax_node = {0: -2, 1: -3, 2: -4}  # node axis of direction d in [.., kn, jn, in, var]
    for d in range(nd):
        ax = ax_node[d]
        for i in range(n):
            for k in range(i + 1, n):
                ui = np.moveaxis(np.take(U, i, axis=ax), -1, 0)
                uk = np.moveaxis(np.take(U, k, axis=ax), -1, 0)
                jai = np.take(JA[..., d, :], i, axis=ax)
                jak = np.take(JA[..., d, :], k, axis=ax)
                normal = np.moveaxis(0.5 * (jai + jak), -1, 0)
                fl = np.moveaxis(f(ui, uk, normal, g), 0, -1)
                sl_i = [slice(None)] * du.ndim
                sl_i[ax] = i
                sl_k = [slice(None)] * du.ndim
                sl_k[ax] = k
                du[tuple(sl_i)] += (scale * Ds[i, k]) * fl
                du[tuple(sl_k)] += (scale * Ds[k, i]) * fl
    return du


def _volume_fv_2d(s: Scheme, U, scale):
    """volume_flux.hpp:449-511 FV subcell integral (2D) with LLF on subcell normals."""
    n = s.n
    g = s.gamma
    iw = s.basis.inv_weights
    n1, n2 = s.geo.subcell
    du = np.zeros_like(U)
    for f in range(1, n):
        uL = np.moveaxis(U[..., :, f - 1, :], -1, 0)
        uR = np.moveaxis(U[..., :, f, :], -1, 0)
        nrm = np.moveaxis(n1[:, :, f - 1, :, :], -1, 0)
        fs = np.moveaxis(flux_llf(uL, uR, nrm, g), 0, -1)
        du[..., :, f - 1, :] += (scale[..., None, None] * iw[f - 1]) * fs
        du[..., :, f, :] -= (scale[..., None, None] * iw[f]) * fs
    for f in range(1, n):
        uL = np.moveaxis(U[..., f - 1, :, :], -1, 0)
        uR = np.moveaxis(U[..., f, :, :], -1, 0)
        nrm = np.moveaxis(n2[:, :, :, f - 1, :], -1, 0)
        fs = np.moveaxis(flux_llf(uL, uR, nrm, g), 0, -1)
        du[..., f - 1, :, :] += (scale[..., None, None] * iw[f - 1]) * fs
        du[..., f, :, :] -= (scale[..., None, None] * iw[f]) * fs
    return du


def dmr_state(x, y, t, gamma):
    """Double Mach reflection state (examples/Euler2D/double_mach_reflection/
    double_mach_reflection_structured.cpp:9-32)."""
    shock = 1.0 / 6.0 + (y + 20.0 * t) / math.sqrt(3.0)
    phi = math.pi / 6.0
    post = prim_to_cons([8.0, 8.25 * math.cos(phi), -8.25 * math.sin(phi), 116.5], gamma)
    pre = prim_to_cons([1.4, 0.0, 0.0, 1.0], gamma)
    x = np.asarray(x, dtype=np.float64)
    return np.array([np.where(x < shock, post[q], pre[q]) for q in range(4)])


def prim_to_cons(prim, gamma):
    """utils/state_conversion.hpp:9-24."""
    nd = len(prim) - 2
    cons = [prim[0]]
    vsq = 0.0
    for d in range(nd):
        cons.append(prim[0] * prim[d + 1])
        vsq = vsq + prim[d + 1] * prim[d + 1]
    cons.append(prim[nd + 1] / (gamma - 1.0) + 0.5 * prim[0] * vsq)
    return cons


def _surface_fluxes(s: Scheme, U, t):
    """Interface + boundary face fluxes, surface_flux(cells, face*n + node, var).

    surface_flux.hpp:45-127 (2D) / :129-271 (3D); boundary faces by
    boundary_set.hpp:70-86 with dirichlet_boundary.hpp:70-120,
    outflow_boundary.hpp:57-110 and dirichlet_boundary.hpp:198-275.
    """
    n = s.n
    nd = s.ndims
    g = s.gamma
    sf = SURFACE_FLUXES[s.surface_flux]
    JA = _grid(s, s.geo.ja)
    cells = U.shape[:nd]
    nv = s.nvars
    if nd == 2:
        nx, ny = cells
        SF = np.zeros((nx, ny, 4, n, nv))
        # x faces: left element ie-1 (node n-1, jn), right element ie (node 0, jn)
        uR = U[:, :, :, 0, :]
        uL = np.roll(U, 1, axis=0)[:, :, :, n - 1, :]
        nrm = JA[:, :, :, 0, 0, :]
        fx = np.moveaxis(sf(np.moveaxis(uL, -1, 0), np.moveaxis(uR, -1, 0), np.moveaxis(nrm, -1, 0), g), 0, -1)
        SF[:, :, 0] = fx
        SF[:, :, 1] = np.roll(fx, -1, axis=0)
        uR = U[:, :, 0, :, :]
        uL = np.roll(U, 1, axis=1)[:, :, n - 1, :, :]
        nrm = JA[:, :, 0, :, 1, :]
        fy = np.moveaxis(sf(np.moveaxis(uL, -1, 0), np.moveaxis(uR, -1, 0), np.moveaxis(nrm, -1, 0), g), 0, -1)
        SF[:, :, 2] = fy
        SF[:, :, 3] = np.roll(fy, -1, axis=1)
        if s.bc == "dmr":
            _dmr_boundary(s, U, JA, SF, t)
        return SF
    nx, ny, nz = cells
    SF = np.zeros((nx, ny, nz, 6, n, n, nv))
    for d, (ax_e, sel_r, sel_l) in enumerate([
            (0, (slice(None),) * 3 + (slice(None), slice(None), 0), (slice(None),) * 3 + (slice(None), slice(None), n - 1)),
            (1, (slice(None),) * 3 + (slice(None), 0, slice(None)), (slice(None),) * 3 + (slice(None), n - 1, slice(None))),
            (2, (slice(None),) * 3 + (0, slice(None), slice(None)), (slice(None),) * 3 + (n - 1, slice(None), slice(None)))]):
        uR = U[sel_r]
        uL = np.roll(U, 1, axis=ax_e)[sel_l]
        nrm = JA[sel_r][..., d, :]
        fl = np.moveaxis(sf(np.moveaxis(uL, -1, 0), np.moveaxis(uR, -1, 0), np.moveaxis(nrm, -1, 0), g), 0, -1)
        SF[:, :, :, 2 * d] = fl
        SF[:, :, :, 2 * d + 1] = np.roll(fl, -1, axis=ax_e)
    return SF


def _dmr_boundary(s: Scheme, U, JA, SF, t):
    """Face BCs of the DMR case: Dirichlet(left), Outflow(right),
    MixedDirichletSlipWall(bottom, Dirichlet for x < 1/6), Dirichlet(top)."""
    n = s.n
    g = s.gamma
    sf = SURFACE_FLUXES[s.surface_flux]
    C = _grid(s, s.geo.coords)
    nx, ny = U.shape[:2]

    def flux(a, b, nrm):
        return np.moveaxis(sf(np.moveaxis(a, -1, 0), np.moveaxis(b, -1, 0), np.moveaxis(nrm, -1, 0), g), 0, -1)

    # face 0 (left, x-dir, inner on the right: flux(outer, inner))
    ui = U[0, :, :, 0, :]
    c = C[0, :, :, 0, :]
    uo = np.moveaxis(dmr_state(c[..., 0], c[..., 1], t, g), 0, -1)
    SF[0, :, 0] = flux(uo, ui, JA[0, :, :, 0, 0, :])
    # face 1 (right): outflow, outer = x-line average, flux(inner, outer)
    ui = U[nx - 1, :, :, n - 1, :]
    avg = np.zeros_like(ui)
    for i in range(n):
        avg = avg + U[nx - 1, :, :, i, :]
    avg = avg / float(n)
    SF[nx - 1, :, 1] = flux(ui, avg, JA[nx - 1, :, :, n - 1, 0, :])
    # face 2 (bottom): mixed Dirichlet / reflecting wall, flux(outer, inner)
    ui = U[:, 0, 0, :, :]
    c = C[:, 0, 0, :, :]
    nrm = JA[:, 0, 0, :, 1, :]
    uo = np.moveaxis(dmr_state(c[..., 0], c[..., 1], t, g), 0, -1)
    rho = ui[..., 0]
    vx = ui[..., 1] / rho
    vy = ui[..., 2] / rho
    nn2 = nrm[..., 0] * nrm[..., 0] + nrm[..., 1] * nrm[..., 1]
    vn = (vx * nrm[..., 0] + vy * nrm[..., 1]) / nn2
    uw = np.stack([rho, rho * (vx - 2.0 * vn * nrm[..., 0]), rho * (vy - 2.0 * vn * nrm[..., 1]), ui[..., 3]], -1)
    use_d = (c[..., 0] < 1.0 / 6.0)[..., None]
    SF[:, 0, 2] = np.where(use_d, flux(uo, ui, nrm), flux(uw, ui, nrm))
    # face 3 (top): Dirichlet, flux(inner, outer)
    ui = U[:, ny - 1, n - 1, :, :]
    c = C[:, ny - 1, n - 1, :, :]
    uo = np.moveaxis(dmr_state(c[..., 0], c[..., 1], t, g), 0, -1)
    SF[:, ny - 1, 3] = flux(ui, uo, JA[:, ny - 1, n - 1, :, 1, :])


def _surface_integral(s: Scheme, du, SF, lift_sign=1.0):
    """surface_integral.hpp:35-80 (2D) / :82-154 (3D)."""
    n = s.n
    lL = s.basis.lhat_left[0]
    lR = s.basis.lhat_right[n - 1]
    if s.ndims == 2:
        du[..., :, 0, :] -= SF[:, :, 0] * lL
        du[..., :, n - 1, :] += SF[:, :, 1] * lR
        du[..., 0, :, :] -= SF[:, :, 2] * lL
        du[..., n - 1, :, :] += SF[:, :, 3] * lR
    else:
        du[..., :, :, 0, :] -= SF[:, :, :, 0] * lL
        du[..., :, :, n - 1, :] += SF[:, :, :, 1] * lR
        du[..., :, 0, :, :] -= SF[:, :, :, 2] * lL
        du[..., :, n - 1, :, :] += SF[:, :, :, 3] * lR
        du[..., 0, :, :, :] -= SF[:, :, :, 4] * lL
        du[..., n - 1, :, :, :] += SF[:, :, :, 5] * lR


def gradient_variables(U, gamma):
    """compressible_navier_stokes2D.hpp:56-69: q = (rho, v1, v2, T=p/rho)."""
    rho = U[..., 0]
    inv_rho = 1.0 / rho
    v1 = U[..., 1] * inv_rho
    v2 = U[..., 2] * inv_rho
    p = (gamma - 1.0) * (U[..., 3] - 0.5 * (U[..., 1] * U[..., 1] + U[..., 2] * U[..., 2]) * inv_rho)
    return np.stack([rho, v1, v2, p * inv_rho], axis=-1)


def br1_gradient(s: Scheme, U):
    """BR1 lifted gradient, 2D periodic (structured_solver.hpp:437-452;
    parabolic_gradient.hpp:480-818).  Returns grad[.., jn, in, var, dim]."""
    n = s.n
    Dh = s.basis.Dhat
    JA = _grid(s, s.geo.ja)
    IJ = _grid(s, s.geo.inv_j)
    q = gradient_variables(U, s.gamma)
    gref = np.zeros(q.shape + (2,))
    # parabolic_gradient.hpp:509-532 weak-form volume term with Dhat
    for i in range(n):
        for ii in range(n):
            gref[..., :, ii, :, 0] += Dh[ii, i] * q[..., :, i, :]
    for jn in range(n):
        for jj in range(n):
            gref[..., jj, :, :, 1] += Dh[jj, jn] * q[..., jn, :, :]
    # :573-585 transform to physical
    ja = JA
    grad = np.zeros_like(gref)
    grad[..., 0] = ja[..., None, 0, 0] * gref[..., 0] + ja[..., None, 1, 0] * gref[..., 1]
    grad[..., 1] = ja[..., None, 0, 1] * gref[..., 0] + ja[..., None, 1, 1] * gref[..., 1]
    # :591-687 interface averages (periodic)
    qx = 0.5 * (np.roll(q, 1, axis=0)[:, :, :, n - 1, :] + q[:, :, :, 0, :])   # face 0 of element
    qy = 0.5 * (np.roll(q, 1, axis=1)[:, :, n - 1, :, :] + q[:, :, 0, :, :])   # face 2
    qx_r = np.roll(qx, -1, axis=0)
    qy_t = np.roll(qy, -1, axis=1)
    lL = s.basis.lhat_left[0]
    lR = s.basis.lhat_right[n - 1]
    # :689-782 lifting with the element's own face normals
    for dim in range(2):
        grad[..., :, 0, :, dim] += (-lL) * qx * JA[..., :, 0, 0, dim][..., None]
        grad[..., :, n - 1, :, dim] += lR * qx_r * JA[..., :, n - 1, 0, dim][..., None]
        grad[..., 0, :, :, dim] += (-lL) * qy * JA[..., 0, :, 1, dim][..., None]
        grad[..., n - 1, :, :, dim] += lR * qy_t * JA[..., n - 1, :, 1, dim][..., None]
    # :784-818 scale by 1/J
    grad *= IJ[..., None, None]
    return grad


def viscous_terms(s: Scheme, U, grad):
    """Viscous weak-form divergence added to du (parabolic_viscous.hpp:343-592,
    structured_solver.hpp:352-361) before the shared -1/J scaling."""
    n = s.n
    g = s.gamma
    mu = s.mu
    kappa = g / ((g - 1.0) * s.prandtl)
    Dh = s.basis.Dhat
    JA = _grid(s, s.geo.ja)
    q = gradient_variables(U, g)
    v1, v2 = q[..., 1], q[..., 2]
    gx, gy = grad[..., 0], grad[..., 1]
    # compressible_navier_stokes2D.hpp:71-106
    tau11 = (4.0 * gx[..., 1] - 2.0 * gy[..., 2]) / 3.0
    tau22 = (4.0 * gy[..., 2] - 2.0 * gx[..., 1]) / 3.0
    tau12 = gy[..., 1] + gx[..., 2]
    q1 = kappa * gx[..., 3]
    q2 = kappa * gy[..., 3]
    zero = np.zeros_like(tau11)
    fx = np.stack([zero, mu * tau11, mu * tau12, mu * (v1 * tau11 + v2 * tau12 + q1)], -1)
    fy = np.stack([zero, mu * tau12, mu * tau22, mu * (v1 * tau12 + v2 * tau22 + q2)], -1)
    Fv = -np.stack([fx, fy], axis=-1)  # stored as -F_v (parabolic_viscous.hpp:383-387)
    du = np.zeros_like(U)
    fxi = JA[..., None, 0, 0] * Fv[..., 0] + JA[..., None, 0, 1] * Fv[..., 1]
    feta = JA[..., None, 1, 0] * Fv[..., 0] + JA[..., None, 1, 1] * Fv[..., 1]
    for i in range(n):
        for ii in range(n):
            du[..., :, ii, :] += Dh[ii, i] * fxi[..., :, i, :]
    for jn in range(n):
        for jj in range(n):
            du[..., jj, :, :] += Dh[jj, jn] * feta[..., jn, :, :]
    # one-sided interface flux: primary (right/upper) element's F_v . n
    fx_face = (Fv[:, :, :, 0, :, 0] * JA[:, :, :, 0, 0, 0][..., None]
               + Fv[:, :, :, 0, :, 1] * JA[:, :, :, 0, 0, 1][..., None])
    fy_face = (Fv[:, :, 0, :, :, 0] * JA[:, :, 0, :, 1, 0][..., None]
               + Fv[:, :, 0, :, :, 1] * JA[:, :, 0, :, 1, 1][..., None])
    SF = np.zeros(U.shape[:2] + (4, n, 4))
    SF[:, :, 0] = fx_face
    SF[:, :, 1] = np.roll(fx_face, -1, axis=0)
    SF[:, :, 2] = fy_face
    SF[:, :, 3] = np.roll(fy_face, -1, axis=1)
    _surface_integral(s, du, SF)
    return du


def rhs(s: Scheme, u, t=0.0, return_alpha=False):
    """StructuredSolver::calc_rhs (structured_solver.hpp:466-480)."""
    U = _grid(s, np.asarray(u, dtype=np.float64))
    JA = _grid(s, s.geo.ja)
    nd = s.ndims
    alpha = None
    if s.shock_capturing:
        alpha = hg_alpha(s, u)
        flagged = np.abs(alpha - 0.0) > hg_atol()
        bshape = alpha.shape + (1,) * nd
        scale_dg = np.where(flagged, 1.0 - alpha, 1.0).reshape(bshape)
        du = _volume_split(s, U, JA, scale_dg)
        if nd != 2:
            raise NotImplementedError("FV subcell integral is restated for 2D")
        du = du + _volume_fv_2d(s, U, np.where(flagged, alpha, 0.0))
    else:
        du = _volume_split(s, U, JA, 1.0)
    SF = _surface_fluxes(s, U, t)
    if s.viscous:
        grad = br1_gradient(s, U)
        du = du + viscous_terms(s, U, grad)
    _surface_integral(s, du, SF)
    du = du * (-_grid(s, s.geo.inv_j))[..., None]
    out = du.reshape(np.asarray(u).shape)
    return (out, alpha) if return_alpha else out


def ssprk3_step(s: Scheme, u, t, dt):
    """SSPRK3::step (time_integrator/SSPRK3.hpp:159-181)."""
    u = np.asarray(u, dtype=np.float64)
    u1 = 1.0 * u + dt * rhs(s, u, t)
    u2 = (3.0 / 4.0) * u + (1.0 / 4.0) * u1 + ((1.0 / 4.0) * dt) * rhs(s, u1, t + dt)
    return (1.0 / 3.0) * u + (2.0 / 3.0) * u2 + ((2.0 / 3.0) * dt) * rhs(s, u2, t + 0.5 * dt)


# ---------------------------------------------------------------------------
# Initial conditions of the benchmark cases (evaluated at node coordinates,
# boundary_condition/initial_functor.hpp:62-118)
# ---------------------------------------------------------------------------


def initial_state(s: Scheme, kind: str, **kw):
    c = s.geo.coords
    g = s.gamma
    if kind == "kh":
        # examples/Euler2D/kelvin_helmholtz_hg/kelvin_helmholtz_hg.cpp
        x, y = c[..., 0], c[..., 1]
        B = np.tanh(15.0 * y + 7.5) - np.tanh(15.0 * y - 7.5)
        rho = 0.5 + 0.75 * B
        v1 = 0.5 * (B - 1.0)
        v2 = 0.1 * np.sin(2.0 * np.pi * x)
        prim = [rho, v1, v2, np.ones_like(rho)]
    elif kind == "tgv3d":
        # examples/Euler3D/inviscid_tgv/inviscid_tgv.cpp:18-35 (Mach 0.1)
        x, y, z = c[..., 0], c[..., 1], c[..., 2]
        rho = np.ones_like(x)
        v1 = np.sin(x) * np.cos(y) * np.cos(z)
        v2 = -np.cos(x) * np.sin(y) * np.cos(z)
        v3 = np.zeros_like(x)
        p = 100.0 / 1.4 + 1.0 / 16.0 * (np.cos(2.0 * x) * np.cos(2.0 * z) + 2.0 * np.cos(2.0 * y)
                                         + 2.0 * np.cos(2.0 * x) + np.cos(2.0 * y) * np.cos(2.0 * z))
        prim = [rho, v1, v2, v3, p]
    elif kind == "dmr":
        return np.moveaxis(dmr_state(c[..., 0], c[..., 1], 0.0, g), 0, -1).copy()
    elif kind == "tgv2d":
        x, y = c[..., 0], c[..., 1]
        p0 = kw.get("p0", 1.0 / (g * 0.01))
        rho = np.ones_like(x)
        v1 = np.sin(x) * np.cos(y)
        v2 = -np.cos(x) * np.sin(y)
        p = p0 + (np.cos(2.0 * x) + np.cos(2.0 * y)) / 4.0
        prim = [rho, v1, v2, p]
    elif kind == "vortex":
        x, y = c[..., 0], c[..., 1]
        beta = kw.get("beta", 5.0)
        x0, y0 = kw.get("center", (0.0, 0.0))
        dx = x - x0
        dy = y - y0
        r2 = dx * dx + dy * dy
        ex = np.exp(1.0 - r2)
        du_ = -beta / (2.0 * np.pi) * np.exp(0.5 * (1.0 - r2)) * dy
        dv_ = beta / (2.0 * np.pi) * np.exp(0.5 * (1.0 - r2)) * dx
        T = 1.0 - (g - 1.0) * beta * beta / (8.0 * g * np.pi * np.pi) * ex
        rho = T ** (1.0 / (g - 1.0))
        prim = [rho, 1.0 + du_, dv_, rho * T]
    else:
        raise ValueError(kind)
    cons = prim_to_cons(prim, g)
    return np.stack(cons, axis=-1)


def volume_averages(s: Scheme, u):
    """(volume, mean kinetic energy, mean entropy) of VolumeAverageEuler
    (analyzer/volume_average_euler.hpp:29-69) with the weights w / |1/J|
    (volume_weighted_analyzer_functor.hpp:80,104); entropy density
    -rho (ln p - gamma ln rho) / (gamma - 1)."""
    U = _grid(s, np.asarray(u))
    w = s.basis.weights
    nd = s.ndims
    if nd == 2:
        W = w[None, :] * w[:, None]
    else:
        W = w[None, None, :] * w[None, :, None] * w[:, None, None]
    IJ = _grid(s, s.geo.inv_j)
    wt = W / np.abs(IJ)
    m2 = 0.0
    for d in range(nd):
        m2 = m2 + U[..., 1 + d] * U[..., 1 + d]
    ke = 0.5 * m2 / U[..., 0]
    p = (s.gamma - 1.0) * (U[..., nd + 1] - ke)
    ent = -U[..., 0] * (np.log(p) - s.gamma * np.log(U[..., 0])) / (s.gamma - 1.0)
    vol = float(np.sum(wt))
    return vol, float(np.sum(wt * ke)) / vol, float(np.sum(wt * ent)) / vol


def kinetic_energy_mean(s: Scheme, u):
    """VolumeAverageEuler kinetic energy with weights w/|1/J|
    (analyzer/volume_average_euler.hpp:9-69, volume_weighted_analyzer_functor.hpp:80,104)."""
    U = _grid(s, np.asarray(u))
    w = s.basis.weights
    nd = s.ndims
    if nd == 2:
        W = w[None, :] * w[:, None]
    else:
        W = w[None, None, :] * w[None, :, None] * w[:, None, None]
    IJ = _grid(s, s.geo.inv_j)
    wt = W / np.abs(IJ)
    ke = 0.0
    for d in range(nd):
        ke = ke + U[..., 1 + d] * U[..., 1 + d]
    ke = 0.5 * ke / U[..., 0]
    return float(np.sum(wt * ke) / np.sum(wt))

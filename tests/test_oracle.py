"""The oracle (numpy restatement) pinned against the reference: the golden
fixtures produced by the unmodified reference solver, and the compiled
reference itself when oracle/_ref is built.  CPU only."""
from __future__ import annotations

import math
import os

import numpy as np
import pytest

from oracle import dgsem_oracle as do
from oracle import ref_binding as rb
from tests._util import RTOL, rel_linf

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

CASE_SCHEMES = {
    "kh": dict(ndims=2, polydeg=3, cells=(8, 8), left=(-1.0, -1.0), right=(1.0, 1.0)),
    "kh_hg": dict(ndims=2, polydeg=3, cells=(8, 8), left=(-1.0, -1.0), right=(1.0, 1.0),
                  shock_capturing=True),
    "dmr": dict(ndims=2, polydeg=3, cells=(24, 6), left=(0.0, 0.0), right=(4.0, 1.0),
                periodic=False, shock_capturing=True, bc="dmr"),
    "tgv": dict(ndims=3, polydeg=3, cells=(4, 4, 4), left=(0.0, 0.0, 0.0),
                right=(2 * math.pi,) * 3),
    "ns": dict(ndims=2, polydeg=4, cells=(6, 6), left=(0.0, 0.0), right=(2 * math.pi,) * 2,
               viscous=True, mu=1.0e-3, prandtl=0.72),
}


@pytest.mark.parametrize("N", range(1, 8))
def test_basis_bitwise_golden(N):
    g = np.load(os.path.join(GOLDEN, f"basis_N{N}.npz"))
    b = do.Basis(N)
    for k in ("nodes", "weights", "inv_weights", "lhat_left", "lhat_right", "D", "Dsplit",
              "Dhat", "Vinv"):
        assert np.array_equal(getattr(b, k), g[k]), k


@pytest.mark.parametrize("name", list(CASE_SCHEMES))
def test_oracle_against_golden(name):
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    s = do.Scheme(**CASE_SCHEMES[name])
    # geometry bitwise (containers/data_container.hpp)
    assert np.array_equal(s.geo.ja, g["ja"])
    assert np.array_equal(s.geo.inv_j, g["inv_j"])
    du, alpha = do.rhs(s, g["u"], float(g["t"]), return_alpha=True)
    assert rel_linf(du, g["du"]) <= RTOL
    if "alpha" in g:
        assert np.array_equal(alpha, g["alpha"])
        assert np.array_equal(alpha > do.hg_atol(), g["alpha"] > do.hg_atol())
    u1 = do.ssprk3_step(s, g["u"], 0.0, float(g["dt"]))
    assert rel_linf(u1, g["u1"]) <= RTOL


@pytest.mark.skipif(not rb.available(), reason="compiled reference (oracle/_ref) not built")
@pytest.mark.parametrize("N", [2, 5])
def test_oracle_against_reference_other_degrees(N):
    """Split form at other degrees, straight from the compiled reference."""
    cells = (5, 4)
    s = do.Scheme(ndims=2, polydeg=N, cells=cells, left=(-5.0, -5.0), right=(5.0, 5.0))
    u = do.initial_state(s, "vortex", beta=4.0, center=(0.5, -1.0))
    rc = rb.RefCase(rb.EULER2D_PERIODIC_SPLIT, N, cells, (-5.0, -5.0), (5.0, 5.0))
    assert rel_linf(do.rhs(s, u, 0.0), rc.rhs(u, 0.0)) <= RTOL


@pytest.mark.skipif(not rb.available(), reason="compiled reference (oracle/_ref) not built")
def test_dmr_flags_against_reference_late_time():
    """Troubled-cell flags on a perturbed DMR state with many flagged cells."""
    kw = CASE_SCHEMES["dmr"]
    s = do.Scheme(**kw)
    u = do.initial_state(s, "dmr")
    rng = np.random.default_rng(7)
    u = u * (1.0 + 0.02 * rng.standard_normal(u.shape))
    rc = rb.RefCase(rb.EULER2D_DMR_HG, 3, kw["cells"], kw["left"], kw["right"])
    a_r = rc.alpha(u)
    a_o = do.hg_alpha(s, u)
    assert np.array_equal(a_o, a_r)
    assert (a_r > do.hg_atol()).sum() > 10


# --------------------------------------------------------------------------
# Known-answer properties of the two-point fluxes the reference does not ship
# (Ranocha, Kennedy-Gruber, 2D HLLC) and of the reference ones.
# --------------------------------------------------------------------------
def _states(nd, npts, seed):
    rng = np.random.default_rng(seed)
    rho = 0.5 + rng.random(npts)
    v = [rng.standard_normal(npts) for _ in range(nd)]
    p = 0.5 + rng.random(npts)
    return np.array(do.prim_to_cons([rho] + v + [p], 1.4))


@pytest.mark.parametrize("nd", [2, 3])
@pytest.mark.parametrize("flux", ["chandrashekar", "ranocha", "kennedy_gruber"])
def test_volume_flux_consistency_and_symmetry(nd, flux):
    f = do.VOLUME_FLUXES[flux]
    u = _states(nd, 64, 1)
    w = _states(nd, 64, 2)
    n = np.random.default_rng(3).standard_normal((nd, 64))
    fuu = f(u, u, n, 1.4)
    assert np.max(np.abs(fuu - do.euler_flux_normal(u, n, 1.4))) <= 1e-12 * np.max(np.abs(fuu))
    assert np.max(np.abs(f(u, w, n, 1.4) - f(w, u, n, 1.4))) <= 1e-12 * np.max(np.abs(fuu))


@pytest.mark.parametrize("nd", [2, 3])
@pytest.mark.parametrize("flux", ["chandrashekar", "ranocha"])
def test_entropy_conservation(nd, flux):
    """Tadmor condition (w_R - w_L) . f* = psi_R - psi_L for the EC fluxes,
    entropy s = -rho * ln(p rho^-gamma) / (gamma - 1), psi = rho v.n."""
    g = 1.4
    uL = _states(nd, 32, 4)
    uR = _states(nd, 32, 5)
    n = np.random.default_rng(6).standard_normal((nd, 32))

    def ent_vars(u):
        rho, v, p, v2 = do._vel_p(u, g)
        s = np.log(p) - g * np.log(rho)
        beta = rho / p
        return np.array([(g - s) / (g - 1.0) - 0.5 * beta * v2] + [beta * vd for vd in v]
                        + [-beta])

    def psi(u):
        rho, v, _, _ = do._vel_p(u, g)
        return rho * sum(v[d] * n[d] for d in range(nd))

    fs = do.VOLUME_FLUXES[flux](uL, uR, n, g)
    lhs = np.sum((ent_vars(uR) - ent_vars(uL)) * fs, axis=0)
    assert np.max(np.abs(lhs - (psi(uR) - psi(uL)))) <= 1e-11


def test_hllc_consistency_and_rotation():
    u = _states(2, 64, 7)
    n = np.random.default_rng(8).standard_normal((2, 64))
    f = do.flux_hllc(u, u, n, 1.4)
    ref = do.euler_flux_normal(u, n, 1.4)
    assert np.max(np.abs(f - ref)) <= 1e-12 * np.max(np.abs(ref))
    # Riemann problem: a right-moving contact keeps mass flux rho_L v_n
    uL = np.array(do.prim_to_cons([1.0, 0.3, 0.1, 1.0], 1.4))[:, None]
    uR = np.array(do.prim_to_cons([0.5, 0.3, -0.2, 1.0], 1.4))[:, None]
    fx = do.flux_hllc(uL, uR, np.array([[1.0], [0.0]]), 1.4)
    assert abs(fx[0, 0] - 0.3) < 1e-12
    # x-normal HLLC equals the unrotated 1D HLLC with a passive transverse momentum
    assert abs(fx[2, 0] - 0.3 * 0.1) < 1e-12


def test_discrete_conservation_periodic():
    """Sum over nodes of w_i J du = 0 for periodic meshes (flux differencing + LLF)."""
    s = do.Scheme(ndims=2, polydeg=3, cells=(6, 5), left=(-1.0, -1.0), right=(1.0, 1.0),
                  volume_flux="ranocha")
    u = do.initial_state(s, "kh")
    du = do.rhs(s, u)
    w = s.basis.weights
    W = (w[None, :] * w[:, None]).reshape(-1)
    tot = np.einsum("ijn,ijnv->v", W[None, None, :] / s.geo.inv_j, du)
    assert np.max(np.abs(tot)) <= 1e-12 * np.max(np.abs(du))


def test_free_stream_preservation_3d():
    s = do.Scheme(ndims=3, polydeg=3, cells=(3, 3, 3), left=(0.0, 0.0, 0.0),
                  right=(2 * math.pi,) * 3)
    u = np.zeros(s.geo.inv_j.shape + (5,))
    u[..., :] = do.prim_to_cons([1.0, 0.3, -0.2, 0.1, 71.4], 1.4)
    assert np.max(np.abs(do.rhs(s, u))) <= 1e-9


# ---- tangent-linear reference (dual-number build of the reference) ---------
from oracle import ref_tlm_binding as tb  # noqa: E402


@pytest.mark.skipif(not (tb.available() and rb.available()),
                    reason="compiled reference (oracle/_ref) not built")
@pytest.mark.parametrize("name", ["kh", "ns"])
def test_tangent_linear_reference_value_and_tangent(name):
    """The dual-number build returns the double build's RHS bit for bit, and
    its tangent matches central differences of the reference RHS at a step
    small enough not to cross the LLF max()/abs() kinks."""
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    c = CASE_SCHEMES[name]
    kind = tb.NS2D if c.get("viscous") else tb.EULER2D
    tc = tb.TangentCase(kind, c["polydeg"], c["cells"], c["left"], c["right"], 1.4,
                        c.get("mu", 0.0), c.get("prandtl", 0.72))
    ref = rb.RefCase(kind=rb.NS2D_PERIODIC_SPLIT if c.get("viscous") else
                     rb.EULER2D_PERIODIC_SPLIT, polydeg=c["polydeg"], n_cells=c["cells"],
                     left=c["left"], right=c["right"], mu=c.get("mu", 0.0),
                     prandtl=c.get("prandtl", 0.72))
    u = np.ascontiguousarray(g["u"])
    t = float(g["t"])
    rng = np.random.default_rng(5)
    d = rng.standard_normal(u.shape)
    r, dr = tc.rhs(u, d, t)
    assert np.array_equal(r, ref.rhs(u, t))
    h = 1.0e-9
    fd = (ref.rhs(u + h * d, t) - ref.rhs(u - h * d, t)) / (2.0 * h)
    assert np.max(np.abs(fd - dr)) <= 1e-5 * np.max(np.abs(dr))


# --------------------------------------------------------------------------
# Kennedy-Gruber known-answer vectors (C. A. Kennedy, A. Gruber, J. Comput.
# Phys. 227 (2008), eq. for the split convective flux with arithmetic means):
#   f_rho = {{rho}} {{v.n}},  f_m = f_rho {{v}} + {{p}} n,
#   f_E = ({{rho}} {{e}} + {{p}}) {{v.n}},  e = E / rho,
# evaluated in exact rational arithmetic on rational states (gamma = 7/5).
# --------------------------------------------------------------------------
def _kg_exact(primL, primR, normal, gamma):
    from fractions import Fraction as F
    nd = len(normal)

    def cons(prim):
        rho, v, p = prim[0], prim[1:1 + nd], prim[1 + nd]
        E = p / (gamma - 1) + F(1, 2) * rho * sum(x * x for x in v)
        return rho, v, p, E / rho

    rL, vL, pL, eL = cons(primL)
    rR, vR, pR, eR = cons(primR)
    half = F(1, 2)
    rho_a, e_a, p_a = half * (rL + rR), half * (eL + eR), half * (pL + pR)
    va = [half * (vL[d] + vR[d]) for d in range(nd)]
    vn = sum(va[d] * normal[d] for d in range(nd))
    f1 = rho_a * vn
    return [f1] + [f1 * va[d] + p_a * normal[d] for d in range(nd)] + [(rho_a * e_a + p_a) * vn]


@pytest.mark.parametrize("nd", [2, 3])
def test_kennedy_gruber_known_answer(nd):
    from fractions import Fraction as F
    gamma = F(7, 5)
    if nd == 2:
        primL = [F(1), F(1, 2), F(-1, 4), F(1)]
        primR = [F(2), F(-1, 2), F(1), F(3, 2)]
        normal = [F(3, 4), F(-1, 8)]
    else:
        primL = [F(1), F(1, 2), F(-1, 4), F(3, 8), F(1)]
        primR = [F(5, 4), F(-1, 2), F(1), F(-1, 16), F(3, 2)]
        normal = [F(3, 4), F(-1, 8), F(1, 2)]
    exact = [float(x) for x in _kg_exact(primL, primR, normal, gamma)]
    uL = np.array(do.prim_to_cons([np.array([float(x)]) for x in primL], 1.4))
    uR = np.array(do.prim_to_cons([np.array([float(x)]) for x in primR], 1.4))
    n = np.array([[float(x)] for x in normal])
    got = do.flux_kennedy_gruber(uL, uR, n, 1.4)[:, 0]
    scale = max(abs(x) for x in exact)
    assert np.max(np.abs(got - np.array(exact))) <= 4e-16 * scale, (got, exact)
    # the 2D vector worked by hand: {{rho}} = 3/2, {{v}} = (0, 3/8), {{p}} = 5/4,
    # {{v.n}} = -3/64, e_L = 85/32, e_R = 5/2, {{e}} = 165/64
    if nd == 2:
        assert _kg_exact(primL, primR, normal, gamma) == [
            F(-9, 128), F(15, 16), F(-187, 1024), F(-1965, 8192)]

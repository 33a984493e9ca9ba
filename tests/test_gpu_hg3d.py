"""Hennemann-Gassner shock capturing in 3D (subcell_limiting/indicator.hpp:
430-585, space_integral/volume_flux.hpp:513-630) on the node-parallel launch
shapes, against the compiled reference's VolumeIntegralShockCapturingHG:
identical troubled-cell flags and alpha, RHS within max(1e-12, the
reference's self-variation), on perturbed Taylor-Green states (4^3 at every
degree, 16^3 at N = 3 with every volume flux)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import dgsem_oracle as do
from oracle import ref_binding as rb
from tests._util import RTOL, alpha_ref_to_dev, dev_to_ref, ref_to_dev, rel_linf

pytestmark = pytest.mark.gpu

VFC = {"chandrashekar": 0, "ranocha": 1, "kennedy_gruber": 2}


def _case(N, cells, vf, noise, seed=5):
    import dgsem_b200 as D
    left, right = (0.0,) * 3, (2 * math.pi,) * 3
    s = do.Scheme(ndims=3, polydeg=N, cells=cells, left=left, right=right)
    u = do.initial_state(s, "tgv3d")
    u = u * (1.0 + noise * np.random.default_rng(seed).standard_normal(u.shape))
    mesh = D.StructuredMesh(left, right, cells)
    flux = {"chandrashekar": D.ChandrashekarFlux, "ranocha": D.RanochaFlux,
            "kennedy_gruber": D.KennedyGruberFlux}[vf]
    basis = D.LobattoLegendreBasis(N)
    solver = D.StructuredSolver(D.CompressibleEuler3D(1.4), basis,
                                D.VolumeIntegralShockCapturingHG(flux), D.LaxFriedrichsFlux(),
                                mesh, D.BoundarySet(*[D.PeriodicBC() for _ in range(6)]))
    solver.set_indicator_parameters(0.5, 0.001, False)
    kw = dict(volume_flux=VFC[vf])
    rc = rb.RefCase(rb.EULER3D_PERIODIC_HG, N, cells, left, right, **kw)
    rcf = rb.RefCase(rb.EULER3D_PERIODIC_HG, N, cells, left, right, build="fma", **kw)
    return s, np.ascontiguousarray(u), solver, rc, rcf


def _check(N, cells, vf, noise, cuda, min_flagged):
    import torch
    if not rb.available() or not rb.available("fma"):
        pytest.skip("compiled reference not built")
    s, u, solver, rc, rcf = _case(N, cells, vf, noise)
    ud = torch.from_numpy(ref_to_dev(u, 3)).to(cuda)
    # flags and alpha
    alpha, flags = solver.indicator(ud)
    torch.cuda.synchronize()
    a_r = alpha_ref_to_dev(rc.alpha(u))
    f_r = a_r > do.hg_atol()
    f_d = flags.cpu().numpy().astype(bool)
    assert np.array_equal(f_d, f_r), int((f_d != f_r).sum())
    assert np.max(np.abs(alpha.cpu().numpy() - a_r)) <= 1e-14
    assert f_r.sum() >= min_flagged, int(f_r.sum())
    # the oracle's 3D energies agree with the reference as well
    assert np.array_equal(alpha_ref_to_dev(do.hg_alpha(s, u)) > do.hg_atol(), f_r)
    # RHS for every launch shape
    du_r = rc.rhs(u, 0.0)
    bar = max(RTOL, rel_linf(rcf.rhs(u, 0.0), du_r))
    du = torch.empty_like(ud)
    for v in range(5):
        solver.set_launch_variant(v)
        solver.rhs(ud, du, 0.0)
        torch.cuda.synchronize()
        err = rel_linf(dev_to_ref(du.cpu().numpy(), cells), du_r)
        print(f"\n  N={N} {vf} shape {v}: {err:.3e} (bar {bar:.3e}, flagged {int(f_r.sum())})")
        assert err <= bar, (v, err, bar)


@pytest.mark.parametrize("N", [1, 2, 3, 4])
def test_hg3d_small_every_degree(N, cuda):
    _check(N, (4, 3, 3), "chandrashekar", 0.05, cuda, min_flagged=5)


@pytest.mark.parametrize("vf", ["chandrashekar", "ranocha", "kennedy_gruber"])
def test_hg3d_tgv16_perturbed(vf, cuda):
    _check(3, (16, 16, 16), vf, 0.02, cuda, min_flagged=20)

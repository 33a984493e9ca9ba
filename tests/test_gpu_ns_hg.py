"""2D Navier-Stokes with Hennemann-Gassner shock capturing, the reference's
viscous Kelvin-Helmholtz setup (examples/NavierStokes2D/KHI/viscous_khi.cpp:
CompressibleNavierStokes2D, VolumeIntegralShockCapturingHG with Chandrashekar
and LLF, HGIndicator<Basis, NS2D>), against the compiled reference
(REF_NS2D_PERIODIC_HG): identical alpha and troubled-cell flags, the RHS for
every launch shape within max(1e-12, the reference's self-variation), the
viscous part separately, and SSPRK3 steps.  The blend (1 - alpha) DG +
alpha FV covers the inviscid volume integral only; the viscous terms are
added unblended, as in the reference."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from oracle import dgsem_oracle as do
from oracle import ref_binding as rb
from tests._util import RTOL, alpha_ref_to_dev, dev_to_ref, ref_to_dev, rel_linf

pytestmark = pytest.mark.gpu

LEFT, RIGHT, PR = (-1.0, -1.0), (1.0, 1.0), 0.72


def _state(N, cells, seed=2):
    s = do.Scheme(ndims=2, polydeg=N, cells=cells, left=LEFT, right=RIGHT)
    u = do.initial_state(s, "kh")
    rng = np.random.default_rng(seed)
    return s, np.ascontiguousarray(u * (1.0 + 0.01 * rng.standard_normal(u.shape)))


def _solver(N, cells, mu):
    import dgsem_b200 as D
    mesh = D.StructuredMesh(LEFT, RIGHT, cells)
    solver = D.StructuredSolver(D.CompressibleNavierStokes2D(1.4, mu, PR), D.LobattoLegendreBasis(N),
                                D.VolumeIntegralShockCapturingHG(D.ChandrashekarFlux),
                                D.LaxFriedrichsFlux(), mesh,
                                D.BoundarySet(*[D.PeriodicBC() for _ in range(4)]))
    solver.set_indicator_parameters(0.5, 0.001, False)
    return solver


def _need_ref():
    if not rb.available() or not rb.available("fma"):
        pytest.skip("compiled reference not built")


@pytest.mark.parametrize("N,cells,mu", [(3, (16, 16), 1.0e-3), (2, (12, 10), 5.0e-3),
                                        (4, (10, 12), 1.0e-3)])
def test_ns_hg_matches_reference(N, cells, mu, cuda):
    import torch
    _need_ref()
    s, u = _state(N, cells)
    kw = dict(mu=mu, prandtl=PR, alpha_max=0.5, alpha_min=0.001)
    rc = rb.RefCase(rb.NS2D_PERIODIC_HG, N, cells, LEFT, RIGHT, **kw)
    rcf = rb.RefCase(rb.NS2D_PERIODIC_HG, N, cells, LEFT, RIGHT, build="fma", **kw)
    rc0 = rb.RefCase(rb.NS2D_PERIODIC_HG, N, cells, LEFT, RIGHT,
                     **dict(kw, mu=0.0))
    solver, solver0 = _solver(N, cells, mu), _solver(N, cells, 0.0)
    ud = torch.from_numpy(ref_to_dev(u, 2)).to(cuda)
    # alpha and troubled-cell flags (the indicator ignores the viscosity)
    alpha, flags = solver.indicator(ud)
    torch.cuda.synchronize()
    a_r = alpha_ref_to_dev(rc.alpha(u))
    f_r = a_r > do.hg_atol()
    assert np.array_equal(flags.cpu().numpy().astype(bool), f_r)
    assert np.max(np.abs(alpha.cpu().numpy() - a_r)) <= 1e-14
    assert f_r.sum() >= 4, int(f_r.sum())  # the shear layers are flagged
    # the RHS and its viscous part
    du_r = rc.rhs(u, 0.0)
    visc_r = du_r - rc0.rhs(u, 0.0)
    bar = max(RTOL, rel_linf(rcf.rhs(u, 0.0), du_r))
    du, du0 = torch.empty_like(ud), torch.empty_like(ud)
    for v in range(5):  # 0-2 run the node-parallel shape with both terms
        solver.set_launch_variant(v)
        solver0.set_launch_variant(v)
        solver.rhs(ud, du, 0.0)
        solver0.rhs(ud, du0, 0.0)
        torch.cuda.synchronize()
        got = dev_to_ref(du.cpu().numpy(), cells)
        err = rel_linf(got, du_r)
        verr = rel_linf(got - dev_to_ref(du0.cpu().numpy(), cells), visc_r)
        print(f"\n  N={N} {cells} shape {v}: {err:.3e} (bar {bar:.3e}), viscous part {verr:.3e},"
              f" flagged {int(f_r.sum())}")
        assert err <= bar, (v, err, bar)
        assert verr <= 1e-10, (v, verr)


def test_ns_hg_steps_match_reference(cuda):
    import torch

    from dgsem_b200 import _capi as C
    _need_ref()
    N, cells, mu = 3, (16, 16), 1.0e-3
    _, u = _state(N, cells, seed=9)
    rc = rb.RefCase(rb.NS2D_PERIODIC_HG, N, cells, LEFT, RIGHT, mu=mu, prandtl=PR,
                    alpha_max=0.5, alpha_min=0.001)
    dt = 2e-4
    u5 = rc.ssprk3(u, 0.0, dt, 5)
    solver = _solver(N, cells, mu)
    ud = torch.from_numpy(ref_to_dev(u, 2)).to(cuda)
    C.check(C.lib().dgsem_ssprk3_steps(solver.handle, ctypes.c_void_p(ud.data_ptr()), 0.0, dt, 5),
            "steps")
    torch.cuda.synchronize()
    ud5 = dev_to_ref(ud.cpu().numpy(), cells)
    assert rel_linf(ud5 - u, u5 - u) <= 1e-9
    assert rel_linf(ud5, u5) <= RTOL
    solver.check_finite()

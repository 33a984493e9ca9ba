"""3D Navier-Stokes (equations/compressible_navier_stokes3D.hpp, BR1 gradient
parabolic_gradient.hpp 3D functors, viscous flux parabolic_viscous.hpp) on
periodic boxes, against the compiled reference's StructuredSolver with
CompressibleNavierStokes3D, Chandrashekar split form and LLF
(REF_NS3D_PERIODIC_SPLIT): the RHS for every launch shape within
max(1e-12, the reference's self-variation), its viscous part (RHS at mu
minus RHS at mu = 0) separately to 1e-10 of its own size, and SSPRK3 steps."""
from __future__ import annotations

import ctypes
import math

import numpy as np
import pytest

from oracle import ref_binding as rb
from tests._util import RTOL, dev_to_ref, ref_to_dev, rel_linf

pytestmark = pytest.mark.gpu

LEFT, RIGHT = (0.0,) * 3, (2 * math.pi,) * 3
PR = 0.72


def _state(N, cells, seed=3):
    """A perturbed Mach-0.1 Taylor-Green vortex on the reference's node
    coordinates (cells..., node, var)."""
    from oracle import dgsem_oracle as do
    s = do.Scheme(ndims=3, polydeg=N, cells=cells, left=LEFT, right=RIGHT)
    u = do.initial_state(s, "tgv3d")
    rng = np.random.default_rng(seed)
    return np.ascontiguousarray(u * (1.0 + 0.01 * rng.standard_normal(u.shape)))


def _solver(N, cells, mu):
    import dgsem_b200 as D
    mesh = D.StructuredMesh(LEFT, RIGHT, cells)
    eq = D.CompressibleNavierStokes3D(1.4, mu, PR)
    return D.StructuredSolver(eq, D.LobattoLegendreBasis(N),
                              D.VolumeIntegralSplitForm(D.ChandrashekarFlux),
                              D.LaxFriedrichsFlux(), mesh,
                              D.BoundarySet(*[D.PeriodicBC() for _ in range(6)]))


def _need_ref():
    if not rb.available() or not rb.available("fma"):
        pytest.skip("compiled reference not built")


@pytest.mark.parametrize("N,cells,mu", [(1, (4, 3, 3), 0.05), (2, (4, 3, 3), 0.05),
                                        (3, (4, 3, 3), 0.05), (4, (3, 3, 2), 0.05),
                                        (3, (8, 8, 8), 1.0 / 160.0)])
def test_ns3d_rhs_matches_reference(N, cells, mu, cuda):
    import torch
    _need_ref()
    u = _state(N, cells)
    kw = dict(mu=mu, prandtl=PR)
    rc = rb.RefCase(rb.NS3D_PERIODIC_SPLIT, N, cells, LEFT, RIGHT, **kw)
    rcf = rb.RefCase(rb.NS3D_PERIODIC_SPLIT, N, cells, LEFT, RIGHT, build="fma", **kw)
    rc0 = rb.RefCase(rb.NS3D_PERIODIC_SPLIT, N, cells, LEFT, RIGHT, mu=0.0, prandtl=PR)
    du_r = rc.rhs(u, 0.0)
    visc_r = du_r - rc0.rhs(u, 0.0)
    bar = max(RTOL, rel_linf(rcf.rhs(u, 0.0), du_r))
    solver, solver0 = _solver(N, cells, mu), _solver(N, cells, 0.0)
    ud = torch.from_numpy(ref_to_dev(u, 3)).to(cuda)
    du, du0 = torch.empty_like(ud), torch.empty_like(ud)
    solver0.rhs(ud, du0, 0.0)
    for v in range(5):  # 0-2 run the node-parallel shape in 3D with viscous terms
        solver.set_launch_variant(v)
        solver0.set_launch_variant(v)
        solver.rhs(ud, du, 0.0)
        solver0.rhs(ud, du0, 0.0)
        torch.cuda.synchronize()
        got = dev_to_ref(du.cpu().numpy(), cells)
        err = rel_linf(got, du_r)
        visc = got - dev_to_ref(du0.cpu().numpy(), cells)
        verr = rel_linf(visc, visc_r)
        print(f"\n  N={N} {cells} shape {v}: {err:.3e} (bar {bar:.3e}), viscous part {verr:.3e}")
        assert err <= bar, (v, err, bar)
        assert verr <= 1e-10, (v, verr)
    assert float(np.abs(visc_r).max()) > 1e-3 * float(np.abs(du_r).max())  # viscosity matters


def test_ns3d_steps_match_reference(cuda):
    import torch

    from dgsem_b200 import _capi as C
    _need_ref()
    N, cells, mu = 3, (4, 4, 4), 0.02
    u = _state(N, cells, seed=7)
    rc = rb.RefCase(rb.NS3D_PERIODIC_SPLIT, N, cells, LEFT, RIGHT, mu=mu, prandtl=PR)
    dt = 2e-4
    u5 = rc.ssprk3(u, 0.0, dt, 5)
    solver = _solver(N, cells, mu)
    ud = torch.from_numpy(ref_to_dev(u, 3)).to(cuda)
    C.check(C.lib().dgsem_ssprk3_steps(solver.handle, ctypes.c_void_p(ud.data_ptr()), 0.0, dt, 5),
            "steps")
    torch.cuda.synchronize()
    ud5 = dev_to_ref(ud.cpu().numpy(), cells)
    assert rel_linf(ud5 - u, u5 - u) <= 1e-9
    assert rel_linf(ud5, u5) <= RTOL
    solver.check_finite()


def test_ns3d_rejects_walls_and_shock_capturing():
    import dgsem_b200 as D
    from dgsem_b200 import _capi as C
    mesh = D.StructuredMesh(LEFT, RIGHT, (2, 2, 2))
    eq = D.CompressibleNavierStokes3D()
    bcs = [D.PeriodicBC() for _ in range(6)]
    bcs[2] = bcs[3] = D.NSNoSlipAdiabaticWallBC()
    with pytest.raises(C.DgsemError):
        D.StructuredSolver(eq, D.LobattoLegendreBasis(3),
                           D.VolumeIntegralSplitForm(D.ChandrashekarFlux),
                           D.LaxFriedrichsFlux(), mesh, D.BoundarySet(*bcs))
    with pytest.raises(C.DgsemError):
        D.StructuredSolver(eq, D.LobattoLegendreBasis(3),
                           D.VolumeIntegralShockCapturingHG(D.ChandrashekarFlux),
                           D.LaxFriedrichsFlux(), mesh,
                           D.BoundarySet(*[D.PeriodicBC() for _ in range(6)]))

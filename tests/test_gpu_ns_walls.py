"""Navier-Stokes with adiabatic walls (boundary_condition/navier_stokes_wall_
boundary.hpp): a channel periodic in x with a no-slip wall at the bottom and
a slip wall at the top, against the compiled reference's
NSNoSlipAdiabaticWallBC / NSSlipAdiabaticWallBC (BR1 gradient wall values,
reflected inviscid state, wall viscous fluxes): RHS for every launch shape
and five SSPRK3 steps within max(1e-12, the reference's self-variation)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import dgsem_oracle as do
from oracle import ref_binding as rb
from tests._util import RTOL, dev_to_ref, ref_to_dev, rel_linf

pytestmark = pytest.mark.gpu

CELLS, LEFT, RIGHT, N = (8, 6), (0.0, 0.0), (2 * math.pi, math.pi), 4
MU, PR = 1.0e-2, 0.72


def _state():
    s = do.Scheme(ndims=2, polydeg=N, cells=CELLS, left=LEFT, right=RIGHT, periodic=False)
    x, y = s.geo.coords[..., 0], s.geo.coords[..., 1]
    rho = 1.0 + 0.1 * np.sin(x) * np.sin(y)
    v1 = np.sin(y) * (1.0 + 0.2 * np.cos(x))
    v2 = 0.1 * np.sin(y) * np.sin(2 * x)
    p = 10.0 + 0.5 * np.cos(x) * np.cos(y)
    u = np.stack([rho, rho * v1, rho * v2, p / 0.4 + 0.5 * rho * (v1 * v1 + v2 * v2)], axis=-1)
    return np.ascontiguousarray(u)


def _solver():
    import dgsem_b200 as D
    mesh = D.StructuredMesh(LEFT, RIGHT, CELLS)
    eq = D.CompressibleNavierStokes2D(1.4, MU, PR)
    basis = D.LobattoLegendreBasis(N)
    bcs = D.BoundarySet(D.PeriodicBC(), D.PeriodicBC(), D.NSNoSlipAdiabaticWallBC(),
                        D.NSSlipAdiabaticWallBC())
    return D.StructuredSolver(eq, basis, D.VolumeIntegralSplitForm(D.ChandrashekarFlux),
                              D.LaxFriedrichsFlux(), mesh, bcs)


def test_ns_channel_walls_match_reference(cuda):
    import ctypes

    import torch

    from dgsem_b200 import _capi as C
    if not rb.available() or not rb.available("fma"):
        pytest.skip("compiled reference not built")
    u = _state()
    kw = dict(mu=MU, prandtl=PR)
    rc = rb.RefCase(rb.NS2D_CHANNEL_WALLS, N, CELLS, LEFT, RIGHT, **kw)
    rcf = rb.RefCase(rb.NS2D_CHANNEL_WALLS, N, CELLS, LEFT, RIGHT, build="fma", **kw)
    du_r = rc.rhs(u, 0.0)
    bar = max(RTOL, rel_linf(rcf.rhs(u, 0.0), du_r))
    solver = _solver()
    ud = torch.from_numpy(ref_to_dev(u, 2)).to(cuda)
    du = torch.empty_like(ud)
    for v in range(5):
        solver.set_launch_variant(v)
        solver.rhs(ud, du, 0.0)
        torch.cuda.synchronize()
        err = rel_linf(dev_to_ref(du.cpu().numpy(), CELLS), du_r)
        print(f"\n  shape {v}: {err:.3e} (bar {bar:.3e})")
        assert err <= bar, (v, err)
    # five SSPRK3 steps against the reference's SSPRK3
    dt = 2e-4
    u5 = rc.ssprk3(u, 0.0, dt, 5)
    C.check(C.lib().dgsem_ssprk3_steps(solver.handle, ctypes.c_void_p(ud.data_ptr()), 0.0, dt, 5),
            "steps")
    torch.cuda.synchronize()
    ud5 = dev_to_ref(ud.cpu().numpy(), CELLS)
    assert rel_linf(ud5 - u, u5 - u) <= 1e-9
    assert rel_linf(ud5, u5) <= RTOL

"""Fused per-step diagnostics (dgsem_set_diagnostics / dgsem_diagnostics):
the volume, mean kinetic energy and mean entropy that the stage-3 epilogue
integrates block by block equal the oracle's VolumeAverageEuler
(analyzer/volume_average_euler.hpp:29-69) of the same state, for every launch
shape; the stepped state is bit for bit the same with the diagnostics on and
off; the second pass is deterministic."""
from __future__ import annotations

import ctypes
import math

import numpy as np
import pytest

from oracle import dgsem_oracle as do
from tests._util import dev_to_ref

pytestmark = pytest.mark.gpu

CASES = {
    "tgv": dict(nd=3, N=3, cells=(6, 5, 4), left=(0.0,) * 3, right=(2 * math.pi,) * 3,
                vf="kennedy_gruber", ic="tgv3d", dt=1e-3),
    "kh": dict(nd=2, N=3, cells=(12, 10), left=(-1.0, -1.0), right=(1.0, 1.0),
               vf="ranocha", ic="kh", dt=1e-3),
    "ns": dict(nd=2, N=4, cells=(6, 6), left=(0.0, 0.0), right=(2 * math.pi,) * 2,
               vf="chandrashekar", ic="tgv2d", dt=1e-3, ns=True),
}


def _solver(c):
    import dgsem_b200 as D
    mesh = D.StructuredMesh(c["left"], c["right"], c["cells"])
    if c.get("ns"):
        eq = D.CompressibleNavierStokes2D(1.4, 1e-3, 0.72)
    else:
        eq = D.CompressibleEuler3D(1.4) if c["nd"] == 3 else D.CompressibleEuler2D(1.4)
    flux = {"chandrashekar": D.ChandrashekarFlux, "ranocha": D.RanochaFlux,
            "kennedy_gruber": D.KennedyGruberFlux}[c["vf"]]
    basis = D.LobattoLegendreBasis(c["N"])
    solver = D.StructuredSolver(eq, basis, D.VolumeIntegralSplitForm(flux),
                                D.LaxFriedrichsFlux(), mesh,
                                D.BoundarySet(*[D.PeriodicBC() for _ in range(2 * c["nd"])]))
    sol = D.Solution(mesh, basis, eq)
    ic = {"tgv3d": D.InviscidTaylorGreenVortex(), "kh": D.KelvinHelmholtzInitial(),
          "tgv2d": D.TaylorGreenVortex2D()}[c["ic"]]
    solver.initialize(ic, sol)
    return solver, sol


@pytest.mark.parametrize("name", list(CASES))
def test_fused_diagnostics_match_oracle(name, cuda):
    import torch

    from dgsem_b200 import _capi as C
    L = C.lib()
    c = CASES[name]
    s = do.Scheme(ndims=c["nd"], polydeg=c["N"], cells=c["cells"], left=c["left"],
                  right=c["right"])
    solver, sol = _solver(c)
    u0 = sol.u.clone()
    ref = sol.u.clone()
    p = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    # diagnostics off: reference trajectory
    C.check(L.dgsem_ssprk3_steps(solver.handle, p(ref), 0.0, c["dt"], 3), "steps")
    C.check(L.dgsem_set_diagnostics(solver.handle, 1), "enable")
    for v in range(7):
        if L.dgsem_set_launch_variant(solver.handle, v) != C.DGSEM_OK:
            continue  # shape not available for this scheme
        sol.u.copy_(u0)
        C.check(L.dgsem_ssprk3_steps(solver.handle, p(sol.u), 0.0, c["dt"], 3), "steps")
        vol, ke, ent = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        C.check(L.dgsem_diagnostics(solver.handle, ctypes.byref(vol), ctypes.byref(ke),
                                    ctypes.byref(ent)), "diagnostics")
        torch.cuda.synchronize()
        u = dev_to_ref(sol.u.cpu().numpy(), c["cells"])
        v_o, ke_o, ent_o = do.volume_averages(s, u)
        assert abs(vol.value - v_o) <= 1e-13 * v_o, (v, vol.value, v_o)
        assert abs(ke.value - ke_o) <= 1e-12 * abs(ke_o), (v, ke.value, ke_o)
        assert abs(ent.value - ent_o) <= 1e-12 * abs(ent_o), (v, ent.value, ent_o)
        if v == 0:
            first = (vol.value, ke.value, ent.value)
            assert torch.equal(sol.u, ref)  # the diagnostics change no state bit
        # deterministic second pass
        vol2, ke2, ent2 = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        C.check(L.dgsem_diagnostics(solver.handle, ctypes.byref(vol2), ctypes.byref(ke2),
                                    ctypes.byref(ent2)), "diagnostics")
        assert (vol2.value, ke2.value, ent2.value) == (vol.value, ke.value, ent.value)
    assert first[0] > 0
    C.check(L.dgsem_set_diagnostics(solver.handle, 0), "disable")
    assert L.dgsem_diagnostics(solver.handle, None, None, None) == C.DGSEM_ERR_INVALID_ARG

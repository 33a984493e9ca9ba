"""Allocation-free SSPRK3 step (dgsem_ssprk3_step_static_scratch) against the
context-temporaries step (dgsem_ssprk3_step), both called through the C ABI.

The two entry points launch the same stage kernels, so the states agree to
the parity tolerance RTOL (in practice bit for bit) after each of two calls
in a row.  The file sorts last so the test also runs after every other GPU
test in one process; it passes alone as well.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from tests._util import RTOL, rel_linf

pytestmark = pytest.mark.gpu


def _case(name):
    import dgsem_b200 as D
    if name == "kh":
        mesh = D.StructuredMesh((-1.0, -1.0), (1.0, 1.0), (8, 8))
        eq, basis = D.CompressibleEuler2D(1.4), D.LobattoLegendreBasis(3)
        vi = D.VolumeIntegralSplitForm(D.ChandrashekarFlux)
        sf, bcs = D.LaxFriedrichsFlux(), D.BoundarySet(*[D.PeriodicBC() for _ in range(4)])
        ic, dt = D.KelvinHelmholtzInitial(), 1e-3
    elif name == "tgv":
        pi = float(np.pi)
        mesh = D.StructuredMesh((-pi,) * 3, (pi,) * 3, (4, 4, 4))
        eq, basis = D.CompressibleEuler3D(1.4), D.LobattoLegendreBasis(3)
        vi = D.VolumeIntegralSplitForm(D.KennedyGruberFlux)
        sf, bcs = D.LaxFriedrichsFlux(), D.BoundarySet(*[D.PeriodicBC() for _ in range(6)])
        ic, dt = D.InviscidTaylorGreenVortex(), 1e-2
    else:  # double Mach reflection with shock capturing and time-dependent BCs
        mesh = D.StructuredMesh((0.0, 0.0), (4.0, 1.0), (16, 4))
        eq, basis = D.CompressibleEuler2D(1.4), D.LobattoLegendreBasis(3)
        vi = D.VolumeIntegralShockCapturingHG(D.ChandrashekarFlux)
        sf = D.HLLCFlux()
        bcs = D.BoundarySet(D.DirichletBC("double_mach"), D.OutflowBC(),
                            D.MixedDirichletSlipWallBC("double_mach"),
                            D.DirichletBC("double_mach"))
        ic, dt = D.DoubleMachReflectionInitial(), 1e-4
    solver = D.StructuredSolver(eq, basis, vi, sf, mesh, bcs)
    sol = D.Solution(mesh, basis, eq)
    solver.initialize(ic, sol)
    return solver, sol, dt


@pytest.mark.parametrize("name", ["kh", "tgv", "dmr"])
def test_static_scratch_step_matches_step(name, cuda):
    import torch

    from dgsem_b200 import _capi as C
    L = C.lib()
    solver, sol, dt = _case(name)
    u_ref = sol.u
    u_new = sol.u.clone()
    torch.cuda.synchronize()
    t = 0.0
    for call in range(2):
        C.check(L.dgsem_ssprk3_step(solver.handle, ctypes.c_void_p(u_ref.data_ptr()), t, dt),
                "dgsem_ssprk3_step")
        C.check(L.dgsem_ssprk3_step_static_scratch(
            solver.handle, ctypes.c_void_p(u_new.data_ptr()), t, dt),
            "dgsem_ssprk3_step_static_scratch")
        torch.cuda.synchronize()
        a, b = u_new.cpu().numpy(), u_ref.cpu().numpy()
        assert np.isfinite(a).all(), call
        assert rel_linf(a, b) <= RTOL, (call, rel_linf(a, b))
        t += dt
    solver.check_finite()


def test_static_scratch_step_allocates_nothing(cuda):
    import torch

    from dgsem_b200 import _capi as C
    L = C.lib()
    solver, sol, dt = _case("kh")
    up = ctypes.c_void_p(sol.u.data_ptr())
    # the first call on the device is the set-up (scratch address look-up)
    C.check(L.dgsem_ssprk3_step_static_scratch(solver.handle, up, 0.0, dt), "first call")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for k in range(3):
        C.check(L.dgsem_ssprk3_step_static_scratch(solver.handle, up, (k + 1) * dt, dt),
                "later call")
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


class _DeviceView:
    """A float64 vector at a raw device address (CUDA array interface)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8",
                                         "data": (ptr, False), "version": 3}


def test_static_scratch_holds_the_stage_states(cuda):
    """The stage states went to the static scratch (not to the context's
    temporaries): after a step, its two slots hold u^(1) and u^(2) bit for bit
    as dgsem_ssprk3_stage computes them into caller buffers."""
    import torch

    from dgsem_b200 import _capi as C
    L = C.lib()
    solver, sol, dt = _case("tgv")
    u0 = sol.u.clone()
    n = u0.numel()
    s1 = torch.empty_like(u0)
    s2 = torch.empty_like(u0)
    C.check(L.dgsem_ssprk3_stage(solver.handle, 1, None, ctypes.c_void_p(u0.data_ptr()),
                                 ctypes.c_void_p(s1.data_ptr()), 0.0, dt), "stage 1")
    C.check(L.dgsem_ssprk3_stage(solver.handle, 2, ctypes.c_void_p(u0.data_ptr()),
                                 ctypes.c_void_p(s1.data_ptr()),
                                 ctypes.c_void_p(s2.data_ptr()), 0.0, dt), "stage 2")
    u = u0.clone()
    C.check(L.dgsem_ssprk3_step_static_scratch(solver.handle, ctypes.c_void_p(u.data_ptr()),
                                               0.0, dt), "static-scratch step")
    torch.cuda.synchronize()
    for k, want in ((0, s1), (1, s2)):
        ptr = ctypes.c_void_p()
        C.check(L.dgsem_static_scratch_state(k, ctypes.byref(ptr)), "scratch state")
        got = torch.as_tensor(_DeviceView(ptr.value, n), device=cuda)
        assert torch.equal(got, want.reshape(-1)), k
    bad = ctypes.c_void_p()
    assert L.dgsem_static_scratch_state(2, ctypes.byref(bad)) == C.DGSEM_ERR_INVALID_ARG


def test_static_scratch_rejects_large_state(cuda):
    import torch

    import dgsem_b200 as D
    from dgsem_b200 import _capi as C
    L = C.lib()
    # 2D, polydeg 3: 64 doubles per element; 192 x 192 elements exceed 2^21
    mesh = D.StructuredMesh((-1.0, -1.0), (1.0, 1.0), (192, 192))
    eq, basis = D.CompressibleEuler2D(1.4), D.LobattoLegendreBasis(3)
    solver = D.StructuredSolver(eq, basis, D.VolumeIntegralSplitForm(D.ChandrashekarFlux),
                                D.LaxFriedrichsFlux(), mesh,
                                D.BoundarySet(*[D.PeriodicBC() for _ in range(4)]))
    sol = D.Solution(mesh, basis, eq)
    solver.initialize(D.KelvinHelmholtzInitial(), sol)
    assert sol.u.numel() > C.STATIC_SCRATCH_MAX_STATE
    before = sol.u.clone()
    launches0 = solver.launch_count()
    st = L.dgsem_ssprk3_step_static_scratch(solver.handle, ctypes.c_void_p(sol.u.data_ptr()),
                                            0.0, 1e-3)
    assert st == C.DGSEM_ERR_SCRATCH_LIMIT
    assert L.dgsem_status_string(st) == b"state larger than the static scratch"
    assert solver.launch_count() == launches0
    torch.cuda.synchronize()
    assert torch.equal(sol.u, before)

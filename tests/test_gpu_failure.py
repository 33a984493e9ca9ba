"""Failure detection without a GPU fault.

The reference's only run-time check is the NaN break of its time loop
(time_integrator/integrator_base.hpp:32-34, observer/analysis_observer.hpp:
56-75).  On top of it this library has two failure paths that these tests
make run, on the host or with a bounded device wait, never by faulting the
GPU:

* a bounded mbarrier wait in the node-parallel stage kernels: with the
  test-only environment settings DGSEM_TEST_SKIP_TILE_COPY=1 and
  DGSEM_TEST_WAIT_LIMIT_NS the kernel arms its u_n barrier without issuing
  the bulk copy (nothing in flight), the wait runs out after 1 ms, the block
  votes, sets the timeout bit and returns; dgsem_check_finite reports
  DGSEM_ERR_TIMEOUT and the GPU keeps answering;
* device allocation failure at context creation: DGSEM_TEST_FAIL_ALLOC_AT=k
  fails the k-th allocation on the host side; the creation returns
  DGSEM_ERR_ALLOC and frees what it had allocated.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _kh_solver(cells=(8, 8)):
    import dgsem_b200 as D
    mesh = D.StructuredMesh((-1.0, -1.0), (1.0, 1.0), cells)
    eq, basis = D.CompressibleEuler2D(1.4), D.LobattoLegendreBasis(3)
    solver = D.StructuredSolver(eq, basis, D.VolumeIntegralSplitForm(D.ChandrashekarFlux),
                                D.LaxFriedrichsFlux(), mesh,
                                D.BoundarySet(*[D.PeriodicBC() for _ in range(4)]))
    sol = D.Solution(mesh, basis, eq)
    solver.initialize(D.KelvinHelmholtzInitial(), sol)
    return solver, sol


def test_bounded_tile_wait_reports_timeout(cuda, monkeypatch):
    import torch

    from dgsem_b200 import _capi as C
    L = C.lib()
    monkeypatch.setenv("DGSEM_TEST_SKIP_TILE_COPY", "1")
    monkeypatch.setenv("DGSEM_TEST_WAIT_LIMIT_NS", "1000000")  # 1 ms
    faulty, sol = _kh_solver()
    monkeypatch.delenv("DGSEM_TEST_SKIP_TILE_COPY")
    monkeypatch.delenv("DGSEM_TEST_WAIT_LIMIT_NS")
    # shape 3 (node-parallel) stages the u_n tile of stages 2 and 3 by bulk copy
    faulty.set_launch_variant(3)
    u = sol.u
    t1, t2 = torch.empty_like(u), torch.empty_like(u)
    ptr = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    C.check(L.dgsem_ssprk3_stage(faulty.handle, 1, None, ptr(u), ptr(t1), 0.0, 1e-4), "stage 1")
    assert L.dgsem_check_finite(faulty.handle) == C.DGSEM_OK  # stage 1 reads no u_n
    C.check(L.dgsem_ssprk3_stage(faulty.handle, 2, ptr(u), ptr(t1), ptr(t2), 0.0, 1e-4),
            "stage 2")
    assert L.dgsem_check_finite(faulty.handle) == C.DGSEM_ERR_TIMEOUT
    # the flag was cleared and the context still launches
    assert L.dgsem_check_finite(faulty.handle) == C.DGSEM_OK
    # the GPU still answers: a normal context steps and agrees with shape 0
    good, sol2 = _kh_solver()
    ref = sol2.u.clone()
    good.set_launch_variant(3)
    C.check(L.dgsem_ssprk3_step(good.handle, ptr(sol2.u), 0.0, 1e-4), "step")
    good.set_launch_variant(0)
    C.check(L.dgsem_ssprk3_step(good.handle, ptr(ref), 0.0, 1e-4), "step")
    torch.cuda.synchronize()
    assert L.dgsem_check_finite(good.handle) == C.DGSEM_OK
    a, b = sol2.u.cpu().numpy(), ref.cpu().numpy()
    assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))


@pytest.mark.parametrize("fail_at", [1, 2, 3, 5])
def test_allocation_failure_returns_alloc_and_frees(cuda, monkeypatch, fail_at):
    import torch

    import dgsem_b200 as D
    from dgsem_b200 import _capi as C
    L = C.lib()
    mesh = D.StructuredMesh((-1.0, -1.0), (1.0, 1.0), (64, 64))
    eq, basis = D.CompressibleEuler2D(1.4), D.LobattoLegendreBasis(3)
    # warm the allocator and the module so the free-memory figure is stable
    D.StructuredSolver(eq, basis, D.VolumeIntegralSplitForm(D.ChandrashekarFlux),
                       D.LaxFriedrichsFlux(), mesh,
                       D.BoundarySet(*[D.PeriodicBC() for _ in range(4)]))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    monkeypatch.setenv("DGSEM_TEST_FAIL_ALLOC_AT", str(fail_at))
    with pytest.raises(C.DgsemError) as err:
        D.StructuredSolver(eq, basis, D.VolumeIntegralSplitForm(D.ChandrashekarFlux),
                           D.LaxFriedrichsFlux(), mesh,
                           D.BoundarySet(*[D.PeriodicBC() for _ in range(4)]))
    assert err.value.status == C.DGSEM_ERR_ALLOC
    monkeypatch.delenv("DGSEM_TEST_FAIL_ALLOC_AT")
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 >= free0  # nothing of the failed creation stays allocated
    # and a normal creation afterwards works
    solver, sol = _kh_solver()
    C.check(L.dgsem_ssprk3_step(solver.handle, ctypes.c_void_p(sol.u.data_ptr()), 0.0, 1e-4),
            "step")
    assert L.dgsem_check_finite(solver.handle) == C.DGSEM_OK


def test_static_scratch_rejects_host_pointer(cuda):
    from dgsem_b200 import _capi as C
    L = C.lib()
    solver, sol = _kh_solver()
    host = np.zeros(sol.u.numel())
    st = L.dgsem_ssprk3_step_static_scratch(solver.handle, host.ctypes.data_as(ctypes.c_void_p),
                                            0.0, 1e-4)
    assert st == C.DGSEM_ERR_INVALID_ARG
    # no stale CUDA error is left for the next launch
    C.check(L.dgsem_ssprk3_step(solver.handle, ctypes.c_void_p(sol.u.data_ptr()), 0.0, 1e-4),
            "step after rejected call")
    assert L.dgsem_check_finite(solver.handle) == C.DGSEM_OK

"""Batched multi-mesh mode: every mesh of a batch (uneven sizes and degrees)
advances exactly like the single-mesh path, and one mesh matches the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import dgsem_oracle as do
from tests._util import RTOL, dev_to_ref, rel_linf

pytestmark = pytest.mark.gpu

SPECS = [  # (cells, polydeg, beta, center)
    ((5, 4), 1, 3.0, (0.5, -1.0)),
    ((7, 6), 2, 4.0, (-1.5, 0.3)),
    ((6, 9), 3, 5.0, (1.0, 1.0)),
    ((4, 4), 5, 2.5, (0.0, 0.0)),
    ((3, 5), 7, 6.0, (-0.4, 1.7)),
]


def _batch(cuda):
    import dgsem_b200 as D
    meshes = [(D.StructuredMesh((-5.0, -5.0), (5.0, 5.0), cells), N) for cells, N, _, _ in SPECS]
    batch = D.BatchSolver(D.CompressibleEuler2D(1.4), meshes, D.ChandrashekarFlux,
                          D.LaxFriedrichsFlux)
    batch.initialize(4, [(beta, c[0], c[1]) for _, _, beta, c in SPECS])
    return batch


def _single(cuda, k):
    import dgsem_b200 as D
    cells, N, beta, c = SPECS[k]
    mesh = D.StructuredMesh((-5.0, -5.0), (5.0, 5.0), cells)
    basis = D.LobattoLegendreBasis(N)
    solver = D.StructuredSolver(D.CompressibleEuler2D(1.4), basis,
                                D.VolumeIntegralSplitForm(D.ChandrashekarFlux),
                                D.LaxFriedrichsFlux(), mesh,
                                D.BoundarySet(*[D.PeriodicBC() for _ in range(4)]))
    sol = D.Solution(mesh, basis, D.CompressibleEuler2D(1.4))
    solver.initialize(D.IsentropicVortex(beta, c), sol)
    return solver, sol


def test_batched_step_equals_single_mesh_steps(cuda):
    import torch

    import dgsem_b200 as D
    batch = _batch(cuda)
    dts = [1e-3 * (1 + 0.1 * k) for k in range(len(SPECS))]
    for k in range(len(SPECS)):
        solver, sol = _single(cuda, k)
        assert torch.equal(batch.mesh_state(k), sol.u)
    batch.step(0.0, dts)
    batch.step(dts[0], dts)
    torch.cuda.synchronize()
    batch.check_finite()
    for k in range(len(SPECS)):
        solver, sol = _single(cuda, k)
        integ = D.SSPRK3(sol, solver.mesh, 0.0)
        integ.solve_steps(solver, sol, dts[k], 2)
        torch.cuda.synchronize()
        assert torch.equal(batch.mesh_state(k), sol.u), k


def test_batched_graph_equals_stream_steps(cuda):
    import torch
    a = _batch(cuda)
    b = _batch(cuda)
    dts = [2e-3] * len(SPECS)
    for s in range(3):
        a.step(s * dts[0], dts)
    g = b.graph(dts, 3)
    g.launch()
    torch.cuda.synchronize()
    assert torch.equal(a.u, b.u)


def test_batched_mesh_matches_oracle(cuda):
    import torch
    batch = _batch(cuda)
    k = 2
    cells, N, beta, c = SPECS[k]
    s = do.Scheme(ndims=2, polydeg=N, cells=cells, left=(-5.0, -5.0), right=(5.0, 5.0))
    u0 = do.initial_state(s, "vortex", beta=beta, center=c)
    dt = 1e-3
    batch.step(0.0, [dt] * len(SPECS))
    torch.cuda.synchronize()
    u1 = dev_to_ref(batch.mesh_state(k).cpu().numpy(), cells)
    u1_o = do.ssprk3_step(s, u0, 0.0, dt)
    assert rel_linf(u1, u1_o) <= RTOL
    assert np.isfinite(u1).all()


def test_batched_autotune_keeps_results(cuda):
    import torch
    a = _batch(cuda)
    b = _batch(cuda)
    dts = [1.5e-3] * len(SPECS)
    u_before = b.u.clone()
    chosen = b.autotune(dts)
    torch.cuda.synchronize()
    assert len(chosen) == len({N for _, N, _, _ in SPECS})
    assert all(v in (0, 1, 2, 3, 4, 5, 6) for v in chosen)
    assert torch.equal(b.u, u_before)
    for s in range(2):
        a.step(s * dts[0], dts)
        b.step(s * dts[0], dts)
    torch.cuda.synchronize()
    # shapes 0-2 are bitwise identical; the node-parallel shapes 3-4 differ in
    # summation order only
    ua, ub = a.u.cpu().numpy(), b.u.cpu().numpy()
    assert np.max(np.abs(ua - ub)) <= 1e-13 * np.max(np.abs(ua))


def test_persistent_launch_equals_per_degree_launches(cuda):
    """One persistent launch per stage over all degrees (work list, 128-thread
    blocks) against the per-degree node-parallel launches: same results to
    rounding, every mesh; stream steps and graph replay agree bit for bit."""
    import torch
    a = _batch(cuda)
    b = _batch(cuda)
    c = _batch(cuda)
    dts = [1.2e-3 * (1 + 0.05 * k) for k in range(len(SPECS))]
    b.set_persistent(True)
    c.set_persistent(True)
    for s in range(3):
        a.step(s * dts[0], dts)
        b.step(s * dts[0], dts)
    g = c.graph(dts, 3)
    g.launch()
    torch.cuda.synchronize()
    b.check_finite()
    ua, ub = a.u.cpu().numpy(), b.u.cpu().numpy()
    assert np.isfinite(ub).all()
    assert np.max(np.abs(ua - ub)) <= 1e-13 * np.max(np.abs(ua))
    assert torch.equal(b.u, c.u)
    # one launch per stage
    n0 = b.launch_count()
    b.step(0.0, dts)
    assert b.launch_count() - n0 == 3


def test_batched_fixed_launch_variant(cuda):
    """dgsem_batch_set_launch_variant: every launch shape of the batched
    engines advances the batch like shape 0 (to rounding); a shape that a
    degree group lacks is refused."""
    import torch

    from dgsem_b200 import _capi as C
    dts = [1.4e-3] * len(SPECS)
    ref = _batch(cuda)
    ref.step(0.0, dts)
    torch.cuda.synchronize()
    ur = ref.u.cpu().numpy()
    for v in (1, 2, 3, 4, 5):
        b = _batch(cuda)
        b.set_launch_variant(v)
        b.step(0.0, dts)
        torch.cuda.synchronize()
        b.check_finite()
        assert np.max(np.abs(b.u.cpu().numpy() - ur)) <= 1e-13 * np.max(np.abs(ur)), v
    b = _batch(cuda)
    with pytest.raises(C.DgsemError):
        b.set_launch_variant(6)  # 2D engines have no shape 6

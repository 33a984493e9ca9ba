"""Discrete adjoint (dgsem_adjoint_*) against the tangent-linear reference.

The tangent-linear reference is the reference solver compiled with a
dual-number scalar (oracle/_ref/libdgsem_ref_tlm.so): exact directional
derivatives of the reference's own RHS and SSPRK3.  Checks:
  * RHS: the adjoint identity <w, dR/du d> = <VJP(w), d> per pair of
    variables (so errors cannot cancel across variables), to 1e-10 of the
    summed magnitudes;
  * objective J (mean kinetic energy) and dJ/du against the oracle;
  * the adjoint workload (tests/_util.py ADJOINT_*): dJ/du0 . d_k against the
    committed tangent-linear fixture (tests/golden/adjoint_tlm.npz) to 1e-8
    relative, and against central finite differences (eps 1e-4 .. 1e-7) to
    1e-6 relative, in 8 seeded momentum directions;
  * checkpoint-interval invariance and determinism of the gradient.
"""
from __future__ import annotations

import math
import os

import numpy as np
import pytest

from oracle import dgsem_oracle as do
from oracle import ref_tlm_binding as tb
from tests import _util as U
from tests._util import ref_to_dev
from tests.test_gpu_parity import initial, make_device, make_oracle

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
NS_RECT = dict(ndims=2, polydeg=3, cells=(5, 4), left=(0.0, 0.0), right=(2 * math.pi, 4.0),
               ic="tgv2d", viscous=True, mu=2.0e-2, prandtl=0.72, noise=1.0e-2)
EULER = dict(ndims=2, polydeg=3, cells=(6, 5), left=(-1.0, -1.0), right=(1.0, 1.0), ic="kh",
             noise=0.02)
ADJ = dict(U.ADJOINT_CASE, ic="tgv2d")
needs_tlm = pytest.mark.skipif(not tb.available(),
                               reason="tangent-linear reference (oracle/_ref) not built")


def _tangent_case(case):
    kind = tb.NS2D if case.get("viscous") else tb.EULER2D
    return tb.TangentCase(kind, case["polydeg"], case["cells"], case["left"], case["right"],
                          1.4, case.get("mu", 0.0), case.get("prandtl", 0.72))


def _adjoint(case, nsteps=1, every=1):
    import dgsem_b200 as D
    solver = make_device(case)
    return solver, D.Adjoint(solver, nsteps, every)


@needs_tlm
@pytest.mark.parametrize("name,case", [("ns_rect", NS_RECT), ("euler", EULER)])
def test_rhs_vjp_adjoint_identity_vs_tangent_linear_reference(name, case, cuda):
    import torch
    s = make_oracle(case)
    u_ref = initial(case, s)
    tc = _tangent_case(case)
    solver, adj = _adjoint(case)
    u_dev = torch.from_numpy(ref_to_dev(u_ref, 2)).to(cuda)
    rng = np.random.default_rng(7)
    scale = np.max(np.abs(u_ref), axis=(0, 1, 2))
    for qd in range(4):
        d_ref = np.zeros_like(u_ref)
        d_ref[..., qd] = rng.standard_normal(u_ref.shape[:-1]) * scale[qd]
        _, jvp = tc.rhs(u_ref, d_ref)
        d_dev = ref_to_dev(d_ref, 2)
        for qw in range(4):
            w_ref = np.zeros_like(u_ref)
            w_ref[..., qw] = rng.standard_normal(u_ref.shape[:-1])
            w_dev = torch.from_numpy(ref_to_dev(w_ref, 2)).to(cuda)
            vjp = adj.rhs_vjp(u_dev, w_dev).cpu().numpy()
            lhs = float(np.sum(w_ref * jvp))
            rhs = float(np.sum(vjp * d_dev))
            mag = float(np.sum(np.abs(w_ref * jvp))) + 1e-300
            assert abs(lhs - rhs) <= 1e-10 * mag, (name, qd, qw, lhs, rhs, mag)


@needs_tlm
def test_rhs_vjp_adjoint_identity_adjoint_mesh(cuda):
    """The same identity on the adjoint workload's mesh, dense directions."""
    import torch
    s, u_ref = U.adjoint_initial_state()
    tc = _tangent_case(ADJ)
    solver, adj = _adjoint(ADJ)
    u = torch.from_numpy(ref_to_dev(u_ref, 2)).to(cuda)
    rng = np.random.default_rng(11)
    scale = np.array([1.0, 1.0, 1.0, 100.0])
    for k in range(3):
        d_ref = rng.standard_normal(u_ref.shape) * scale
        w_ref = rng.standard_normal(u_ref.shape)
        _, jvp = tc.rhs(u_ref, d_ref)
        vjp = adj.rhs_vjp(u, torch.from_numpy(ref_to_dev(w_ref, 2)).to(cuda)).cpu().numpy()
        lhs = float(np.sum(w_ref * jvp))
        rhs = float(np.sum(vjp * ref_to_dev(d_ref, 2)))
        mag = float(np.sum(np.abs(w_ref * jvp)))
        assert abs(lhs - rhs) <= 1e-10 * mag, (k, lhs, rhs, mag)


def test_kinetic_energy_matches_oracle(cuda):
    import torch
    s = make_oracle(NS_RECT)
    u_ref = initial(NS_RECT, s)
    solver, adj = _adjoint(NS_RECT)
    u = torch.from_numpy(ref_to_dev(u_ref, 2)).to(cuda)
    val, g = adj.kinetic_energy(u, grad=True)
    ref = do.kinetic_energy_mean(s, u_ref)
    assert abs(val - ref) <= 1e-13 * abs(ref)
    rng = np.random.default_rng(3)
    d_ref = rng.standard_normal(u_ref.shape)
    h = 1e-6  # J is a smooth rational function of u: no kinks
    fd = (do.kinetic_energy_mean(s, u_ref + h * d_ref)
          - do.kinetic_energy_mean(s, u_ref - h * d_ref)) / (2 * h)
    ad = float(np.sum(g.cpu().numpy() * ref_to_dev(d_ref, 2)))
    assert abs(fd - ad) <= 1e-7 * abs(ad)


def _J(solver, adj, u0, dt, nsteps):
    import ctypes

    from dgsem_b200 import _capi as C
    u = u0.clone()
    C.check(C.lib().dgsem_ssprk3_steps(solver.handle, ctypes.c_void_p(u.data_ptr()), 0.0, dt,
                                       nsteps), "dgsem_ssprk3_steps")
    return adj.kinetic_energy(u)


def _adjoint_workload(cuda):
    import torch

    import dgsem_b200 as D
    s, u_ref = U.adjoint_initial_state()
    solver = make_device(ADJ)
    adj = D.Adjoint(solver, U.ADJOINT_STEPS, U.ADJOINT_EVERY)
    u0 = torch.from_numpy(ref_to_dev(u_ref, 2)).to(cuda)
    dirs = [torch.from_numpy(ref_to_dev(d, 2)).to(cuda) for d in U.adjoint_directions(u_ref)]
    return solver, adj, u0, dirs


def test_adjoint_gradient_vs_tangent_linear_fixture(cuda):
    import torch
    fx = np.load(os.path.join(HERE, "golden", "adjoint_tlm.npz"))
    assert int(fx["steps"]) == U.ADJOINT_STEPS and float(fx["dt"]) == U.ADJOINT_DT
    solver, adj, u0, dirs = _adjoint_workload(cuda)
    J, g = adj.gradient(u0, 0.0, U.ADJOINT_DT)
    assert abs(J - float(fx["J"])) <= 1e-12 * abs(float(fx["J"]))
    for k, d in enumerate(dirs):
        ad = float(torch.sum(g * d))
        ref = float(fx["dJ"][k])
        assert abs(ad - ref) <= 1e-8 * abs(ref), (k, ad, ref)


def test_adjoint_gradient_vs_central_differences(cuda):
    import torch
    solver, adj, u0, dirs = _adjoint_workload(cuda)
    J, g = adj.gradient(u0, 0.0, U.ADJOINT_DT)
    assert J == _J(solver, adj, u0, U.ADJOINT_DT, U.ADJOINT_STEPS)
    for k, d in enumerate(dirs):
        ad = float(torch.sum(g * d))
        errs = []
        for eps in (1e-4, 1e-5, 1e-6, 1e-7):
            fd = (_J(solver, adj, u0 + eps * d, U.ADJOINT_DT, U.ADJOINT_STEPS)
                  - _J(solver, adj, u0 - eps * d, U.ADJOINT_DT, U.ADJOINT_STEPS)) / (2.0 * eps)
            errs.append(abs(fd - ad) / abs(ad))
        assert min(errs) <= 1e-6, (k, errs)


def test_adjoint_gradient_checkpoint_invariant_and_deterministic(cuda):
    import torch

    import dgsem_b200 as D
    s = make_oracle(NS_RECT)
    u_ref = initial(NS_RECT, s)
    solver = make_device(NS_RECT)
    u0 = torch.from_numpy(ref_to_dev(u_ref, 2)).to(cuda)
    out = []
    for every in (30, 7, 4, 1):
        adj = D.Adjoint(solver, 30, every)
        out.append(adj.gradient(u0, 0.0, 2e-3))
    for J, g in out[1:]:
        assert J == out[0][0]
        assert torch.equal(g, out[0][1])
    adj = D.Adjoint(solver, 30, 7)
    J2, g2 = adj.gradient(u0, 0.0, 2e-3)
    assert torch.equal(g2, out[1][1])

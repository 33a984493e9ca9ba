"""The node-parallel launch shapes at every supported degree: their pair
sharing of the volume term takes three forms (warp shuffles where a line lies
in one warp, a shared exchange buffer for the other x/y lines, both nodes
evaluating the pair on z lines), chosen from n at compile time.  For each
degree and two-point flux the right-hand side of shapes 3, 4 (and 5 where it
exists) must agree with each other and with the line-parallel shape to
rounding, and with the oracle within the parity bar; each shape must be
deterministic.  (Shapes 3-5 run the same source, but shape 3 is compiled
under a register cap, which can change where the compiler fuses a multiply
and an add: at n = 7 with the Ranocha flux they differ by ~1e-14.)  The
meshes leave the last node-parallel block partly empty for most degrees.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import dgsem_oracle as do
from tests._util import RTOL, dev_to_ref, ref_to_dev, rel_linf
from tests.test_gpu_parity import make_device, make_oracle

pytestmark = pytest.mark.gpu

CASES = []
for polydeg in range(1, 8):
    for vf in ("chandrashekar", "ranocha", "kennedy_gruber"):
        CASES.append(dict(ndims=2, polydeg=polydeg, cells=(5, 3), left=(-5.0, -5.0),
                          right=(5.0, 5.0), ic="vortex", noise=0.02, vf=vf))
for polydeg in range(1, 5):
    for vf in ("chandrashekar", "ranocha", "kennedy_gruber"):
        CASES.append(dict(ndims=3, polydeg=polydeg, cells=(3, 2, 2), left=(0.0,) * 3,
                          right=(2 * math.pi,) * 3, ic="tgv3d", noise=0.02, vf=vf))


@pytest.mark.parametrize("case", CASES,
                         ids=[f"{c['ndims']}d_p{c['polydeg']}_{c['vf']}" for c in CASES])
def test_node_shapes_every_degree(case, cuda):
    import torch
    vf = case["vf"]
    kw = {k: v for k, v in case.items() if k != "vf"}
    s = make_oracle(kw, volume_flux=vf)
    u_ref = do.initial_state(s, case["ic"])
    rng = np.random.default_rng(case["polydeg"])
    u_ref = u_ref * (1.0 + case["noise"] * rng.standard_normal(u_ref.shape))
    solver = make_device(kw, volume_flux=vf)
    nd = case["ndims"]
    u = torch.from_numpy(ref_to_dev(u_ref, nd)).to(cuda)
    outs = {}
    for v in range(7):
        try:
            solver.set_launch_variant(v)
        except Exception:
            continue  # shape not available for this scheme
        du, du2 = torch.empty_like(u), torch.empty_like(u)
        solver.rhs(u, du, 0.0)
        solver.rhs(u, du2, 0.0)
        torch.cuda.synchronize()
        assert torch.equal(du, du2), v  # deterministic
        outs[v] = du
    assert 0 in outs and 3 in outs and 4 in outs, sorted(outs)
    node = outs[3].cpu().numpy()
    for v in (0, 1, 2, 4, 5, 6):
        if v in outs:
            assert rel_linf(node, outs[v].cpu().numpy()) <= RTOL, v
    ref = do.rhs(s, u_ref, 0.0)
    assert rel_linf(dev_to_ref(node, solver.mesh.n_cells), ref) <= RTOL

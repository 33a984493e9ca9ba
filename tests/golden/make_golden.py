"""Generates the golden fixtures in this directory from the compiled reference.

The fixtures are outputs of the UNMODIFIED reference solver (RetrO598/DGSEM
headers compiled against the project's Kokkos shim, oracle/_ref) on seeded
inputs of the benchmark cases at small sizes:
  basis_N{1..7}.npz     LobattoLegendreBasis tables
  <case>.npz            u, du = calc_rhs(u, t), alpha (HG cases), u1 = one
                        SSPRK3 step, and the per-node metrics.
Regenerate with:  make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import dgsem_oracle as do  # noqa: E402
from oracle import ref_binding as rb  # noqa: E402

T_RHS = 0.013
DT = 2.0e-4

CASES = {
    "kh": (rb.EULER2D_PERIODIC_SPLIT, dict(ndims=2, polydeg=3, cells=(8, 8), left=(-1.0, -1.0),
                                           right=(1.0, 1.0)), "kh", 0.0),
    "kh_hg": (rb.EULER2D_PERIODIC_HG, dict(ndims=2, polydeg=3, cells=(8, 8), left=(-1.0, -1.0),
                                           right=(1.0, 1.0), shock_capturing=True), "kh", 0.05),
    "dmr": (rb.EULER2D_DMR_HG, dict(ndims=2, polydeg=3, cells=(24, 6), left=(0.0, 0.0),
                                    right=(4.0, 1.0), periodic=False, shock_capturing=True,
                                    bc="dmr"), "dmr", 0.0),
    "tgv": (rb.EULER3D_PERIODIC_SPLIT, dict(ndims=3, polydeg=3, cells=(4, 4, 4),
                                            left=(0.0, 0.0, 0.0), right=(2 * math.pi,) * 3),
            "tgv3d", 0.0),
    "ns": (rb.NS2D_PERIODIC_SPLIT, dict(ndims=2, polydeg=4, cells=(6, 6), left=(0.0, 0.0),
                                        right=(2 * math.pi,) * 2, viscous=True, mu=1.0e-3,
                                        prandtl=0.72), "tgv2d", 0.0),
}


def main():
    for N in range(1, 8):
        t = rb.basis_tables(N)
        np.savez_compressed(os.path.join(HERE, f"basis_N{N}.npz"), **t)
    for name, (kind, kw, ic, noise) in CASES.items():
        s = do.Scheme(**kw)
        u = do.initial_state(s, ic)
        rng = np.random.default_rng(1234)
        if noise:
            u = u * (1.0 + noise * rng.standard_normal(u.shape))
        if name == "ns":
            u[..., 1:3] += 1.0e-3 * rng.standard_normal(u[..., 1:3].shape)
        rc = rb.RefCase(kind, kw["polydeg"], kw["cells"], kw["left"], kw["right"],
                        mu=kw.get("mu", 0.0), prandtl=kw.get("prandtl", 0.72))
        du = rc.rhs(u, T_RHS)
        u1 = rc.ssprk3(u, 0.0, DT, 1)
        _, ja, inv_j = rc.geometry()
        out = dict(u=u, du=du, u1=u1, ja=ja, inv_j=inv_j, t=T_RHS, dt=DT)
        if kw.get("shock_capturing"):
            out["alpha"] = rc.alpha(u)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, {k: np.shape(v) for k, v in out.items()})


if __name__ == "__main__":
    main()

"""Shared helpers for the tests: layout conversion and case builders.

Reference logical layout: u_ref[ie, je(, ke), dof, var] (LayoutRight).
Device layout:            u_dev[e, var, dof], e = ie + nx*(je + ny*ke).
"""
from __future__ import annotations

import math

import numpy as np

# Parity bar of the RHS against the reference: relative L-infinity.
RTOL = 1.0e-12


def ref_to_dev(u_ref: np.ndarray, ndims: int) -> np.ndarray:
    if ndims == 2:
        nx, ny, nd, nv = u_ref.shape
        return np.ascontiguousarray(np.transpose(u_ref, (1, 0, 3, 2))).reshape(nx * ny, nv, nd)
    nx, ny, nz, nd, nv = u_ref.shape
    return np.ascontiguousarray(np.transpose(u_ref, (2, 1, 0, 4, 3))).reshape(nx * ny * nz, nv, nd)


def dev_to_ref(u_dev: np.ndarray, cells: tuple) -> np.ndarray:
    E, nv, nd = u_dev.shape
    if len(cells) == 2:
        nx, ny = cells
        return np.ascontiguousarray(np.transpose(u_dev.reshape(ny, nx, nv, nd), (1, 0, 3, 2)))
    nx, ny, nz = cells
    return np.ascontiguousarray(np.transpose(u_dev.reshape(nz, ny, nx, nv, nd), (2, 1, 0, 4, 3)))


def alpha_ref_to_dev(a_ref: np.ndarray) -> np.ndarray:
    """alpha[ie, je(, ke)] -> alpha[e]."""
    return np.ascontiguousarray(a_ref.T).reshape(-1)


def rel_linf(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


# Benchmark-shaped cases at small sizes (the oracle finishes in well under a second).
CASES = {
    "kh": dict(ndims=2, polydeg=3, cells=(8, 8), left=(-1.0, -1.0), right=(1.0, 1.0),
               ic="kh"),
    "kh_hg": dict(ndims=2, polydeg=3, cells=(8, 8), left=(-1.0, -1.0), right=(1.0, 1.0),
                  ic="kh", shock_capturing=True, noise=0.05),
    "dmr": dict(ndims=2, polydeg=3, cells=(24, 6), left=(0.0, 0.0), right=(4.0, 1.0),
                ic="dmr", shock_capturing=True, periodic=False, bc="dmr"),
    "tgv": dict(ndims=3, polydeg=3, cells=(4, 4, 4), left=(0.0, 0.0, 0.0),
                right=(2 * math.pi,) * 3, ic="tgv3d"),
    "vortex_n6": dict(ndims=2, polydeg=5, cells=(5, 7), left=(-5.0, -5.0), right=(5.0, 5.0),
                      ic="vortex"),
    "ns": dict(ndims=2, polydeg=4, cells=(6, 6), left=(0.0, 0.0), right=(2 * math.pi,) * 2,
               ic="tgv2d", viscous=True, mu=1.0e-3, prandtl=0.72, noise=1.0e-3),
    # element counts that leave the last block of the node-parallel shapes
    # partly empty (8 and 2 elements per block): idle lanes in whole warps
    "kh_hg_partial": dict(ndims=2, polydeg=3, cells=(5, 3), left=(-1.0, -1.0),
                          right=(1.0, 1.0), ic="kh", shock_capturing=True, noise=0.05),
    "tgv_partial": dict(ndims=3, polydeg=3, cells=(3, 3, 3), left=(0.0, 0.0, 0.0),
                        right=(2 * math.pi,) * 3, ic="tgv3d"),
}


# The adjoint workload: 2D Navier-Stokes Taylor-Green vortex on [0, 2 pi]^2,
# 32 x 32 elements, N = 4, Re = 1000 (mu = 1e-3), Pr = 0.72, plus 1e-3
# seeded Gaussian noise on the momentum; 200 SSPRK3 steps of dt = 1e-3
# (CFL ~0.5 for lambda_max ~11 with the reference's dt rule), checkpoints
# every 20 steps; objective = mean kinetic energy of the final state.
ADJOINT_CASE = dict(ndims=2, polydeg=4, cells=(32, 32), left=(0.0, 0.0),
                    right=(2 * math.pi, 2 * math.pi), viscous=True, mu=1.0e-3, prandtl=0.72)
ADJOINT_NOISE, ADJOINT_SEED = 1.0e-3, 0
ADJOINT_STEPS, ADJOINT_DT, ADJOINT_EVERY = 200, 1.0e-3, 20
ADJOINT_DIRECTION_SEED, ADJOINT_DIRECTIONS = 2024, 8


def adjoint_initial_state():
    """(oracle scheme, u0 in the reference layout u(i, j, dof, var))."""
    from oracle import dgsem_oracle as do
    s = do.Scheme(**ADJOINT_CASE)
    u = do.initial_state(s, "tgv2d")
    rng = np.random.default_rng(ADJOINT_SEED)
    u[..., 1:3] += ADJOINT_NOISE * rng.standard_normal(u[..., 1:3].shape)
    return s, np.ascontiguousarray(u)


def adjoint_directions(u0: np.ndarray):
    """Seeded Gaussian directions in the initial momentum (reference layout)."""
    rng = np.random.default_rng(ADJOINT_DIRECTION_SEED)
    out = []
    for _ in range(ADJOINT_DIRECTIONS):
        d = np.zeros_like(u0)
        d[..., 1:3] = rng.standard_normal(u0[..., 1:3].shape)
        out.append(d)
    return out

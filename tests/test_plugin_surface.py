"""The open plugin surface (include/dgsem_b200_kernels.cuh): a user
translation unit (tests/cpp/plugin_central.cu) brings its own two-point
volume flux (the reference's CentralFlux contract, base/numerical_flux.hpp:
230-258) and its own time-dependent Dirichlet function f(x, t)
(DirichletBC<Func>, boundary_condition/dirichlet_boundary.hpp:70-120) into
the library's fused stage kernel.  The reference runs the same case with its
own CentralFlux and DirichletBC (oracle/ref_harness.cpp,
EULER2D_CENTRAL_DIRICHLET).

CPU: the user unit compiles and links against the library.  GPU: its RHS and
its SSPRK3 steps match the reference's within max(1e-12, the reference's
self-variation) relative L-infinity.
"""
from __future__ import annotations

import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from tests._util import RTOL, dev_to_ref, ref_to_dev, rel_linf

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "plugin_central.cu")
LIBDIR = os.path.join(ROOT, "dgsem_b200", "_lib")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
CELLS, LEFT, RIGHT = (10, 8), (0.0, 0.0), (1.0, 1.0)


def _build(out_dir: str) -> str:
    so = os.path.join(out_dir, "plugin_central.so")
    cmd = [NVCC, "-std=c++17", "--expt-relaxed-constexpr", "-O3",
           "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC", "-shared",
           "-I", os.path.join(ROOT, "include"), SRC, "-L", LIBDIR, "-ldgsem_b200",
           "-Xlinker", "-rpath", "-Xlinker", LIBDIR, "-o", so]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return so


needs_toolchain = pytest.mark.skipif(
    not (os.path.exists(NVCC) and os.path.exists(os.path.join(LIBDIR, "libdgsem_b200.so"))),
    reason="nvcc or the library missing")


@needs_toolchain
def test_user_plugin_unit_compiles(tmp_path):
    so = _build(str(tmp_path))
    assert os.path.getsize(so) > 0


def _load(tmp_path):
    so = _build(str(tmp_path))
    L = ctypes.CDLL(so)
    L.plugin_create.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 4
    L.plugin_state_len.restype = ctypes.c_int64
    L.plugin_rhs.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double]
    L.plugin_steps.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int]
    assert L.plugin_create(CELLS[0], CELLS[1], LEFT[0], LEFT[1], RIGHT[0], RIGHT[1]) == 0
    return L


def _initial():
    """The user's Dirichlet state at t = 0 on the nodes, perturbed."""
    from oracle import dgsem_oracle as do
    s = do.Scheme(ndims=2, polydeg=3, cells=CELLS, left=LEFT, right=RIGHT, periodic=False)
    x, y = s.geo.coords[..., 0], s.geo.coords[..., 1]
    rho = 1.0 + 0.2 * np.sin(np.pi * (x + y))
    p = 1.0 + 0.1 * np.cos(np.pi * (x - y))
    u = np.stack([rho, 0.3 * rho, -0.2 * rho, p / 0.4 + 0.5 * rho * (0.09 + 0.04)], axis=-1)
    rng = np.random.default_rng(11)
    return np.ascontiguousarray(u * (1.0 + 0.02 * rng.standard_normal(u.shape)))


@needs_toolchain
@pytest.mark.gpu
def test_user_central_flux_and_dirichlet_match_reference(tmp_path, cuda):
    import torch

    from oracle import ref_binding as rb
    if not rb.available() or not rb.available("fma"):
        pytest.skip("compiled reference not built")
    L = _load(tmp_path)
    u0 = _initial()
    assert L.plugin_state_len() == u0.size
    rc = rb.RefCase(rb.EULER2D_CENTRAL_DIRICHLET, 3, CELLS, LEFT, RIGHT)
    rcf = rb.RefCase(rb.EULER2D_CENTRAL_DIRICHLET, 3, CELLS, LEFT, RIGHT, build="fma")
    ud = torch.from_numpy(ref_to_dev(u0, 2)).to(cuda)
    du = torch.empty_like(ud)
    for t in (0.0, 0.37):
        assert L.plugin_rhs(ud.data_ptr(), du.data_ptr(), t) == 0
        du_p = dev_to_ref(du.cpu().numpy(), CELLS)
        du_r = rc.rhs(u0, t)
        bar = max(RTOL, rel_linf(rcf.rhs(u0, t), du_r))
        err = rel_linf(du_p, du_r)
        print(f"\n  t = {t}: plugin vs reference {err:.3e} (bar {bar:.3e})")
        assert err <= bar
    # 20 SSPRK3 steps through the user plugins against the reference's SSPRK3
    dt = 2e-3
    assert L.plugin_steps(ud.data_ptr(), 0.0, dt, 20) == 0
    u_p = dev_to_ref(ud.cpu().numpy(), CELLS)
    u_r = rc.ssprk3(u0, 0.0, dt, 20)
    err = rel_linf(u_p - u0, u_r - u0)
    print(f"  20 steps: increment error {err:.3e}, state error {rel_linf(u_p, u_r):.3e}")
    assert rel_linf(u_p, u_r) <= RTOL
    assert err <= 1e-9

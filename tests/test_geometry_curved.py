"""Curvilinear meshes: the device geometry initializer
(dgsem_geometry_from_coordinates) and the fused stage kernel of the plugin
path on a non-linear mapping, against the reference's own
StructuredElementInitializer with the same mapping and its StructuredSolver
on that container (oracle/ref_harness.cpp: CurvedMapping, MappedRefCase).

* the initializer fed the reference's node coordinates reproduces its
  contravariant vectors and inverse Jacobian bit for bit (2D n = 4 and 3D
  n = 3, 4);
* a user translation unit (tests/cpp/plugin_curved.cu) maps the nodes on the
  device with the same formula (coordinates within a few ulps of the
  reference's: device sin), computes the metrics on the device and its RHS
  matches the reference's RHS on the curvilinear mesh within max(1e-12, the
  reference's self-variation).
"""
from __future__ import annotations

import ctypes
import math
import os
import shutil
import subprocess

import numpy as np
import pytest

from tests._util import RTOL, dev_to_ref, ref_to_dev, rel_linf

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "plugin_curved.cu")
LIBDIR = os.path.join(ROOT, "dgsem_b200", "_lib")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def _ref_geometry_to_dev(coords, ja, inv_j, nd):
    """Reference logical layout (cells..., dof, ...) -> device layout
    x[e][c][node], ja[e][a][c][node], inv_j[e][node], e = i + nx*(j + ny*k)."""
    if nd == 2:
        perm = (1, 0)
    else:
        perm = (2, 1, 0)
    c = np.transpose(coords, perm + (nd + 1, nd)).reshape(-1, nd, coords.shape[nd])
    j = np.transpose(ja, perm + (nd + 1, nd + 2, nd)).reshape(-1, nd, nd, ja.shape[nd])
    ij = np.transpose(inv_j, perm + (nd,)).reshape(-1, inv_j.shape[nd])
    return (np.ascontiguousarray(c), np.ascontiguousarray(j), np.ascontiguousarray(ij))


CASES = [
    (2, 3, (6, 5), (0.0, -1.0), (2.0, 1.0)),
    (3, 2, (3, 4, 2), (0.0, 0.0, 0.0), (2 * math.pi,) * 3),
    (3, 3, (4, 3, 3), (-1.0, 0.0, 0.0), (1.0, 2.0, 3.0)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("nd,N,cells,left,right", CASES)
def test_device_geometry_equals_reference_bitwise(nd, N, cells, left, right, cuda):
    import torch

    from dgsem_b200 import _capi as C
    from oracle import ref_binding as rb
    if not rb.available():
        pytest.skip("compiled reference not built")
    kind = rb.EULER2D_CURVED_CENTRAL if nd == 2 else rb.EULER3D_CURVED
    rc = rb.RefCase(kind, N, cells, left, right)
    coords, ja, inv_j = rc.geometry()
    x_d, ja_r, ij_r = _ref_geometry_to_dev(coords, ja, inv_j, nd)
    # the mapping is really curved: the metrics vary inside an element
    assert np.ptp(ij_r[0]) > 1e-3 * np.abs(ij_r[0]).max()
    x = torch.from_numpy(x_d).to(cuda)
    ja_g = torch.empty(ja_r.shape, dtype=torch.float64, device=cuda)
    ij_g = torch.empty(ij_r.shape, dtype=torch.float64, device=cuda)
    c64 = (ctypes.c_int64 * 3)(*(list(cells) + [1] * (3 - nd)))
    C.check(C.lib().dgsem_geometry_from_coordinates(
        nd, N, c64, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(ja_g.data_ptr()),
        ctypes.c_void_p(ij_g.data_ptr()), None), "geometry")
    torch.cuda.synchronize()
    assert np.array_equal(ja_g.cpu().numpy(), ja_r)
    assert np.array_equal(ij_g.cpu().numpy(), ij_r)


def _build(out_dir: str) -> str:
    so = os.path.join(out_dir, "plugin_curved.so")
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
def test_curved_plugin_unit_compiles(tmp_path):
    assert os.path.getsize(_build(str(tmp_path))) > 0


@needs_toolchain
@pytest.mark.gpu
def test_curved_mesh_rhs_matches_reference(tmp_path, cuda):
    import torch

    from oracle import ref_binding as rb
    if not rb.available() or not rb.available("fma"):
        pytest.skip("compiled reference not built")
    cells, left, right = (10, 8), (0.0, -1.0), (2.0, 1.0)
    L = ctypes.CDLL(_build(str(tmp_path)))
    L.curved_create.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 4
    L.curved_rhs.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double]
    L.curved_geometry.argtypes = [ctypes.c_void_p] * 3
    L.curved_create_from_coordinates.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    assert L.curved_create(cells[0], cells[1], left[0], left[1], right[0], right[1]) == 0
    rc = rb.RefCase(rb.EULER2D_CURVED_CENTRAL, 3, cells, left, right)
    rcf = rb.RefCase(rb.EULER2D_CURVED_CENTRAL, 3, cells, left, right, build="fma")
    coords, ja, inv_j = rc.geometry()
    x_r, ja_r, ij_r = _ref_geometry_to_dev(coords, ja, inv_j, 2)
    E = cells[0] * cells[1]
    xg = torch.empty((E, 2, 16), dtype=torch.float64, device=cuda)
    jg = torch.empty((E, 2, 2, 16), dtype=torch.float64, device=cuda)
    ig = torch.empty((E, 16), dtype=torch.float64, device=cuda)
    assert L.curved_geometry(xg.data_ptr(), jg.data_ptr(), ig.data_ptr()) == 0
    # device node coordinates from the user's mapping: a few ulps from the
    # reference's (device sin against the host's)
    assert np.max(np.abs(xg.cpu().numpy() - x_r)) <= 1e-15 * 4
    assert rel_linf(jg.cpu().numpy(), ja_r) <= 1e-13
    assert rel_linf(ig.cpu().numpy(), ij_r) <= 1e-13
    # a smooth state on the curvilinear mesh
    X, Y = coords[..., 0], coords[..., 1]
    rho = 1.0 + 0.2 * np.sin(np.pi * X) * np.cos(np.pi * Y)
    v1, v2 = 0.3 + 0.1 * np.cos(np.pi * Y), -0.2 + 0.1 * np.sin(np.pi * X)
    p = 1.0 + 0.1 * np.cos(np.pi * (X - Y))
    u = np.ascontiguousarray(np.stack([rho, rho * v1, rho * v2,
                                       p / 0.4 + 0.5 * rho * (v1 * v1 + v2 * v2)], axis=-1))
    du_r = rc.rhs(u, 0.0)
    bar = max(RTOL, rel_linf(rcf.rhs(u, 0.0), du_r))
    ud = torch.from_numpy(ref_to_dev(u, 2)).to(cuda)
    du = torch.empty_like(ud)
    assert L.curved_rhs(ud.data_ptr(), du.data_ptr(), 0.0) == 0
    err = rel_linf(dev_to_ref(du.cpu().numpy(), cells), du_r)
    print(f"\n  curvilinear RHS (device mapping): plugin vs reference {err:.3e} (bar {bar:.3e})")
    # the device mapping's coordinates differ from the reference's by ulps of
    # sin, which the metric derivatives and flux differences amplify; the
    # bar applies to the same coordinates below
    assert err <= 1e-10
    # the reference's own node coordinates: metrics identical bit for bit
    xd = torch.from_numpy(x_r).to(cuda)
    assert L.curved_create_from_coordinates(cells[0], cells[1], xd.data_ptr()) == 0
    assert L.curved_rhs(ud.data_ptr(), du.data_ptr(), 0.0) == 0
    err = rel_linf(dev_to_ref(du.cpu().numpy(), cells), du_r)
    print(f"  curvilinear RHS (reference coordinates): {err:.3e} (bar {bar:.3e})")
    assert err <= bar
    # free-stream preservation on the curvilinear mesh (discrete metric
    # identities of the reference's metric formulas)
    fs = np.zeros_like(u)
    fs[..., 0], fs[..., 1], fs[..., 2], fs[..., 3] = 1.0, 0.3, -0.2, 1.0 / 0.4 + 0.5 * 0.13
    fsd = torch.from_numpy(ref_to_dev(fs, 2)).to(cuda)
    assert L.curved_rhs(fsd.data_ptr(), du.data_ptr(), 0.0) == 0
    assert float(du.abs().max()) <= 1e-11

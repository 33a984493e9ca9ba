"""C-ABI checks that need no GPU: the library loads, exports every entry
point include/dgsem_b200.h declares, its host-side basis and metric tables
agree bitwise with the oracle (and thus the reference), and descriptor
validation rejects bad input before touching the device."""
from __future__ import annotations

import ctypes
import math
import os
import re

import numpy as np
import pytest

import dgsem_b200._capi as C
from oracle import dgsem_oracle as do

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            with open(os.path.join(ROOT, "include", f)) as fh:
                text = fh.read()
            names |= set(re.findall(r"^\s*(?:dgsem_status|const char\s*\*)\s*(dgsem_[a-z0-9_]+)\s*\(",
                                    text, flags=re.M))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = C.lib()
    decl = declared_functions()
    assert len(decl) >= 20
    for name in decl:
        assert hasattr(L, name), name
    assert sorted(C.EXPORTED) == decl


def _f64p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@pytest.mark.parametrize("N", range(1, 8))
def test_host_basis_tables_bitwise(N):
    n = N + 1
    out = np.zeros(5 * n + 4 * n * n)
    assert C.lib().dgsem_basis_tables_host(N, _f64p(out)) == 0
    b = do.Basis(N)
    o = 0
    for k in ("nodes", "weights", "inv_weights", "lhat_left", "lhat_right"):
        assert np.array_equal(out[o:o + n], getattr(b, k)), k
        o += n
    for k in ("D", "Dsplit", "Dhat", "Vinv"):
        assert np.array_equal(out[o:o + n * n].reshape(n, n), getattr(b, k)), k
        o += n * n


def _mesh(nd, N, cells, left, right):
    m = C.MeshDesc()
    m.ndims = nd
    m.polydeg = N
    for a in range(3):
        m.n_cells[a] = cells[a] if a < nd else 1
        m.domain_left[a] = left[a] if a < nd else 0.0
        m.domain_right[a] = right[a] if a < nd else 1.0
    return m


@pytest.mark.parametrize("nd,N,cells,left,right", [
    (2, 3, (8, 8), (-1.0, -1.0), (1.0, 1.0)),
    (2, 3, (24, 6), (0.0, 0.0), (4.0, 1.0)),
    (2, 6, (5, 7), (-5.0, -5.0), (5.0, 5.0)),
    (3, 3, (4, 5, 6), (0.0, 0.0, 0.0), (2 * math.pi,) * 3),
    (3, 2, (3, 4, 2), (-1.0, 0.5, 2.0), (1.0, 3.0, 7.0)),
])
def test_separable_metric_tables_reproduce_reference_bitwise(nd, N, cells, left, right):
    """The kernels' per-node metrics (tables factored over element axes)
    equal the reference's StructuredElementInitializer output bitwise."""
    m = _mesh(nd, N, cells, left, right)
    ndof = (N + 1) ** nd
    E = math.prod(cells)
    ja = np.zeros(E * ndof * nd * nd)
    ij = np.zeros(E * ndof)
    assert C.lib().dgsem_metrics_host(ctypes.byref(m), _f64p(ja), _f64p(ij)) == 0
    geo = (do.geometry_2d if nd == 2 else do.geometry_3d)(do.Basis(N), cells, left, right,
                                                          (True,) * nd)
    assert np.array_equal(ja.reshape(geo.ja.shape), geo.ja)
    assert np.array_equal(ij.reshape(geo.inv_j.shape), geo.inv_j)


def _scheme(**kw):
    s = C.SchemeDesc()
    s.equation = kw.get("equation", C.EULER_2D)
    s.volume_flux = kw.get("volume_flux", 0)
    s.surface_flux = kw.get("surface_flux", 0)
    s.volume_integral = kw.get("volume_integral", 0)
    for f, b in enumerate(kw.get("bc", [0] * 6)):
        s.bc[f] = b
    s.gamma = kw.get("gamma", 1.4)
    s.alpha_max, s.alpha_min = 0.5, 0.001
    return s


@pytest.mark.parametrize("mesh_kw,scheme_kw,expect", [
    (dict(nd=4), {}, 1),                                      # bad dimension
    (dict(N=0), {}, 2),                                       # degree out of range
    (dict(N=8), {}, 2),
    (dict(cells=(0, 4)), {}, 1),                              # empty mesh
    (dict(right=(-2.0, 1.0)), {}, 1),                         # inverted domain
    ({}, dict(equation=C.EULER_3D), 1),                       # equation/mesh mismatch
    ({}, dict(volume_flux=7), 1),
    ({}, dict(gamma=1.0), 1),
    ({}, dict(bc=[0, 2, 0, 0, 0, 0]), 1),                     # half-periodic direction
    (dict(nd=3, cells=(2, 2, 2)), dict(equation=C.EULER_3D, surface_flux=C.SF_HLLC), 2),
])
def test_descriptor_validation_without_gpu(mesh_kw, scheme_kw, expect):
    nd = mesh_kw.get("nd", 2)
    m = _mesh(min(nd, 3), mesh_kw.get("N", 3), mesh_kw.get("cells", (4, 4, 4)),
              (0.0, 0.0, 0.0), mesh_kw.get("right", (1.0, 1.0, 1.0)))
    m.ndims = nd
    s = _scheme(**scheme_kw)
    h = ctypes.c_void_p()
    rc = C.lib().dgsem_ctx_create(ctypes.byref(m), ctypes.byref(s), None, ctypes.byref(h))
    assert rc == expect
    assert not h.value


def test_null_arguments_rejected():
    L = C.lib()
    assert L.dgsem_rhs(None, None, None, 0.0) == 1
    assert L.dgsem_ssprk3_step(None, None, 0.0, 0.0) == 1
    assert L.dgsem_ctx_destroy(None) == 1
    assert L.dgsem_graph_launch(None, 0.0) == 1
    assert L.dgsem_status_string(4) == b"non-finite value in state"


def test_product_has_no_cpu_path(monkeypatch, tmp_path):
    """Without the built library the product raises; it never computes on the CPU.
    (monkeypatch restores the loaded library afterwards.)"""
    monkeypatch.setattr(C, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(C, "_lib", None)
    with pytest.raises(FileNotFoundError):
        C.lib()

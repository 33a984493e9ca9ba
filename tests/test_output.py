"""On-disk output: the VTK-free VTU writer (the reference's
VTUOutputObserver, observer/vtu_output_observer.hpp:65-235, with Lagrange
cells) and the binary checkpoint / restart.

CPU tests drive the host entry points (no GPU): the file is parsed back (XML
header + appended raw blocks with UInt64 sizes) and every array checked
against the mesh coordinates and the state; VTK's Lagrange point order is
checked against the fixed orders of VTK's quadratic cells (biquadratic quad,
order 2) and for being a permutation.  GPU tests check that the device entry
points write the same bytes and that a restart continues bit for bit.
"""
from __future__ import annotations

import ctypes
import re
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from dgsem_b200 import _capi as C


def _mesh(nd, N, cells, left, right):
    m = C.MeshDesc()
    m.ndims, m.polydeg = nd, N
    for a in range(3):
        m.n_cells[a] = cells[a] if a < nd else 1
        m.domain_left[a] = left[a] if a < nd else 0.0
        m.domain_right[a] = right[a] if a < nd else 1.0
    return m


def _coords_dev_order(m, nd, N, cells):
    """Node coordinates [e][node][dim] in the device element order."""
    n = N + 1
    nn = n ** nd
    ref = np.zeros(tuple(cells) + (nn, nd))
    C.check(C.lib().dgsem_coordinates_host(ctypes.byref(m),
                                           ref.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
            "coords")
    # reference logical order (i, j[, k]) -> device order e = i + nx*(j + ny*k)
    if nd == 2:
        return np.transpose(ref, (1, 0, 2, 3)).reshape(-1, nn, nd)
    return np.transpose(ref, (2, 1, 0, 3, 4)).reshape(-1, nn, nd)


def _read_vtu(path):
    raw = open(path, "rb").read()
    head, _, rest = raw.partition(b"<AppendedData encoding=\"raw\">")
    start = rest.index(b"_") + 1
    data = rest[start:]
    root = ET.fromstring(head.decode() + "</VTKFile>")
    piece = root.find("UnstructuredGrid/Piece")
    arrays = {}
    for da in root.iter("DataArray"):
        off = int(da.get("offset"))
        nbytes = int(np.frombuffer(data[off:off + 8], dtype="<u8")[0])
        dt = {"Float64": "<f8", "Int64": "<i8", "UInt8": "u1"}[da.get("type")]
        name = da.get("Name") or "Points"
        arrays[name] = np.frombuffer(data[off + 8:off + 8 + nbytes], dtype=dt)
    assert rest.rstrip().endswith(b"</VTKFile>")
    return root, piece, arrays


def vtk_quad_order2():
    # VTK biquadratic quadrilateral: corners, edge mid-points (0-1, 1-2, 2-3,
    # 3-0), centre; as (i, j) node indices of an order-2 element
    return [(0, 0), (2, 0), (2, 2), (0, 2), (1, 0), (2, 1), (1, 2), (0, 1), (1, 1)]


@pytest.mark.parametrize("nd,N,cells", [(2, 3, (3, 2)), (2, 2, (2, 2)), (3, 2, (2, 2, 1)),
                                        (3, 3, (1, 2, 2))])
def test_vtu_host_arrays(tmp_path, nd, N, cells):
    n = N + 1
    nn = n ** nd
    nv = nd + 2
    left, right = (-1.0, 0.5, 0.0), (2.0, 1.5, 3.0)
    m = _mesh(nd, N, cells, left, right)
    E = int(np.prod(cells))
    rng = np.random.default_rng(7)
    u = rng.random((E, nv, nn)) + 1.0
    u[:, nv - 1, :] += 5.0
    path = str(tmp_path / "out.vtu")
    C.check(C.lib().dgsem_write_vtu_host(ctypes.byref(m), 1.4,
                                         u.ctypes.data_as(ctypes.c_void_p), path.encode()), "vtu")
    root, piece, a = _read_vtu(path)
    assert root.get("type") == "UnstructuredGrid" and root.get("header_type") == "UInt64"
    assert int(piece.get("NumberOfPoints")) == E * nn and int(piece.get("NumberOfCells")) == E
    assert np.all(a["types"] == (70 if nd == 2 else 72))
    assert np.array_equal(a["offsets"], (np.arange(E) + 1) * nn)
    assert np.array_equal(a["connectivity"], np.arange(E * nn))
    names = (["rho", "rhou", "rhov", "rhoE", "pressure"] if nd == 2 else
             ["rho", "rhou", "rhov", "rhow", "rhoE", "pressure"])
    assert [da.get("Name") for da in piece.find("PointData")] == names
    pts = a["Points"].reshape(E, nn, 3)
    xyz = _coords_dev_order(m, nd, N, cells)
    # recover the permutation from the coordinates, then check the values
    perm = np.zeros((E, nn), dtype=int)
    for e in range(E):
        for node in range(nn):
            d = np.abs(pts[e, :, :nd] - xyz[e, node]).sum(axis=1)
            k = int(np.argmin(d))
            assert d[k] == 0.0
            perm[e, node] = k
        assert sorted(perm[e]) == list(range(nn))
    assert np.all(perm == perm[0])
    for q in range(nv):
        vals = a[names[q]].reshape(E, nn)
        assert np.array_equal(np.take_along_axis(vals, perm, axis=1), u[:, q, :])
    p = a["pressure"].reshape(E, nn)
    mom2 = sum(u[:, 1 + d, :] ** 2 for d in range(nd))
    p_ref = 0.4 * (u[:, nv - 1, :] - 0.5 * mom2 / u[:, 0, :])
    assert np.max(np.abs(np.take_along_axis(p, perm, axis=1) - p_ref)) <= 1e-14 * np.max(p_ref)
    # VTK Lagrange order: vertices first (counter-clockwise, bottom then top)
    idx = {}
    for node in range(nn):
        ijk = (node % n, (node // n) % n, node // (n * n))
        idx[ijk[:nd]] = perm[0, node]
    if nd == 2:
        assert [idx[c] for c in [(0, 0), (N, 0), (N, N), (0, N)]] == [0, 1, 2, 3]
        if N == 2:
            assert [idx[c] for c in vtk_quad_order2()] == list(range(9))
    else:
        corners = [(0, 0, 0), (N, 0, 0), (N, N, 0), (0, N, 0), (0, 0, N), (N, 0, N), (N, N, N),
                   (0, N, N)]
        assert [idx[c] for c in corners] == list(range(8))
        if N == 2:
            # edges along i, j at k = 0 then k = N, then the edges along k
            edges = [(1, 0, 0), (2, 1, 0), (1, 2, 0), (0, 1, 0), (1, 0, 2), (2, 1, 2), (1, 2, 2),
                     (0, 1, 2)]
            assert [idx[c] for c in edges] == list(range(8, 16))
            assert idx[(1, 1, 1)] == 26  # the body node is last


def test_checkpoint_host_round_trip(tmp_path):
    m = _mesh(2, 3, (4, 3), (0.0, 0.0), (1.0, 1.0))
    s = C.SchemeDesc()
    s.gamma = 1.4
    u = np.random.default_rng(3).random(4 * 3 * 4 * 16)
    path = str(tmp_path / "ck.bin")
    L = C.lib()
    C.check(L.dgsem_checkpoint_write_host(ctypes.byref(m), ctypes.byref(s),
                                          u.ctypes.data_as(ctypes.c_void_p), 1.25, 42,
                                          path.encode()), "write")
    v = np.zeros_like(u)
    t, k = ctypes.c_double(), ctypes.c_int64()
    C.check(L.dgsem_checkpoint_read_host(ctypes.byref(m), v.ctypes.data_as(ctypes.c_void_p),
                                         ctypes.byref(t), ctypes.byref(k), path.encode()), "read")
    assert np.array_equal(u, v) and t.value == 1.25 and k.value == 42
    # another mesh is refused
    m2 = _mesh(2, 3, (4, 4), (0.0, 0.0), (1.0, 1.0))
    w = np.zeros(4 * 4 * 4 * 16)
    assert L.dgsem_checkpoint_read_host(ctypes.byref(m2), w.ctypes.data_as(ctypes.c_void_p),
                                        None, None, path.encode()) == C.DGSEM_ERR_INVALID_ARG
    # a damaged file is refused
    raw = bytearray(open(path, "rb").read())
    raw[0] ^= 0xFF
    open(path, "wb").write(bytes(raw))
    assert L.dgsem_checkpoint_read_host(ctypes.byref(m), v.ctypes.data_as(ctypes.c_void_p),
                                        None, None, path.encode()) == C.DGSEM_ERR_INVALID_ARG


@pytest.mark.gpu
def test_vtu_observer_and_restart_on_gpu(tmp_path, cuda):
    import torch

    import dgsem_b200 as D
    mesh = D.StructuredMesh((-1.0, -1.0), (1.0, 1.0), (8, 8))
    eq, basis = D.CompressibleEuler2D(1.4), D.LobattoLegendreBasis(3)
    solver = D.StructuredSolver(eq, basis, D.VolumeIntegralSplitForm(D.ChandrashekarFlux),
                                D.LaxFriedrichsFlux(), mesh,
                                D.BoundarySet(*[D.PeriodicBC() for _ in range(4)]))
    sol = D.Solution(mesh, basis, eq)
    solver.initialize(D.KelvinHelmholtzInitial(), sol)
    dt = 1e-3
    integ = D.SSPRK3(sol, mesh, 10 * dt - 1e-12)
    obs = D.VTUOutputObserver(str(tmp_path / "kh"), solver, sol, output_interval=4)
    integ.add_observer(obs)
    integ.solve(solver, sol, dt)
    assert [re.sub(r".*_step", "", f) for f in obs.written] == ["0.vtu", "4.vtu", "8.vtu",
                                                                 "10.vtu"]
    # the device writer equals the host writer on the same state
    host = sol.u.cpu().numpy().copy()
    hpath = str(tmp_path / "host.vtu")
    C.check(C.lib().dgsem_write_vtu_host(ctypes.byref(solver._mesh_desc), 1.4,
                                         host.ctypes.data_as(ctypes.c_void_p), hpath.encode()),
            "vtu host")
    assert open(hpath, "rb").read() == open(obs.written[-1], "rb").read()
    # restart: checkpoint after 10 steps, 5 more steps, against a continuous run
    ck = str(tmp_path / "kh.ckpt")
    D.write_checkpoint(ck, solver, sol, integ.time, integ.iter)
    cont = sol.u.clone()
    C.check(C.lib().dgsem_ssprk3_steps(solver.handle, ctypes.c_void_p(cont.data_ptr()),
                                       integ.time, dt, 5), "steps")
    sol.u.zero_()
    t, k = D.read_checkpoint(ck, solver, sol)
    assert k == 10 and t == integ.time
    C.check(C.lib().dgsem_ssprk3_steps(solver.handle, ctypes.c_void_p(sol.u.data_ptr()), t, dt,
                                       5), "steps")
    torch.cuda.synchronize()
    assert torch.equal(sol.u, cont)

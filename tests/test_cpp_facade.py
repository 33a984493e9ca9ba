"""The header-only C++ facade (include/dgsem_b200.hpp): a reference-style
Kelvin-Helmholtz program (tests/cpp/kelvin_helmholtz.cpp, user initial
condition functor, StructuredSolver / Solution / SSPRK3 / observers) compiles
and links against the library (CPU), and on the GPU its trajectory equals the
Python/C-ABI path's bit for bit from the same initial state, with and without
shock capturing."""
from __future__ import annotations

import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "kelvin_helmholtz.cpp")
LIBDIR = os.path.join(ROOT, "dgsem_b200", "_lib")
CUDA = "/usr/local/cuda"


def _compile(out_dir: str) -> str:
    cxx = shutil.which("g++") or "/usr/bin/g++"
    exe = os.path.join(out_dir, "kelvin_helmholtz")
    cmd = [cxx, "-std=c++20", "-O2", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"), SRC,
           "-L", LIBDIR, "-ldgsem_b200", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


needs_toolchain = pytest.mark.skipif(
    not (os.path.exists(os.path.join(LIBDIR, "libdgsem_b200.so"))
         and os.path.exists(os.path.join(CUDA, "include", "cuda_runtime.h"))),
    reason="library or CUDA headers missing")


@needs_toolchain
def test_facade_example_compiles_and_links(tmp_path):
    exe = _compile(str(tmp_path))
    assert os.path.exists(exe)


@needs_toolchain
@pytest.mark.gpu
@pytest.mark.parametrize("hg", [0, 1])
def test_facade_trajectory_equals_c_abi_path(hg, tmp_path, cuda):
    import ctypes

    import torch

    import dgsem_b200 as D
    from dgsem_b200 import _capi as C
    exe = _compile(str(tmp_path))
    nx, ny, steps, dt = 12, 10, 25, 1.0e-3
    prefix = str(tmp_path / "kh")
    r = subprocess.run([exe, str(nx), str(ny), str(steps), repr(dt), str(hg), prefix],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "nan 0" in r.stdout
    n = 4
    shape = (nx, ny, n * n, 4)
    u0 = np.fromfile(prefix + "_u0.bin", dtype=np.float64).reshape(shape)
    uT = np.fromfile(prefix + "_uT.bin", dtype=np.float64).reshape(shape)
    mesh = D.StructuredMesh((-1.0, -1.0), (1.0, 1.0), (nx, ny))
    vflux = D.ChandrashekarFlux
    vi = D.VolumeIntegralShockCapturingHG(vflux) if hg else D.VolumeIntegralSplitForm(vflux)
    solver = D.StructuredSolver(D.CompressibleEuler2D(1.4), D.LobattoLegendreBasis(3), vi,
                                D.LaxFriedrichsFlux(), mesh,
                                D.BoundarySet(*[D.PeriodicBC() for _ in range(4)]))
    u = solver.from_reference_layout(torch.from_numpy(u0).to(cuda))
    # integrator_base.hpp:24-44 clock: while (t < final) { step(t); t += dt }
    t, final = 0.0, steps * dt
    while t < final:
        C.check(C.lib().dgsem_ssprk3_step(solver.handle, ctypes.c_void_p(u.data_ptr()), t, dt),
                "dgsem_ssprk3_step")
        t += dt
    torch.cuda.synchronize()
    got = solver.to_reference_layout(u).cpu().numpy().reshape(shape)
    assert np.array_equal(got, uT)
    # the host-evaluated initial state agrees with the library's own KH initial condition
    sol = D.Solution(mesh, D.LobattoLegendreBasis(3), D.CompressibleEuler2D(1.4))
    solver.initialize(D.KelvinHelmholtzInitial(), sol)
    ic = solver.to_reference_layout(sol.u).cpu().numpy().reshape(shape)
    assert np.max(np.abs(ic - u0)) <= 1e-14 * np.max(np.abs(u0))

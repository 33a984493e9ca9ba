"""Parity of the CUDA path (through the C ABI) with the oracle and the
compiled reference, on benchmark-shaped cases at small sizes.

Bar: relative L-infinity <= 1e-12 per RHS and per SSPRK3 step (FP64), and
identical Hennemann-Gassner troubled-cell flags.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import dgsem_oracle as do
from oracle import ref_binding as rb
from tests._util import CASES, RTOL, alpha_ref_to_dev, dev_to_ref, ref_to_dev, rel_linf

pytestmark = pytest.mark.gpu

VF = {"chandrashekar": "ChandrashekarFlux", "ranocha": "RanochaFlux",
      "kennedy_gruber": "KennedyGruberFlux"}
SF = {"llf": "LaxFriedrichsFlux", "hllc": "HLLCFlux"}
REF_KIND = {("kh", False): rb.EULER2D_PERIODIC_SPLIT, ("kh", True): rb.EULER2D_PERIODIC_HG,
            ("dmr", True): rb.EULER2D_DMR_HG, ("tgv3d", False): rb.EULER3D_PERIODIC_SPLIT,
            ("vortex", False): rb.EULER2D_PERIODIC_SPLIT}


def make_oracle(case: dict, volume_flux="chandrashekar", surface_flux="llf"):
    kw = {k: v for k, v in case.items() if k not in ("ic", "noise")}
    return do.Scheme(volume_flux=volume_flux, surface_flux=surface_flux, **kw)


def make_device(case: dict, volume_flux="chandrashekar", surface_flux="llf"):
    import dgsem_b200 as D
    nd = case["ndims"]
    mesh = D.StructuredMesh(case["left"], case["right"], case["cells"])
    eq = D.CompressibleEuler2D(1.4) if nd == 2 else D.CompressibleEuler3D(1.4)
    vflux = getattr(D, VF[volume_flux])
    if case.get("shock_capturing"):
        vi = D.VolumeIntegralShockCapturingHG(vflux)
    else:
        vi = D.VolumeIntegralSplitForm(vflux)
    if case.get("bc") == "dmr":
        bcs = D.BoundarySet(D.DirichletBC("double_mach"), D.OutflowBC(),
                            D.MixedDirichletSlipWallBC("double_mach"),
                            D.DirichletBC("double_mach"))
    else:
        bcs = D.BoundarySet(*[D.PeriodicBC() for _ in range(2 * nd)])
    solver = D.StructuredSolver(eq, D.LobattoLegendreBasis(case["polydeg"]), vi,
                                getattr(D, SF[surface_flux])(), mesh, bcs)
    return solver


def initial(case: dict, s: do.Scheme, seed: int = 0):
    u = do.initial_state(s, case["ic"])
    if case.get("noise"):
        rng = np.random.default_rng(seed)
        u = u * (1.0 + case["noise"] * rng.standard_normal(u.shape))
    return u


def device_rhs(solver, u_ref: np.ndarray, t: float, cuda):
    import torch
    nd = solver.mesh.ndims
    u = torch.from_numpy(ref_to_dev(u_ref, nd)).to(cuda)
    du = torch.empty_like(u)
    solver.rhs(u, du, t)
    torch.cuda.synchronize()
    return dev_to_ref(du.cpu().numpy(), solver.mesh.n_cells)


@pytest.mark.parametrize("name", list(CASES))
def test_rhs_matches_oracle(name, cuda):
    case = CASES[name]
    s = make_oracle(case)
    u = initial(case, s)
    du_o = do.rhs(s, u, 0.013)
    solver = make_device(case)
    du_d = device_rhs(solver, u, 0.013, cuda)
    assert rel_linf(du_d, du_o) <= RTOL, rel_linf(du_d, du_o)


@pytest.mark.parametrize("name", list(CASES))
def test_rhs_matches_reference(name, cuda):
    if not rb.available():
        pytest.skip("compiled reference not built")
    case = CASES[name]
    s = make_oracle(case)
    u = initial(case, s)
    kind = REF_KIND[(case["ic"], bool(case.get("shock_capturing")))]
    rc = rb.RefCase(kind, case["polydeg"], case["cells"], case["left"], case["right"])
    du_r = rc.rhs(u, 0.013)
    solver = make_device(case)
    du_d = device_rhs(solver, u, 0.013, cuda)
    assert rel_linf(du_d, du_r) <= RTOL, rel_linf(du_d, du_r)


@pytest.mark.parametrize("name", ["kh_hg", "dmr"])
def test_indicator_flags_identical(name, cuda):
    import torch
    case = CASES[name]
    s = make_oracle(case)
    u = initial(case, s)
    a_o = alpha_ref_to_dev(do.hg_alpha(s, u))
    solver = make_device(case)
    ud = torch.from_numpy(ref_to_dev(u, 2)).to(cuda)
    alpha, flags = solver.indicator(ud)
    alpha = alpha.cpu().numpy()
    flags = flags.cpu().numpy().astype(bool)
    assert np.array_equal(flags, a_o > do.hg_atol())
    assert np.max(np.abs(alpha - a_o)) <= 1e-15
    assert flags.any()


@pytest.mark.parametrize("name", ["kh", "dmr", "tgv"])
def test_ssprk3_step_matches_oracle(name, cuda):
    import torch

    import dgsem_b200 as D
    case = CASES[name]
    s = make_oracle(case)
    u = initial(case, s)
    dt = 2e-4
    u1_o = do.ssprk3_step(s, u, 0.0, dt)
    solver = make_device(case)
    sol = D.Solution(solver.mesh, solver.basis, solver.eq)
    sol.u.copy_(torch.from_numpy(ref_to_dev(u, case["ndims"])))
    integ = D.SSPRK3(sol, solver.mesh, dt)
    integ.step(solver, sol, dt)
    torch.cuda.synchronize()
    u1_d = dev_to_ref(sol.u.cpu().numpy(), solver.mesh.n_cells)
    assert rel_linf(u1_d - u, u1_o - u) <= 1e-10
    assert rel_linf(u1_d, u1_o) <= RTOL


@pytest.mark.parametrize("vf", ["ranocha", "kennedy_gruber"])
@pytest.mark.parametrize("sf", ["llf", "hllc"])
def test_other_fluxes_match_oracle(vf, sf, cuda):
    case = CASES["kh_hg"]
    s = make_oracle(case, vf, sf)
    u = initial(case, s)
    du_o = do.rhs(s, u, 0.0)
    solver = make_device(case, vf, sf)
    du_d = device_rhs(solver, u, 0.0, cuda)
    assert rel_linf(du_d, du_o) <= RTOL, rel_linf(du_d, du_o)


@pytest.mark.parametrize("vf", ["ranocha", "kennedy_gruber"])
def test_other_fluxes_3d(vf, cuda):
    case = CASES["tgv"]
    s = make_oracle(case, vf)
    u = initial(case, s)
    du_o = do.rhs(s, u, 0.0)
    solver = make_device(case, vf)
    du_d = device_rhs(solver, u, 0.0, cuda)
    assert rel_linf(du_d, du_o) <= RTOL, rel_linf(du_d, du_o)


@pytest.mark.parametrize("name", ["kh", "dmr", "tgv", "vortex_n6"])
def test_initial_condition_matches_oracle(name, cuda):
    import torch

    import dgsem_b200 as D
    case = CASES[name]
    s = make_oracle(case)
    u_o = initial(dict(case, noise=0), s)
    solver = make_device(case)
    sol = D.Solution(solver.mesh, solver.basis, solver.eq)
    ic = {"kh": D.KelvinHelmholtzInitial(), "dmr": D.DoubleMachReflectionInitial(),
          "tgv3d": D.InviscidTaylorGreenVortex(), "vortex": D.IsentropicVortex()}[case["ic"]]
    solver.initialize(ic, sol)
    torch.cuda.synchronize()
    u_d = dev_to_ref(sol.u.cpu().numpy(), solver.mesh.n_cells)
    assert rel_linf(u_d, u_o) <= 1e-14


def test_layout_round_trip(cuda):
    import torch
    case = CASES["tgv"]
    solver = make_device(case)
    rng = np.random.default_rng(3)
    u_ref = rng.standard_normal(tuple(case["cells"]) + (64, 5))
    ud = torch.from_numpy(ref_to_dev(u_ref, 3)).to(cuda)
    back = solver.to_reference_layout(ud).cpu().numpy()
    assert np.array_equal(back, u_ref)
    again = solver.from_reference_layout(torch.from_numpy(u_ref).to(cuda))
    assert torch.equal(again, ud)

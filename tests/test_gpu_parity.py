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
            ("vortex", False): rb.EULER2D_PERIODIC_SPLIT, ("tgv2d", False): rb.NS2D_PERIODIC_SPLIT}


def make_oracle(case: dict, volume_flux="chandrashekar", surface_flux="llf"):
    kw = {k: v for k, v in case.items() if k not in ("ic", "noise")}
    kw.setdefault("mu", 0.0)
    return do.Scheme(volume_flux=volume_flux, surface_flux=surface_flux, **kw)


def make_device(case: dict, volume_flux="chandrashekar", surface_flux="llf"):
    import dgsem_b200 as D
    nd = case["ndims"]
    mesh = D.StructuredMesh(case["left"], case["right"], case["cells"])
    eq = D.CompressibleEuler2D(1.4) if nd == 2 else D.CompressibleEuler3D(1.4)
    if case.get("viscous"):
        eq = D.CompressibleNavierStokes2D(1.4, case["mu"], case["prandtl"])
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
    if case.get("viscous") and case.get("noise"):
        rng = np.random.default_rng(seed)
        u[..., 1:3] += case["noise"] * rng.standard_normal(u[..., 1:3].shape)
    elif case.get("noise"):
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
    rc = rb.RefCase(kind, case["polydeg"], case["cells"], case["left"], case["right"],
                    mu=case.get("mu", 0.0), prandtl=case.get("prandtl", 0.72))
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


@pytest.mark.parametrize("name", ["kh", "dmr", "tgv", "ns"])
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


@pytest.mark.parametrize("name", ["kh", "dmr", "tgv", "vortex_n6", "ns"])
def test_initial_condition_matches_oracle(name, cuda):
    import torch

    import dgsem_b200 as D
    case = CASES[name]
    s = make_oracle(case)
    u_o = initial(dict(case, noise=0), s)
    solver = make_device(case)
    sol = D.Solution(solver.mesh, solver.basis, solver.eq)
    ic = {"kh": D.KelvinHelmholtzInitial(), "dmr": D.DoubleMachReflectionInitial(),
          "tgv3d": D.InviscidTaylorGreenVortex(), "vortex": D.IsentropicVortex(),
          "tgv2d": D.TaylorGreenVortex2D()}[case["ic"]]
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


def test_graph_replay_equals_stream_steps(cuda):
    """A captured CUDA graph of SSPRK3 steps (device clock for the
    time-dependent DMR boundary state) reproduces stream launches bitwise."""
    import ctypes

    import torch

    from dgsem_b200 import _capi as C
    case = CASES["dmr"]
    s = make_oracle(case)
    u0 = torch.from_numpy(ref_to_dev(initial(case, s), 2)).to(cuda)
    solver = make_device(case)
    L, h = C.lib(), solver.handle
    dt, t0 = 1.0e-4, 0.01
    a = u0.clone()
    C.check(L.dgsem_ssprk3_steps(h, ctypes.c_void_p(a.data_ptr()), t0, dt, 2), "steps")
    b = u0.clone()
    g = ctypes.c_void_p()
    C.check(L.dgsem_graph_create(h, ctypes.c_void_p(b.data_ptr()), dt, 2, ctypes.byref(g)),
            "graph")
    C.check(L.dgsem_graph_launch(g, t0), "launch")
    torch.cuda.synchronize()
    C.check(L.dgsem_graph_destroy(g), "destroy")
    assert torch.equal(a, b)


def test_host_buffer_steps_equal_device_steps(cuda):
    import ctypes

    import torch

    from dgsem_b200 import _capi as C
    case = CASES["tgv"]
    s = make_oracle(case)
    u0 = torch.from_numpy(ref_to_dev(initial(case, s), 3)).to(cuda)
    solver = make_device(case)
    L, h = C.lib(), solver.handle
    a = u0.clone()
    C.check(L.dgsem_ssprk3_steps(h, ctypes.c_void_p(a.data_ptr()), 0.0, 1e-3, 3), "steps")
    host = u0.cpu().pin_memory()
    C.check(L.dgsem_ssprk3_steps_host(h, ctypes.c_void_p(host.data_ptr()), 0.0, 1e-3, 3),
            "host steps")
    torch.cuda.synchronize()
    assert torch.equal(a.cpu(), host)


def test_deterministic_and_nonfinite_flag(cuda):
    import torch
    case = CASES["kh_hg"]
    s = make_oracle(case)
    u = torch.from_numpy(ref_to_dev(initial(case, s), 2)).to(cuda)
    solver = make_device(case)
    d1, d2 = torch.empty_like(u), torch.empty_like(u)
    solver.rhs(u, d1, 0.0)
    solver.rhs(u, d2, 0.0)
    torch.cuda.synchronize()
    assert torch.equal(d1, d2)
    solver.check_finite()
    bad = u.clone()
    bad[3, 0, 5] = float("nan")
    solver.rhs(bad, d1, 0.0)
    import dgsem_b200
    with pytest.raises(dgsem_b200.DgsemError):
        solver.check_finite()
    solver.check_finite()  # flag cleared


def test_conservation_and_free_stream_large(cuda):
    """Size-independent properties at a benchmark size (TGV 16^3):
    discrete conservation sum_i w_i J du_i = 0 and free-stream preservation."""
    import torch

    import dgsem_b200 as D
    mesh = D.StructuredMesh((0.0,) * 3, (2 * np.pi,) * 3, (16, 16, 16))
    solver = D.StructuredSolver(D.CompressibleEuler3D(1.4), D.LobattoLegendreBasis(3),
                                D.VolumeIntegralSplitForm(D.KennedyGruberFlux),
                                D.LaxFriedrichsFlux(), mesh,
                                D.BoundarySet(*[D.PeriodicBC() for _ in range(6)]))
    sol = D.Solution(mesh, D.LobattoLegendreBasis(3), D.CompressibleEuler3D(1.4))
    solver.initialize(D.InviscidTaylorGreenVortex(), sol)
    solver.calc_rhs(sol, 0.0)
    w = torch.tensor(do.Basis(3).weights, dtype=torch.float64, device=cuda)
    W = (w[None, None, :] * w[None, :, None] * w[:, None, None]).reshape(-1)
    jac = (2 * np.pi / 16 / 2) ** 3
    tot = (sol.du * W[None, None, :]).sum(dim=(0, 2)) * jac
    assert float(tot.abs().max()) <= 1e-10 * float(sol.du.abs().max()) * sol.du.shape[0]
    fs = torch.empty_like(sol.u)
    fs[:, 0], fs[:, 1], fs[:, 2], fs[:, 3] = 1.0, 0.3, -0.2, 0.1
    fs[:, 4] = 71.4 / 0.4 + 0.5 * (0.09 + 0.04 + 0.01)
    du = torch.empty_like(fs)
    solver.rhs(fs, du, 0.0)
    # the residual is the reference metric round-off (~1e-12 relative in 3D,
    # curl-form metrics) times the flux scale |u| / h
    h = 2 * np.pi / 16
    assert float(du.abs().max()) <= 1e-10 * float(fs.abs().max()) / h


@pytest.mark.parametrize("name", ["kh", "kh_hg", "dmr", "tgv", "tgv_partial", "ns", "vortex_n6"])
def test_launch_variants(name, cuda):
    """The line-parallel launch shapes give the same bits, the node-parallel
    shape agrees to rounding and with the oracle, and the autotuner leaves
    the state untouched and keeps a valid shape."""
    import torch
    case = CASES[name]
    s = make_oracle(case)
    u_ref = initial(case, s)
    solver = make_device(case)
    nd = solver.mesh.ndims
    u = torch.from_numpy(ref_to_dev(u_ref, nd)).to(cuda)
    u_copy = u.clone()
    outs = []
    for v in range(3):
        solver.set_launch_variant(v)
        du = torch.empty_like(u)
        solver.rhs(u, du, 0.05)
        outs.append(du)
    torch.cuda.synchronize()
    for v in (1, 2):
        assert torch.equal(outs[0], outs[v]), v
    # node-parallel shapes 3-4 (also with shock capturing or Navier-Stokes)
    # and the persistent shape 5 (neither): same arithmetic per flux,
    # different summation order; 3, 4 and 5 give the same bits
    node_variant = True
    pipe_variant = not case.get("shock_capturing") and not case.get("viscous")
    if node_variant:
        node_outs = []
        for v in ((3, 4, 5) if pipe_variant else (3, 4)):
            solver.set_launch_variant(v)
            du3 = torch.empty_like(u)
            solver.rhs(u, du3, 0.05)
            node_outs.append(du3)
        torch.cuda.synchronize()
        for other in node_outs[1:]:
            assert torch.equal(node_outs[0], other)
        a, b = node_outs[0].cpu().numpy(), outs[0].cpu().numpy()
        assert rel_linf(a, b) <= RTOL
        assert rel_linf(dev_to_ref(a, solver.mesh.n_cells), do.rhs(s, u_ref, 0.05)) <= RTOL
    else:
        with pytest.raises(Exception):
            solver.set_launch_variant(3)
    if not pipe_variant:
        with pytest.raises(Exception):
            solver.set_launch_variant(5)
    # two nodes per thread (3D, n = 2 or 4, split form): the same fluxes, z
    # pairs shared between threads (another summation order)
    node2_variant = pipe_variant and nd == 3 and case["polydeg"] in (1, 3)
    if node2_variant:
        solver.set_launch_variant(6)
        du6 = torch.empty_like(u)
        solver.rhs(u, du6, 0.05)
        torch.cuda.synchronize()
        a = du6.cpu().numpy()
        assert rel_linf(a, outs[0].cpu().numpy()) <= RTOL
        assert rel_linf(dev_to_ref(a, solver.mesh.n_cells), do.rhs(s, u_ref, 0.05)) <= RTOL
    else:
        with pytest.raises(Exception):
            solver.set_launch_variant(6)
    nvar = 7 if node2_variant else 6 if pipe_variant else 5 if node_variant else 3
    chosen, times = solver.autotune(u, retime=True)
    torch.cuda.synchronize()
    assert chosen in range(nvar)
    assert all(t > 0.0 for t in times[:nvar])
    assert torch.equal(u, u_copy)
    du = torch.empty_like(u)
    solver.rhs(u, du, 0.05)
    torch.cuda.synchronize()
    if chosen < 3:
        assert torch.equal(du, outs[0])


@pytest.mark.parametrize("vf", ["chandrashekar", "ranocha", "kennedy_gruber"])
@pytest.mark.parametrize("sf", ["llf", "hllc"])
def test_node_parallel_variant_other_fluxes(vf, sf, cuda):
    """The node-parallel launch shape with every two-point / surface flux
    (plain split form) against the oracle, 2D KH and (LLF) 3D TGV."""
    for name in (["kh", "tgv"] if sf == "llf" else ["kh"]):
        case = CASES[name]
        s = make_oracle(case, vf, sf)
        u = initial(case, s, seed=3)
        du_o = do.rhs(s, u, 0.0)
        solver = make_device(case, vf, sf)
        solver.set_launch_variant(3)
        du_d = device_rhs(solver, u, 0.0, cuda)
        assert rel_linf(du_d, du_o) <= RTOL, (name, rel_linf(du_d, du_o))


def test_node_parallel_variant_dmr_boundaries(cuda):
    """Node-parallel shape with the DMR boundary conditions (no shock
    capturing: the same BC code path as the line-parallel shapes)."""
    case = dict(CASES["dmr"])
    case.pop("shock_capturing")
    s = make_oracle(case, "chandrashekar", "llf")
    u = initial(case, s)
    t = 0.02
    du_o = do.rhs(s, u, t)
    solver = make_device(case)
    solver.set_launch_variant(3)
    du_d = device_rhs(solver, u, t, cuda)
    assert rel_linf(du_d, du_o) <= RTOL, rel_linf(du_d, du_o)


@pytest.mark.parametrize("name,sf", [("kh_hg", "llf"), ("kh_hg", "hllc"), ("dmr", "llf"),
                                     ("dmr", "hllc")])
def test_node_parallel_shock_capturing(name, sf, cuda):
    """Node-parallel shapes with Hennemann-Gassner blending (same alpha and
    flags as the line-parallel kernel: any flag flip would move the RHS by far
    more than the bar) against the oracle, incl. the DMR boundary states."""
    case = CASES[name]
    s = make_oracle(case, "chandrashekar", sf)
    u = initial(case, s, seed=5)
    t = 0.02 if name == "dmr" else 0.0
    du_o = do.rhs(s, u, t)
    solver = make_device(case, "chandrashekar", sf)
    for v in (3, 4):
        solver.set_launch_variant(v)
        du_d = device_rhs(solver, u, t, cuda)
        assert rel_linf(du_d, du_o) <= RTOL, (v, rel_linf(du_d, du_o))

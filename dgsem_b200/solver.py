"""Host-side mirror of the reference's solver interface over the C ABI.

Names and argument meaning follow RetrO598/DGSEM:
  StructuredMesh(domain_left, domain_right, n_cells)   mesh/structured_mesh.hpp:10-71
  LobattoLegendreBasis(polydeg)                         polynomial_basis/basis.hpp:12-182
  CompressibleEuler2D/3D, CompressibleNavierStokes2D/3D equations/*.hpp
  ChandrashekarFlux, LaxFriedrichsFlux (+ RanochaFlux, KennedyGruberFlux, HLLCFlux)
  VolumeIntegralSplitForm, VolumeIntegralShockCapturingHG, HGIndicator
                                                        space_integral/volume_flux.hpp:686-879
  PeriodicBC, DirichletBC, OutflowBC, MixedDirichletSlipWallBC, BoundarySet
                                                        boundary_condition/*.hpp
  StructuredSolver(eq, basis, volume, surface, mesh, boundaries)
      .initialize(ic, sol) .calc_rhs(sol, t) .set_indicator_parameters(...)
      .get_ndofs()                                      solver/structured_solver.hpp:18-143
  Solution(mesh, basis, eq) .state() .rhs() .clone_shape()
                                                        containers/solution_container.hpp:157-234
  SSPRK3(sol, mesh, final_time) .step(solver, sol, dt) .solve(solver, sol, dt)
                                                        time_integrator/SSPRK3.hpp:145-187
Templates become descriptor objects; state arrays are caller-visible CUDA
tensors in the device layout u[e][var][node] (include/dgsem_b200.h).  Every
compute call runs the CUDA kernels of libdgsem_b200.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import torch

from . import _capi as C


# ---------------------------------------------------------------- mesh/basis
@dataclass
class StructuredMesh:
    domain_left: tuple
    domain_right: tuple
    n_cells: tuple

    @property
    def ndims(self) -> int:
        return len(self.n_cells)

    def get_num_cells(self):
        return tuple(self.n_cells)

    def get_nelem(self) -> int:
        return int(math.prod(self.n_cells))


@dataclass(frozen=True)
class LobattoLegendreBasis:
    polydeg: int

    @property
    def NNodes(self) -> int:
        return self.polydeg + 1


# ---------------------------------------------------------------- equations
@dataclass(frozen=True)
class CompressibleEuler2D:
    gamma: float = 1.4
    NDIMS = 2
    NVARS = 4
    code = C.EULER_2D


@dataclass(frozen=True)
class CompressibleEuler3D:
    gamma: float = 1.4
    NDIMS = 3
    NVARS = 5
    code = C.EULER_3D


@dataclass(frozen=True)
class CompressibleNavierStokes2D:
    gamma: float = 1.4
    mu: float = 5.0e-3
    prandtl: float = 0.73
    NDIMS = 2
    NVARS = 4
    code = C.NAVIER_STOKES_2D


@dataclass(frozen=True)
class CompressibleNavierStokes3D:
    """equations/compressible_navier_stokes3D.hpp (periodic boxes: the
    reference's 3D Navier-Stokes setups are periodic)."""
    gamma: float = 1.4
    mu: float = 6.25e-4
    prandtl: float = 0.72
    NDIMS = 3
    NVARS = 5
    code = C.NAVIER_STOKES_3D


# ---------------------------------------------------------------- fluxes
class ChandrashekarFlux:
    code = C.VF_CHANDRASHEKAR


class RanochaFlux:
    code = C.VF_RANOCHA


class KennedyGruberFlux:
    code = C.VF_KENNEDY_GRUBER


class LaxFriedrichsFlux:
    code = C.SF_LAX_FRIEDRICHS


class HLLCFlux:
    code = C.SF_HLLC


class HGIndicator:
    """Hennemann-Gassner indicator (subcell_limiting/indicator.hpp)."""


@dataclass(frozen=True)
class VolumeIntegralSplitForm:
    numerical_flux: type = ChandrashekarFlux
    code = C.VI_SPLIT_FORM


@dataclass(frozen=True)
class VolumeIntegralShockCapturingHG:
    numerical_flux: type = ChandrashekarFlux
    fv_flux: type = LaxFriedrichsFlux
    indicator: type = HGIndicator
    code = C.VI_SHOCK_CAPTURING_HG

    def __post_init__(self):
        if self.fv_flux is not LaxFriedrichsFlux:
            raise ValueError("the FV subcell flux is LaxFriedrichsFlux")


# ---------------------------------------------------------------- boundaries
class PeriodicBC:
    code = C.BC_PERIODIC


class OutflowBC:
    code = C.BC_OUTFLOW


@dataclass(frozen=True)
class DirichletBC:
    """Dirichlet state: a constant conserved state, or "double_mach" for the
    double Mach reflection state f(x, t) of the reference example."""

    func: object = "double_mach"

    @property
    def code(self):
        return C.BC_DIRICHLET_DMR if self.func == "double_mach" else C.BC_DIRICHLET_CONST


@dataclass(frozen=True)
class MixedDirichletSlipWallBC:
    """Dirichlet (double Mach state) where x < 1/6, reflecting wall elsewhere."""

    func: object = "double_mach"
    code = C.BC_MIXED_DMR_WALL


class SlipWallBC:
    code = C.BC_SLIP_WALL


class NSNoSlipAdiabaticWallBC:
    """navier_stokes_wall_boundary.hpp:33-132 (Navier-Stokes only)."""
    code = C.BC_NS_NOSLIP_ADIABATIC_WALL


class NSSlipAdiabaticWallBC:
    """navier_stokes_wall_boundary.hpp:134-219 (Navier-Stokes only)."""
    code = C.BC_NS_SLIP_ADIABATIC_WALL


class BoundarySet:
    """One boundary condition per face: left, right, bottom, top(, back, front)."""

    def __init__(self, *bcs):
        self.faces = list(bcs)
        self.NFACES = len(bcs)


# ---------------------------------------------------------------- initial conditions
@dataclass(frozen=True)
class KelvinHelmholtzInitial:
    code = C.IC_KELVIN_HELMHOLTZ
    params = None


@dataclass(frozen=True)
class DoubleMachReflectionInitial:
    gamma: float = 1.4
    code = C.IC_DOUBLE_MACH
    params = None


@dataclass(frozen=True)
class InviscidTaylorGreenVortex:
    code = C.IC_TAYLOR_GREEN_3D
    params = None


@dataclass(frozen=True)
class TaylorGreenVortex2D:
    p0: float = 1.0 / (1.4 * 0.01)
    code = C.IC_TAYLOR_GREEN_2D

    @property
    def params(self):
        return (self.p0, 0.0, 0.0)


@dataclass(frozen=True)
class IsentropicVortex:
    beta: float = 5.0
    center: tuple = (0.0, 0.0)
    code = C.IC_ISENTROPIC_VORTEX

    @property
    def params(self):
        return (self.beta, self.center[0], self.center[1])


# ---------------------------------------------------------------- solution
class Solution:
    """State (u) and RHS (du) device arrays, shape (nelem, nvars, n^d)."""

    def __init__(self, mesh: StructuredMesh, basis: LobattoLegendreBasis, equations,
                 device=None):
        self.mesh, self.basis, self.equations = mesh, basis, equations
        self.shape = (mesh.get_nelem(), equations.NVARS, basis.NNodes ** mesh.ndims)
        dev = device or torch.device("cuda", torch.cuda.current_device())
        self.u = torch.zeros(self.shape, dtype=torch.float64, device=dev)
        self.du = torch.zeros_like(self.u)

    def state(self) -> torch.Tensor:
        return self.u

    def rhs(self) -> torch.Tensor:
        return self.du

    def clone_shape(self) -> "Solution":
        return Solution(self.mesh, self.basis, self.equations, device=self.u.device)


def _ptr(t: torch.Tensor):
    if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
        raise ValueError("expected a contiguous float64 CUDA tensor")
    return ctypes.c_void_p(t.data_ptr())


# ---------------------------------------------------------------- solver
class StructuredSolver:
    def __init__(self, equations, basis: LobattoLegendreBasis, volume_integral,
                 surface_flux, mesh: StructuredMesh, boundary_set: BoundarySet,
                 stream: torch.cuda.Stream | None = None):
        if not torch.cuda.is_available():
            raise RuntimeError("StructuredSolver needs a CUDA device (no CPU path)")
        if boundary_set.NFACES != 2 * mesh.ndims:
            raise ValueError("one boundary condition per mesh face is required "
                             "(2 for 1D, 4 for 2D, 6 for 3D)")
        self.eq, self.basis, self.vi, self.sf = equations, basis, volume_integral, surface_flux
        self.mesh, self.boundary_set = mesh, boundary_set
        m = C.MeshDesc()
        m.ndims = mesh.ndims
        m.polydeg = basis.polydeg
        for a in range(3):
            m.n_cells[a] = int(mesh.n_cells[a]) if a < mesh.ndims else 1
            m.domain_left[a] = float(mesh.domain_left[a]) if a < mesh.ndims else 0.0
            m.domain_right[a] = float(mesh.domain_right[a]) if a < mesh.ndims else 1.0
        s = C.SchemeDesc()
        s.equation = equations.code
        s.volume_flux = volume_integral.numerical_flux.code
        s.surface_flux = surface_flux.code
        s.volume_integral = volume_integral.code
        for f, bc in enumerate(boundary_set.faces):
            s.bc[f] = bc.code
            if isinstance(bc, DirichletBC) and bc.func != "double_mach":
                for q, v in enumerate(bc.func):
                    s.bc_state[q] = float(v)
        s.gamma = equations.gamma
        s.mu = getattr(equations, "mu", 0.0)
        s.prandtl = getattr(equations, "prandtl", 0.72)
        s.alpha_max, s.alpha_min, s.alpha_smooth = 0.5, 0.001, 0
        self._mesh_desc, self._scheme_desc = m, s
        self.stream = stream or torch.cuda.current_stream()
        h = ctypes.c_void_p()
        C.check(C.lib().dgsem_ctx_create(ctypes.byref(m), ctypes.byref(s),
                                         ctypes.c_void_p(self.stream.cuda_stream),
                                         ctypes.byref(h)), "dgsem_ctx_create")
        self._ctx = h

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx is not None and ctx.value:
            C.lib().dgsem_ctx_destroy(ctx)
            self._ctx = None

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._ctx

    def get_ndofs(self) -> int:
        return self.basis.NNodes ** self.mesh.ndims

    def set_indicator_parameters(self, alpha_max: float, alpha_min: float,
                                 alpha_smooth: bool = False) -> None:
        C.check(C.lib().dgsem_set_indicator_parameters(self._ctx, alpha_max, alpha_min,
                                                       int(alpha_smooth)),
                "dgsem_set_indicator_parameters")

    def initialize(self, initial_condition, sol: Solution) -> None:
        params = initial_condition.params
        arr = (ctypes.c_double * 3)(*params) if params is not None else None
        C.check(C.lib().dgsem_initial_condition(self._ctx, initial_condition.code, arr,
                                                _ptr(sol.u)), "dgsem_initial_condition")

    def calc_rhs(self, sol: Solution, time: float) -> None:
        C.check(C.lib().dgsem_rhs(self._ctx, _ptr(sol.u), _ptr(sol.du), float(time)),
                "dgsem_rhs")

    def rhs(self, u: torch.Tensor, du: torch.Tensor, time: float = 0.0) -> None:
        C.check(C.lib().dgsem_rhs(self._ctx, _ptr(u), _ptr(du), float(time)), "dgsem_rhs")

    def indicator(self, u: torch.Tensor):
        """HG alpha per element and troubled-cell flags (uint8)."""
        n = self.mesh.get_nelem()
        alpha = torch.empty(n, dtype=torch.float64, device=u.device)
        flags = torch.empty(n, dtype=torch.uint8, device=u.device)
        C.check(C.lib().dgsem_indicator(self._ctx, _ptr(u), ctypes.c_void_p(alpha.data_ptr()),
                                        ctypes.c_void_p(flags.data_ptr())), "dgsem_indicator")
        return alpha, flags

    def to_reference_layout(self, u: torch.Tensor) -> torch.Tensor:
        out = torch.empty_like(u)
        C.check(C.lib().dgsem_to_reference_layout(self._ctx, _ptr(u), _ptr(out)),
                "dgsem_to_reference_layout")
        return out.reshape(tuple(self.mesh.n_cells) + (u.shape[2], u.shape[1]))

    def from_reference_layout(self, u_ref: torch.Tensor) -> torch.Tensor:
        n = self.mesh.get_nelem()
        src = u_ref.contiguous().reshape(n, -1)
        out = torch.empty((n, self.eq.NVARS, self.get_ndofs()), dtype=torch.float64,
                          device=u_ref.device)
        C.check(C.lib().dgsem_from_reference_layout(self._ctx, _ptr(src), _ptr(out)),
                "dgsem_from_reference_layout")
        return out

    def check_finite(self) -> None:
        C.check(C.lib().dgsem_check_finite(self._ctx), "dgsem_check_finite")

    def autotune(self, u: torch.Tensor, retime: bool = False):
        """Picks the fastest launch shape for this mesh (results are identical
        across shapes); returns (variant, per-variant ms or None)."""
        chosen = ctypes.c_int()
        times = (ctypes.c_double * 7)() if retime else None
        C.check(C.lib().dgsem_autotune(self._ctx, _ptr(u), ctypes.byref(chosen), times),
                "dgsem_autotune")
        return chosen.value, (list(times) if retime else None)

    def set_launch_variant(self, variant: int) -> None:
        C.check(C.lib().dgsem_set_launch_variant(self._ctx, int(variant)),
                "dgsem_set_launch_variant")

    def launch_count(self) -> int:
        c = ctypes.c_int64()
        C.check(C.lib().dgsem_launch_count(self._ctx, ctypes.byref(c)), "dgsem_launch_count")
        return c.value


# ---------------------------------------------------------------- time integration
class SSPRK3:
    """Shu-Osher SSPRK3 with each stage one fused kernel (SSPRK3.hpp:145-187)."""

    def __init__(self, sol: Solution, mesh: StructuredMesh, final_time: float = 0.0):
        self.mesh = mesh
        self.time = 0.0
        self.final_time = final_time
        self.iter = 0
        self.has_nan = False
        self.observers = []
        self.tmp1 = sol.clone_shape()
        self.tmp2 = sol.clone_shape()

    def add_observer(self, observer) -> None:
        self.observers.append(observer)

    def step(self, solver: StructuredSolver, sol: Solution, dt: float) -> None:
        L, h = C.lib(), solver.handle
        t = self.time
        C.check(L.dgsem_ssprk3_stage(h, 1, None, _ptr(sol.u), _ptr(self.tmp1.u), t, dt), "stage 1")
        C.check(L.dgsem_ssprk3_stage(h, 2, _ptr(sol.u), _ptr(self.tmp1.u), _ptr(self.tmp2.u),
                                     t, dt), "stage 2")
        C.check(L.dgsem_ssprk3_stage(h, 3, _ptr(sol.u), _ptr(self.tmp2.u), _ptr(sol.u), t, dt),
                "stage 3")

    def solve_steps(self, solver: StructuredSolver, sol: Solution, dt: float, nsteps: int) -> None:
        for _ in range(nsteps):
            self.step(solver, sol, dt)
            self.time += dt
            self.iter += 1

    def solve(self, solver: StructuredSolver, sol: Solution, dt: float) -> None:
        """integrator_base.hpp:21-40: fixed dt until final_time, NaN stops.

        Observers are objects with the reference's on_step(step, time) ->
        stop flag and on_finish(step, time) (observer/observer_base.hpp:4-9),
        or plain callables obs(step, time, sol)."""
        stop = False
        while self.time < self.final_time and not stop:
            for obs in self.observers:
                if hasattr(obs, "on_step"):
                    stop = bool(obs.on_step(self.iter, self.time)) or stop
                else:
                    obs(self.iter, self.time, sol)
            if stop:
                break
            self.step(solver, sol, dt)
            self.time += dt
            self.iter += 1
            try:
                solver.check_finite()
            except C.DgsemError:
                self.has_nan = True
                break
        for obs in self.observers:
            if hasattr(obs, "on_finish"):
                obs.on_finish(self.iter, self.time)


# ---------------------------------------------------------------- output
class VTUOutputObserver:
    """VTUOutputObserver (observer/vtu_output_observer.hpp:17-235) without VTK:
    writes <output_path>_step<step>.vtu at step 0, every output_interval
    steps (never when it is negative) and at the end if the last step was not
    written; Lagrange cells, point data rho, momentum, rhoE, pressure
    (dgsem_write_vtu)."""

    def __init__(self, output_path: str, solver: StructuredSolver, sol: Solution,
                 output_interval: int = -1):
        self.output_path, self.solver, self.sol = output_path, solver, sol
        self.output_interval = output_interval
        self.last_written_step = -1
        self.written = []

    def filename(self, step: int) -> str:
        return f"{self.output_path}_step{step}.vtu"

    def write(self, step: int) -> None:
        torch.cuda.synchronize()
        name = self.filename(step)
        C.check(C.lib().dgsem_write_vtu(self.solver.handle, _ptr(self.sol.u), name.encode()),
                "dgsem_write_vtu")
        self.last_written_step = step
        self.written.append(name)

    def on_step(self, step: int, time: float) -> bool:
        if step == 0 or (self.output_interval > 0 and step % self.output_interval == 0):
            if step != self.last_written_step:
                self.write(step)
        return False

    def on_finish(self, step: int, time: float) -> None:
        if step != self.last_written_step:
            self.write(step)


def write_checkpoint(path: str, solver: StructuredSolver, sol: Solution, time: float,
                     step: int) -> None:
    """Binary checkpoint of the state, time and step (dgsem_checkpoint_write)."""
    torch.cuda.synchronize()
    C.check(C.lib().dgsem_checkpoint_write(solver.handle, _ptr(sol.u), float(time), int(step),
                                           path.encode()), "dgsem_checkpoint_write")


def read_checkpoint(path: str, solver: StructuredSolver, sol: Solution):
    """Restores the state from a checkpoint of the same mesh; returns (time, step)."""
    t, k = ctypes.c_double(), ctypes.c_int64()
    C.check(C.lib().dgsem_checkpoint_read(solver.handle, _ptr(sol.u), ctypes.byref(t),
                                          ctypes.byref(k), path.encode()),
            "dgsem_checkpoint_read")
    return t.value, k.value


# ---------------------------------------------------------------- discrete adjoint
class Adjoint:
    """Discrete adjoint of a StructuredSolver's right-hand side and of SSPRK3
    (dgsem_adjoint_* in include/dgsem_b200.h): 2D periodic meshes, the
    Chandrashekar split form with the LLF surface flux, Euler or
    Navier-Stokes.  `nsteps` SSPRK3 steps with a checkpoint every
    `checkpoint_every` steps."""

    def __init__(self, solver: StructuredSolver, nsteps: int, checkpoint_every: int = 20):
        self.solver = solver
        self.nsteps, self.checkpoint_every = int(nsteps), int(checkpoint_every)
        h = ctypes.c_void_p()
        C.check(C.lib().dgsem_adjoint_create(solver.handle, self.nsteps, self.checkpoint_every,
                                             ctypes.byref(h)), "dgsem_adjoint_create")
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            C.lib().dgsem_adjoint_destroy(h)
            self._h = None

    def rhs_vjp(self, u: torch.Tensor, w: torch.Tensor) -> torch.Tensor:
        """(dR/du(u))^T w."""
        out = torch.empty_like(w)
        C.check(C.lib().dgsem_adjoint_rhs_vjp(self._h, _ptr(u), _ptr(w), _ptr(out)),
                "dgsem_adjoint_rhs_vjp")
        return out

    def kinetic_energy(self, u: torch.Tensor, grad: bool = False):
        """Mean kinetic energy J(u) (and dJ/du when grad is True)."""
        val = ctypes.c_double()
        g = torch.empty_like(u) if grad else None
        C.check(C.lib().dgsem_kinetic_energy(self._h, _ptr(u), ctypes.byref(val),
                                             _ptr(g) if grad else None),
                "dgsem_kinetic_energy")
        return (val.value, g) if grad else val.value

    def gradient(self, u0: torch.Tensor, t0: float, dt: float):
        """J(u(t0 + nsteps dt)) and dJ/du0 (all variables; u0 is not modified)."""
        val = ctypes.c_double()
        g = torch.empty_like(u0)
        C.check(C.lib().dgsem_adjoint_gradient(self._h, _ptr(u0), float(t0), float(dt),
                                               ctypes.byref(val), _ptr(g)),
                "dgsem_adjoint_gradient")
        return val.value, g


# ---------------------------------------------------------------- batched mode
class BatchSolver:
    """Many independent periodic meshes (uneven sizes and degrees) sharing one
    scheme, advanced together (dgsem_batch_* in include/dgsem_b200.h).

    `meshes` is a list of (StructuredMesh, polydeg); the states of all meshes
    live in one device array `u` of length offsets[-1]; mesh m's state is
    u[offsets[m]:offsets[m+1]] in the single-mesh layout.
    """

    def __init__(self, equations, meshes, volume_flux=ChandrashekarFlux,
                 surface_flux=LaxFriedrichsFlux, stream: torch.cuda.Stream | None = None):
        if not torch.cuda.is_available():
            raise RuntimeError("BatchSolver needs a CUDA device (no CPU path)")
        self.eq = equations
        self.meshes = list(meshes)
        n = len(self.meshes)
        arr = (C.MeshDesc * n)()
        for k, (mesh, N) in enumerate(self.meshes):
            d = arr[k]
            d.ndims = mesh.ndims
            d.polydeg = int(N)
            for a in range(3):
                d.n_cells[a] = int(mesh.n_cells[a]) if a < mesh.ndims else 1
                d.domain_left[a] = float(mesh.domain_left[a]) if a < mesh.ndims else 0.0
                d.domain_right[a] = float(mesh.domain_right[a]) if a < mesh.ndims else 1.0
        s = C.SchemeDesc()
        s.equation = equations.code
        s.volume_flux = volume_flux.code
        s.surface_flux = surface_flux.code
        s.volume_integral = C.VI_SPLIT_FORM
        s.gamma = equations.gamma
        s.alpha_max, s.alpha_min = 0.5, 0.001
        self.stream = stream or torch.cuda.current_stream()
        h = ctypes.c_void_p()
        C.check(C.lib().dgsem_batch_create(arr, n, ctypes.byref(s),
                                           ctypes.c_void_p(self.stream.cuda_stream),
                                           ctypes.byref(h)), "dgsem_batch_create")
        self._h = h
        offs = (ctypes.c_int64 * (n + 1))()
        C.check(C.lib().dgsem_batch_offsets(h, offs), "dgsem_batch_offsets")
        self.offsets = list(offs)
        self.u = torch.zeros(self.offsets[-1], dtype=torch.float64,
                             device=torch.device("cuda", torch.cuda.current_device()))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            C.lib().dgsem_batch_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def mesh_state(self, m: int, u: torch.Tensor | None = None) -> torch.Tensor:
        mesh, N = self.meshes[m]
        u = self.u if u is None else u
        nodes = (N + 1) ** mesh.ndims
        return u[self.offsets[m]:self.offsets[m + 1]].view(mesh.get_nelem(),
                                                            self.eq.NVARS, nodes)

    def initialize(self, kind: int, params=None) -> None:
        arr = None
        if params is not None:
            flat = [float(x) for p in params for x in p]
            arr = (ctypes.c_double * len(flat))(*flat)
        C.check(C.lib().dgsem_batch_initial_condition(self._h, int(kind), arr,
                                                      ctypes.c_void_p(self.u.data_ptr())),
                "dgsem_batch_initial_condition")

    def step(self, t: float, dt, u: torch.Tensor | None = None) -> None:
        u = self.u if u is None else u
        dts = (ctypes.c_double * len(self.meshes))(*[float(x) for x in dt])
        C.check(C.lib().dgsem_batch_ssprk3_step(self._h, ctypes.c_void_p(u.data_ptr()),
                                                float(t), dts), "dgsem_batch_ssprk3_step")

    def graph(self, dt, nsteps: int, u: torch.Tensor | None = None) -> "BatchGraph":
        return BatchGraph(self, dt, nsteps, self.u if u is None else u)

    def check_finite(self) -> None:
        C.check(C.lib().dgsem_batch_check_finite(self._h), "dgsem_batch_check_finite")

    def autotune(self, dt, u: torch.Tensor | None = None):
        u = self.u if u is None else u
        ndeg = len({N for _, N in self.meshes})
        chosen = (ctypes.c_int * ndeg)()
        dts = (ctypes.c_double * len(self.meshes))(*[float(x) for x in dt])
        C.check(C.lib().dgsem_batch_autotune(self._h, ctypes.c_void_p(u.data_ptr()), dts,
                                             chosen), "dgsem_batch_autotune")
        return list(chosen)

    def set_launch_variant(self, variant: int) -> None:
        """One launch shape for every degree group (dgsem_batch_set_launch_variant)."""
        C.check(C.lib().dgsem_batch_set_launch_variant(self._h, int(variant)),
                "dgsem_batch_set_launch_variant")

    def set_persistent(self, enable: bool = True) -> None:
        """One persistent launch per stage over all meshes (dgsem_batch_set_persistent)."""
        C.check(C.lib().dgsem_batch_set_persistent(self._h, int(enable)),
                "dgsem_batch_set_persistent")

    def launch_count(self) -> int:
        c = ctypes.c_int64()
        C.check(C.lib().dgsem_batch_launch_count(self._h, ctypes.byref(c)),
                "dgsem_batch_launch_count")
        return c.value


class BatchGraph:
    """CUDA graph of `nsteps` batched SSPRK3 steps (replayed with launch())."""

    def __init__(self, batch: BatchSolver, dt, nsteps: int, u: torch.Tensor):
        self.batch = batch
        dts = (ctypes.c_double * len(batch.meshes))(*[float(x) for x in dt])
        g = ctypes.c_void_p()
        C.check(C.lib().dgsem_batch_graph_create(batch.handle, ctypes.c_void_p(u.data_ptr()),
                                                 dts, int(nsteps), ctypes.byref(g)),
                "dgsem_batch_graph_create")
        self._g = g

    def launch(self) -> None:
        C.check(C.lib().dgsem_batch_graph_launch(self._g), "dgsem_batch_graph_launch")

    def __del__(self):
        g = getattr(self, "_g", None)
        if g is not None and g.value:
            C.lib().dgsem_batch_graph_destroy(g)
            self._g = None

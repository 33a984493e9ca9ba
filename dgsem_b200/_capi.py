"""ctypes declarations of the C ABI in include/dgsem_b200.h.

The library is dgsem_b200/_lib/libdgsem_b200.so, built in-tree by
``python -m dgsem_b200.build``.  There is no fallback: if the library is
missing, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libdgsem_b200.so")

DGSEM_OK = 0
STATUS_NAMES = {0: "ok", 1: "invalid argument", 2: "unsupported combination",
                3: "CUDA error", 4: "non-finite value in state",
                5: "device wait timed out", 6: "allocation failed",
                7: "state larger than the static scratch"}
DGSEM_ERR_INVALID_ARG, DGSEM_ERR_UNSUPPORTED, DGSEM_ERR_CUDA = 1, 2, 3
DGSEM_ERR_NONFINITE, DGSEM_ERR_TIMEOUT, DGSEM_ERR_ALLOC = 4, 5, 6
DGSEM_ERR_SCRATCH_LIMIT = 7
STATIC_SCRATCH_MAX_STATE = 2097152  # DGSEM_STATIC_SCRATCH_MAX_STATE (doubles per stage state)

# enums (include/dgsem_b200.h)
EULER_2D, EULER_3D, NAVIER_STOKES_2D, NAVIER_STOKES_3D = 0, 1, 2, 3
VF_CHANDRASHEKAR, VF_RANOCHA, VF_KENNEDY_GRUBER = 0, 1, 2
SF_LAX_FRIEDRICHS, SF_HLLC = 0, 1
VI_SPLIT_FORM, VI_SHOCK_CAPTURING_HG = 0, 1
BC_PERIODIC, BC_DIRICHLET_DMR, BC_OUTFLOW, BC_MIXED_DMR_WALL = 0, 1, 2, 3
BC_DIRICHLET_CONST, BC_SLIP_WALL = 4, 5
BC_NS_NOSLIP_ADIABATIC_WALL, BC_NS_SLIP_ADIABATIC_WALL = 6, 7
IC_KELVIN_HELMHOLTZ, IC_DOUBLE_MACH, IC_TAYLOR_GREEN_3D = 0, 1, 2
IC_TAYLOR_GREEN_2D, IC_ISENTROPIC_VORTEX = 3, 4

EXPORTED = [
    "dgsem_status_string", "dgsem_ctx_create", "dgsem_ctx_destroy",
    "dgsem_ctx_set_stream", "dgsem_get_sizes", "dgsem_set_indicator_parameters",
    "dgsem_rhs", "dgsem_ssprk3_stage", "dgsem_ssprk3_step", "dgsem_ssprk3_steps",
    "dgsem_indicator", "dgsem_initial_condition", "dgsem_to_reference_layout",
    "dgsem_from_reference_layout", "dgsem_check_finite", "dgsem_launch_count",
    "dgsem_basis_tables_host", "dgsem_metrics_host", "dgsem_ssprk3_steps_host",
    "dgsem_graph_create", "dgsem_graph_launch", "dgsem_graph_destroy",
    "dgsem_batch_create", "dgsem_batch_destroy", "dgsem_batch_offsets",
    "dgsem_batch_initial_condition", "dgsem_batch_ssprk3_step", "dgsem_batch_graph_create",
    "dgsem_batch_graph_launch", "dgsem_batch_graph_destroy", "dgsem_batch_check_finite",
    "dgsem_batch_launch_count", "dgsem_autotune", "dgsem_set_launch_variant",
    "dgsem_batch_autotune", "dgsem_batch_set_launch_variant", "dgsem_ssprk3_step_static_scratch",
    "dgsem_static_scratch_state",
    "dgsem_adjoint_create", "dgsem_adjoint_destroy", "dgsem_adjoint_rhs_vjp",
    "dgsem_kinetic_energy", "dgsem_adjoint_gradient", "dgsem_coordinates_host",
    "dgsem_fp64_fma_peak", "dgsem_write_vtu", "dgsem_write_vtu_host",
    "dgsem_checkpoint_write", "dgsem_checkpoint_read", "dgsem_checkpoint_write_host",
    "dgsem_checkpoint_read_host", "dgsem_set_diagnostics", "dgsem_diagnostics",
    "dgsem_geometry_from_coordinates", "dgsem_batch_set_persistent",
]


class MeshDesc(ctypes.Structure):
    _fields_ = [("ndims", ctypes.c_int), ("polydeg", ctypes.c_int),
                ("n_cells", ctypes.c_int64 * 3),
                ("domain_left", ctypes.c_double * 3),
                ("domain_right", ctypes.c_double * 3)]


class SchemeDesc(ctypes.Structure):
    _fields_ = [("equation", ctypes.c_int), ("volume_flux", ctypes.c_int),
                ("surface_flux", ctypes.c_int), ("volume_integral", ctypes.c_int),
                ("bc", ctypes.c_int * 6), ("bc_state", ctypes.c_double * 4),
                ("gamma", ctypes.c_double), ("mu", ctypes.c_double),
                ("prandtl", ctypes.c_double), ("alpha_max", ctypes.c_double),
                ("alpha_min", ctypes.c_double), ("alpha_smooth", ctypes.c_int)]


class DgsemError(RuntimeError):
    def __init__(self, status: int, where: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(status, 'unknown')} (status {status})")
        self.status = status


_lib = None


def lib() -> ctypes.CDLL:
    """Loads libdgsem_b200.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(
            f"{LIB_PATH} is missing; build it with `python -m dgsem_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    vp, dp, c = ctypes.c_void_p, ctypes.c_void_p, ctypes
    L.dgsem_status_string.restype = ctypes.c_char_p
    L.dgsem_status_string.argtypes = [c.c_int]
    L.dgsem_ctx_create.argtypes = [c.POINTER(MeshDesc), c.POINTER(SchemeDesc), vp, c.POINTER(vp)]
    L.dgsem_ctx_destroy.argtypes = [vp]
    L.dgsem_ctx_set_stream.argtypes = [vp, vp]
    L.dgsem_get_sizes.argtypes = [vp, c.POINTER(c.c_int64), c.POINTER(c.c_int),
                                  c.POINTER(c.c_int), c.POINTER(c.c_int64)]
    L.dgsem_set_indicator_parameters.argtypes = [vp, c.c_double, c.c_double, c.c_int]
    L.dgsem_rhs.argtypes = [vp, dp, dp, c.c_double]
    L.dgsem_ssprk3_stage.argtypes = [vp, c.c_int, dp, dp, dp, c.c_double, c.c_double]
    L.dgsem_ssprk3_step.argtypes = [vp, dp, c.c_double, c.c_double]
    L.dgsem_ssprk3_steps.argtypes = [vp, dp, c.c_double, c.c_double, c.c_int]
    L.dgsem_indicator.argtypes = [vp, dp, dp, dp]
    L.dgsem_initial_condition.argtypes = [vp, c.c_int, c.POINTER(c.c_double), dp]
    L.dgsem_to_reference_layout.argtypes = [vp, dp, dp]
    L.dgsem_from_reference_layout.argtypes = [vp, dp, dp]
    L.dgsem_check_finite.argtypes = [vp]
    L.dgsem_launch_count.argtypes = [vp, c.POINTER(c.c_int64)]
    L.dgsem_basis_tables_host.argtypes = [c.c_int, c.POINTER(c.c_double)]
    L.dgsem_metrics_host.argtypes = [c.POINTER(MeshDesc), c.POINTER(c.c_double),
                                     c.POINTER(c.c_double)]
    L.dgsem_coordinates_host.argtypes = [c.POINTER(MeshDesc), c.POINTER(c.c_double)]
    L.dgsem_ssprk3_steps_host.argtypes = [vp, vp, c.c_double, c.c_double, c.c_int]
    L.dgsem_graph_create.argtypes = [vp, dp, c.c_double, c.c_int, c.POINTER(vp)]
    L.dgsem_graph_launch.argtypes = [vp, c.c_double]
    L.dgsem_graph_destroy.argtypes = [vp]
    L.dgsem_batch_create.argtypes = [c.POINTER(MeshDesc), c.c_int, c.POINTER(SchemeDesc), vp,
                                     c.POINTER(vp)]
    L.dgsem_batch_destroy.argtypes = [vp]
    L.dgsem_batch_offsets.argtypes = [vp, c.POINTER(c.c_int64)]
    L.dgsem_batch_initial_condition.argtypes = [vp, c.c_int, c.POINTER(c.c_double), dp]
    L.dgsem_batch_ssprk3_step.argtypes = [vp, dp, c.c_double, c.POINTER(c.c_double)]
    L.dgsem_batch_graph_create.argtypes = [vp, dp, c.POINTER(c.c_double), c.c_int,
                                           c.POINTER(vp)]
    L.dgsem_batch_graph_launch.argtypes = [vp]
    L.dgsem_batch_graph_destroy.argtypes = [vp]
    L.dgsem_batch_check_finite.argtypes = [vp]
    L.dgsem_batch_launch_count.argtypes = [vp, c.POINTER(c.c_int64)]
    L.dgsem_autotune.argtypes = [vp, dp, c.POINTER(c.c_int), c.POINTER(c.c_double)]
    L.dgsem_set_launch_variant.argtypes = [vp, c.c_int]
    L.dgsem_batch_autotune.argtypes = [vp, dp, c.POINTER(c.c_double), c.POINTER(c.c_int)]
    L.dgsem_batch_set_launch_variant.argtypes = [vp, c.c_int]
    L.dgsem_ssprk3_step_static_scratch.argtypes = [vp, dp, c.c_double, c.c_double]
    L.dgsem_static_scratch_state.argtypes = [c.c_int, c.POINTER(c.c_void_p)]
    L.dgsem_adjoint_create.argtypes = [vp, c.c_int, c.c_int, c.POINTER(vp)]
    L.dgsem_adjoint_destroy.argtypes = [vp]
    L.dgsem_adjoint_rhs_vjp.argtypes = [vp, dp, dp, dp]
    L.dgsem_kinetic_energy.argtypes = [vp, dp, c.POINTER(c.c_double), dp]
    L.dgsem_adjoint_gradient.argtypes = [vp, dp, c.c_double, c.c_double,
                                         c.POINTER(c.c_double), dp]
    L.dgsem_fp64_fma_peak.argtypes = [vp, c.c_int, c.POINTER(c.c_double), c.POINTER(c.c_double)]
    L.dgsem_write_vtu.argtypes = [vp, dp, c.c_char_p]
    L.dgsem_write_vtu_host.argtypes = [c.POINTER(MeshDesc), c.c_double, vp, c.c_char_p]
    L.dgsem_checkpoint_write.argtypes = [vp, dp, c.c_double, c.c_int64, c.c_char_p]
    L.dgsem_checkpoint_read.argtypes = [vp, dp, c.POINTER(c.c_double), c.POINTER(c.c_int64),
                                        c.c_char_p]
    L.dgsem_checkpoint_write_host.argtypes = [c.POINTER(MeshDesc), c.POINTER(SchemeDesc), vp,
                                              c.c_double, c.c_int64, c.c_char_p]
    L.dgsem_checkpoint_read_host.argtypes = [c.POINTER(MeshDesc), vp, c.POINTER(c.c_double),
                                             c.POINTER(c.c_int64), c.c_char_p]
    L.dgsem_set_diagnostics.argtypes = [vp, c.c_int]
    L.dgsem_diagnostics.argtypes = [vp, c.POINTER(c.c_double), c.POINTER(c.c_double),
                                    c.POINTER(c.c_double)]
    L.dgsem_geometry_from_coordinates.argtypes = [c.c_int, c.c_int, c.POINTER(c.c_int64), vp, vp,
                                                   vp, vp]
    L.dgsem_batch_set_persistent.argtypes = [vp, c.c_int]
    for name in EXPORTED:
        f = getattr(L, name)
        if name != "dgsem_status_string":
            f.restype = ctypes.c_int
    _lib = L
    return L


def check(status: int, where: str) -> None:
    if status != DGSEM_OK:
        raise DgsemError(status, where)

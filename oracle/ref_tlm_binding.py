"""ctypes binding to oracle/_ref/libdgsem_ref_tlm.so (test infrastructure only).

The library is the reference solver (RetrO598/DGSEM ``src/``) compiled
unmodified with a dual-number scalar type by ``oracle/Makefile``
(``ref_tlm.cpp``): its RHS and SSPRK3 return exact directional derivatives,
i.e. the FP64 tangent-linear model of the reference's own code.  Arrays use
the reference's logical layout ``u(i, j, dof, var)``.

Only tests and the fixture script under tests/golden may use this module.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
TLM_LIB_PATH = os.path.join(_HERE, "_ref", "libdgsem_ref_tlm.so")

EULER2D = 0
NS2D = 5


class _Case(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("polydeg", ctypes.c_int),
                ("n_cells", ctypes.c_int * 2), ("left", ctypes.c_double * 2),
                ("right", ctypes.c_double * 2), ("gamma", ctypes.c_double),
                ("mu", ctypes.c_double), ("prandtl", ctypes.c_double)]


_lib = None


def available() -> bool:
    return os.path.exists(TLM_LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{TLM_LIB_PATH} missing: run `make -C oracle ref`")
        L = ctypes.CDLL(TLM_LIB_PATH)
        vp = ctypes.c_void_p
        L.dgsem_tlm_create.restype = vp
        L.dgsem_tlm_create.argtypes = [ctypes.POINTER(_Case)]
        L.dgsem_tlm_destroy.argtypes = [vp]
        L.dgsem_tlm_state_size.restype = ctypes.c_longlong
        L.dgsem_tlm_state_size.argtypes = [vp]
        L.dgsem_tlm_rhs.argtypes = [vp, vp, vp, ctypes.c_double, vp, vp]
        L.dgsem_tlm_objective.argtypes = [vp, vp, vp, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                          ctypes.POINTER(ctypes.c_double)]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class TangentCase:
    """One 2D periodic case (Chandrashekar split form, LLF surface flux)."""

    def __init__(self, kind: int, polydeg: int, cells, left, right, gamma=1.4, mu=0.0,
                 prandtl=0.72):
        c = _Case(kind, polydeg, (ctypes.c_int * 2)(*cells), (ctypes.c_double * 2)(*left),
                  (ctypes.c_double * 2)(*right), gamma, mu, prandtl)
        self._h = lib().dgsem_tlm_create(ctypes.byref(c))
        if not self._h:
            raise ValueError("unsupported tangent-linear case")
        self.size = int(lib().dgsem_tlm_state_size(self._h))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().dgsem_tlm_destroy(h)
            self._h = None

    def rhs(self, u: np.ndarray, d: np.ndarray | None = None, t: float = 0.0):
        """(R(u), dR/du . d) in the reference layout."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        d = None if d is None else np.ascontiguousarray(d, dtype=np.float64)
        r = np.empty_like(u)
        dr = np.empty_like(u) if d is not None else None
        lib().dgsem_tlm_rhs(self._h, _ptr(u), _ptr(d), float(t), _ptr(r), _ptr(dr))
        return r, dr

    def objective(self, u0: np.ndarray, d0: np.ndarray | None, t0: float, dt: float,
                  nsteps: int):
        """(J, dJ/du0 . d0) with J the mean kinetic energy after nsteps SSPRK3 steps."""
        u0 = np.ascontiguousarray(u0, dtype=np.float64)
        d0 = None if d0 is None else np.ascontiguousarray(d0, dtype=np.float64)
        J, dJ = ctypes.c_double(), ctypes.c_double()
        lib().dgsem_tlm_objective(self._h, _ptr(u0), _ptr(d0), float(t0), float(dt),
                                  int(nsteps), ctypes.byref(J), ctypes.byref(dJ))
        return J.value, (dJ.value if d0 is not None else None)

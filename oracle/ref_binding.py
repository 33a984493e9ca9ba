"""ctypes binding to oracle/_ref/libdgsem_ref.so (test infrastructure only).

The library is the reference's own header-only solver (RetrO598/DGSEM ``src/``)
compiled unmodified against the project's Kokkos-compatible shim by
``oracle/Makefile``.  Arrays use the reference's LayoutRight logical order
``u(i, j[, k], dof, var)`` with ``dof = local_dof(inode, jnode[, knode])``
(``utils/local_dof.hpp:9-19``).

Only tests, ``__graft_entry__.smoke`` and the CPU-baseline leg of ``bench.py``
may use this module; the product never does.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB_PATH = os.path.join(_HERE, "_ref", "libdgsem_ref.so")
# the same reference sources built with floating-point contraction on
# (oracle/Makefile): the reference against itself under a legal change of
# rounding, used as the conditioning floor of the full-size parity tests
REF_FMA_LIB_PATH = os.path.join(_HERE, "_ref", "libdgsem_ref_fma.so")

EULER2D_PERIODIC_SPLIT = 0
EULER2D_PERIODIC_HG = 1
EULER2D_DMR_HG = 2
EULER3D_PERIODIC_SPLIT = 3
EULER3D_PERIODIC_HG = 4
NS2D_PERIODIC_SPLIT = 5
EULER2D_CENTRAL_DIRICHLET = 6  # the reference's CentralFlux + a user DirichletBC (polydeg 3)
EULER2D_CURVED_CENTRAL = 7     # curvilinear periodic mesh, CentralFlux + LLF (polydeg 3)
EULER3D_CURVED = 8             # curvilinear periodic mesh, Chandrashekar + LLF (polydeg <= 4)
NS2D_CHANNEL_WALLS = 9         # Navier-Stokes, x periodic, no-slip bottom / slip top wall
NS3D_PERIODIC_SPLIT = 10       # 3D Navier-Stokes BR1 + Chandrashekar/LLF, periodic (polydeg <= 4)
NS2D_PERIODIC_HG = 11          # 2D Navier-Stokes + HG shock capturing, periodic (viscous KHI)

_DIMS = {0: 2, 1: 2, 2: 2, 3: 3, 4: 3, 5: 2, 6: 2, 7: 2, 8: 3, 9: 2, 10: 3, 11: 2}


class _Case(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int),
        ("polydeg", ctypes.c_int),
        ("n_cells", ctypes.c_int * 3),
        ("left", ctypes.c_double * 3),
        ("right", ctypes.c_double * 3),
        ("gamma", ctypes.c_double),
        ("mu", ctypes.c_double),
        ("prandtl", ctypes.c_double),
        ("alpha_max", ctypes.c_double),
        ("alpha_min", ctypes.c_double),
        ("volume_flux", ctypes.c_int),
        ("surface_flux", ctypes.c_int),
    ]


_lib = None
_libs: dict = {}


def available(build: str = "exact") -> bool:
    return os.path.exists(REF_FMA_LIB_PATH if build == "fma" else REF_LIB_PATH)


def lib(build: str = "exact"):
    """The compiled reference: build "exact" (no contraction, the parity
    reference) or "fma" (contraction on)."""
    global _lib
    if build not in _libs:
        path = REF_FMA_LIB_PATH if build == "fma" else REF_LIB_PATH
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: build it with `make -C oracle ref`")
        L = ctypes.CDLL(path)
        L.dgsem_ref_create.restype = ctypes.c_void_p
        L.dgsem_ref_create.argtypes = [ctypes.POINTER(_Case)]
        L.dgsem_ref_destroy.argtypes = [ctypes.c_void_p]
        L.dgsem_ref_state_size.restype = ctypes.c_longlong
        L.dgsem_ref_state_size.argtypes = [ctypes.c_void_p]
        dp = ctypes.POINTER(ctypes.c_double)
        L.dgsem_ref_rhs.argtypes = [ctypes.c_void_p, dp, dp, ctypes.c_double]
        L.dgsem_ref_alpha.argtypes = [ctypes.c_void_p, dp, dp]
        L.dgsem_ref_ssprk3.argtypes = [ctypes.c_void_p, dp, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_int]
        L.dgsem_ref_geometry.argtypes = [ctypes.c_void_p, dp, dp, dp]
        L.dgsem_ref_basis.argtypes = [ctypes.c_int, dp]
        L.dgsem_ref_omp_threads.restype = ctypes.c_int
        _libs[build] = L
        if build == "exact":
            _lib = L
    return _libs[build]


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def basis_tables(polydeg: int) -> dict:
    n = polydeg + 1
    out = np.zeros(5 * n + 4 * n * n)
    rc = lib().dgsem_ref_basis(polydeg, _ptr(out))
    if rc != 0:
        raise ValueError(f"unsupported polydeg {polydeg}")
    o = 0
    res = {}
    for name in ("nodes", "weights", "inv_weights", "lhat_left", "lhat_right"):
        res[name] = out[o:o + n].copy()
        o += n
    for name in ("D", "Dsplit", "Dhat", "Vinv"):
        res[name] = out[o:o + n * n].reshape(n, n).copy()
        o += n * n
    return res


@dataclass
class RefCase:
    """One reference solver instance (mesh + scheme), kept alive for reuse."""

    kind: int
    polydeg: int
    n_cells: tuple
    left: tuple
    right: tuple
    gamma: float = 1.4
    mu: float = 0.0
    prandtl: float = 0.72
    alpha_max: float = 0.5
    alpha_min: float = 0.001
    volume_flux: int = 0    # 0 Chandrashekar, 1 Ranocha (plugin), 2 Kennedy-Gruber (plugin)
    surface_flux: int = 0   # 0 Lax-Friedrichs, 1 HLLC 2D (plugin)
    build: str = "exact"    # "exact" (no contraction) or "fma" (contraction on)
    _h: int = field(default=0, repr=False)

    def __post_init__(self):
        c = _Case()
        c.kind = self.kind
        c.polydeg = self.polydeg
        nd = _DIMS[self.kind]
        for i in range(3):
            c.n_cells[i] = int(self.n_cells[i]) if i < nd else 1
            c.left[i] = float(self.left[i]) if i < nd else 0.0
            c.right[i] = float(self.right[i]) if i < nd else 1.0
        c.gamma = self.gamma
        c.mu = self.mu
        c.prandtl = self.prandtl
        c.alpha_max = self.alpha_max
        c.alpha_min = self.alpha_min
        c.volume_flux = self.volume_flux
        c.surface_flux = self.surface_flux
        self._c = c
        self._L = lib(self.build)
        self._h = self._L.dgsem_ref_create(ctypes.byref(c))
        if not self._h:
            raise ValueError("reference harness rejected the case")

    def __del__(self):
        if getattr(self, "_h", 0) and getattr(self, "_L", None) is not None:
            self._L.dgsem_ref_destroy(self._h)
            self._h = 0

    @property
    def ndims(self) -> int:
        return _DIMS[self.kind]

    @property
    def nvars(self) -> int:
        return 5 if self.ndims == 3 else 4

    @property
    def n(self) -> int:
        return self.polydeg + 1

    def state_shape(self):
        nd = self.ndims
        return tuple(self.n_cells[:nd]) + (self.n ** nd, self.nvars)

    def rhs(self, u: np.ndarray, t: float = 0.0) -> np.ndarray:
        u = np.ascontiguousarray(u, dtype=np.float64)
        assert u.shape == self.state_shape()
        du = np.zeros_like(u)
        self._L.dgsem_ref_rhs(self._h, _ptr(u), _ptr(du), float(t))
        return du

    def alpha(self, u: np.ndarray) -> np.ndarray:
        u = np.ascontiguousarray(u, dtype=np.float64)
        a = np.zeros(tuple(self.n_cells[:self.ndims]))
        self._L.dgsem_ref_alpha(self._h, _ptr(u), _ptr(a))
        return a

    def ssprk3(self, u: np.ndarray, t0: float, dt: float, nsteps: int) -> np.ndarray:
        u = np.array(u, dtype=np.float64, order="C", copy=True)
        self._L.dgsem_ref_ssprk3(self._h, _ptr(u), float(t0), float(dt), int(nsteps))
        return u

    def geometry(self):
        nd = self.ndims
        cells = tuple(self.n_cells[:nd])
        nn = self.n ** nd
        coords = np.zeros(cells + (nn, nd))
        ja = np.zeros(cells + (nn, nd, nd))
        inv_j = np.zeros(cells + (nn,))
        self._L.dgsem_ref_geometry(self._h, _ptr(coords), _ptr(ja), _ptr(inv_j))
        return coords, ja, inv_j

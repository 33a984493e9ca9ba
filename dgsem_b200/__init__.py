"""dgsem_b200: B200-native (sm_100a) FP64 DGSEM right-hand side and fused
SSPRK3 stage update, with the reference solver's plugin surface.

The compute path is libdgsem_b200.so (hand-written CUDA kernels behind the C
ABI in include/dgsem_b200.h); this package is its host-side mirror.
"""
from ._capi import DgsemError, lib  # noqa: F401
from .solver import (  # noqa: F401
    BoundarySet, ChandrashekarFlux, CompressibleEuler2D, CompressibleEuler3D,
    CompressibleNavierStokes2D, CompressibleNavierStokes3D, DirichletBC,
    DoubleMachReflectionInitial, HGIndicator,
    HLLCFlux, InviscidTaylorGreenVortex, IsentropicVortex, KelvinHelmholtzInitial,
    KennedyGruberFlux, LaxFriedrichsFlux, LobattoLegendreBasis,
    MixedDirichletSlipWallBC, NSNoSlipAdiabaticWallBC, NSSlipAdiabaticWallBC, OutflowBC,
    PeriodicBC, RanochaFlux, SlipWallBC, Solution,
    SSPRK3, StructuredMesh, StructuredSolver, TaylorGreenVortex2D,
    VolumeIntegralShockCapturingHG, VolumeIntegralSplitForm,
)
from .solver import Adjoint, BatchGraph, BatchSolver  # noqa: F401,E402
from .solver import VTUOutputObserver, read_checkpoint, write_checkpoint  # noqa: F401,E402

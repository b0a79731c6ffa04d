"""phipict_b200: phiPICT's PISO/MHD step on NVIDIA B200 (sm_100a).

A drop-in for the parts of ``phipict`` on the PISO step: ``Domain``/``Block``/boundaries,
``Simulation``, ``MHDSimulation``, ``SolverTolerance``, hooks, and the backend protocol
module ``phipict_b200._C``. The compute runs in the in-tree CUDA library
``libphipict_b200.so`` (C ABI: ``include/phipict_b200.h``); there is no CPU fallback.
"""
from . import _C
from .batch import DomainBatch
from .domain import (
    AdvectionScheme,
    Block,
    Boundary,
    BoundaryConditionType,
    BoundaryType,
    ConnectedBoundary,
    CSRmatrix,
    Domain,
    FixedBoundary,
    PeriodicBoundary,
    PotentialBC,
)
from .hooks import Hook, Hooks
from .mhd import MHDSimulation
from .simulation import Simulation
from .solvers import ConvergenceCriterion, LinearSolverResultInfo, LinsolveError
from .tolerance import SolverTolerance

__all__ = [
    "AdvectionScheme", "Block", "Boundary", "BoundaryConditionType", "BoundaryType", "ConnectedBoundary",
    "ConvergenceCriterion", "CSRmatrix", "Domain", "DomainBatch", "FixedBoundary", "Hook", "Hooks", "LinearSolverResultInfo", "LinsolveError",
    "MHDSimulation", "PeriodicBoundary", "PotentialBC", "Simulation", "SolverTolerance", "_C",
]

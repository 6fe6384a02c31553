"""B200-native per-stage update of FVHOE's compressible Euler solver.

`EulerSolver` keeps the constructor, steppers, snapshots and files of
jpalafou/FVHOE's solver (fvhoe/solver.py) and runs every right-hand-side
evaluation and time step in hand-written sm_100a CUDA kernels behind a C ABI
(include/fvh.h, fvhoe_b200/_lib/libfvh.so). PyTorch only provides device
memory and the current stream.
"""

from .array_management import ArrayManager
from .boundary_conditions import BoundaryCondition
from .hydro import HydroState, advection_dt
from .initial_conditions import (
    ArrayIC,
    DoubleMachReflection2D,
    DoubleShock1D,
    FourQuadrant2D,
    InitialCondition,
    KelvinHelmholtz2D,
    KelvinHelmholtzNoise2D,
    SedovBlast,
    ShockTube,
    Shock1D,
    ShuOsher1D,
    Sinus,
    Square,
)
from .solver import EulerSolver
from .timer import Timer

__all__ = [
    "ArrayIC",
    "ArrayManager",
    "BoundaryCondition",
    "DoubleMachReflection2D",
    "DoubleShock1D",
    "Ensemble",
    "EulerSolver",
    "FourQuadrant2D",
    "HydroState",
    "InitialCondition",
    "KelvinHelmholtz2D",
    "KelvinHelmholtzNoise2D",
    "SedovBlast",
    "ShockTube",
    "Shock1D",
    "ShuOsher1D",
    "Sinus",
    "Square",
    "Timer",
    "TroubledCellPredictor",
    "advection_dt",
    "collect_training_data",
]


def __getattr__(name):
    # these modules bind libfvh.so at import; load them on first use
    if name in ("TroubledCellPredictor", "collect_training_data"):
        from . import predictor

        return getattr(predictor, name)
    if name == "Ensemble":
        from .ensemble import Ensemble

        return Ensemble
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")

"""B200-native hybrid-mesh DG residual-and-update path.

A drop-in for the solver hot path of superboss2300/jax-fluid-sim: the classes
keep the reference's names, arguments and ``{element_type: (E, Np, nvars)}``
state layout; the arithmetic runs in hand-written sm_100a CUDA kernels in
``libdgb200.so`` (C ABI in ``include/dgb200.h``), called through ctypes.
"""

from .boundary import FarfieldWallBoundary
from .air11 import AIR11_REACTIONS, AIR11_SPECIES
from .chemistry import Air11ParkMechanism, ReactingFlowCoupler, ReactionMechanism
from .mechanism import Reaction, Species, make_nasa7
from .limiter import (HybridMOODSubcellLimiter, HybridPositivityLimiter, HybridSubcellFV,
                      HybridTroubledCellSensor)
from .mesh import HybridMesh
from .meshgen import MeshSource
from .operators import HybridEulerOperator, HybridNavierStokesOperator, polynomial_br2_penalty
from .solver import CompressibleStateLayout, HybridCompressibleSolver
from .time_integration import HybridSSPRK3

__all__ = [
    "AIR11_REACTIONS", "AIR11_SPECIES", "Air11ParkMechanism", "ReactingFlowCoupler", "Reaction", "ReactionMechanism",
    "Species", "make_nasa7",
    "CompressibleStateLayout", "FarfieldWallBoundary", "HybridCompressibleSolver", "HybridEulerOperator",
    "HybridMOODSubcellLimiter", "HybridMesh", "HybridNavierStokesOperator", "HybridPositivityLimiter",
    "HybridSSPRK3", "HybridSubcellFV", "HybridTroubledCellSensor", "MeshSource", "polynomial_br2_penalty",
]

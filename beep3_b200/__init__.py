"""beep3_b200: B200 (sm_100a) BEM/FMM matvec and GMRES for the linearised
Poisson-Boltzmann boundary integral equations, behind libBEEP's solver API.

Importing the package loads ``libbeep3_b200.so``; there is no CPU fallback.
"""
from . import _native
from ._native import BeepError, BudgetExceeded, NotConverged
from .batch import BatchSolve, ScenarioBatch
from .beep import BEEP, EngineContext, Mesh, MeshInstance, RunInfo
from .geometry import (PatchSet, charges_in_sphere, charges_in_star, icosphere, prepare_patches,
                       quaternion_matrix, random_quaternion, star_shape, star_surface)

_native.lib()

__all__ = [
    "BEEP", "BatchSolve", "ScenarioBatch", "EngineContext", "Mesh", "MeshInstance", "RunInfo", "BeepError", "BudgetExceeded", "NotConverged", "PatchSet",
    "charges_in_sphere", "charges_in_star", "icosphere", "prepare_patches", "quaternion_matrix",
    "random_quaternion", "star_shape", "star_surface",
]

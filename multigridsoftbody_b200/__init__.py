"""B200-native projective-dynamics multigrid soft-body solver.

The compute path is libmgsb.so (hand-written sm_100a CUDA behind a C ABI,
include/mgsb.h); this package is its Python host mirror.
"""
from ._lib import (PRECISION_FP32, PRECISION_MIXED, SOLVER_MULTIGRID, SOLVER_REFERENCE_JACOBI, MgsbError, Params,
                   load)
from .api import (Solver, TetMesh, TwoLevel, blob_mesh, box_mesh, default_params, extract_surface, params_dict,
                  read_msh, value_noise)
from .pdsolver import PDSolver, SphereCollider, SphereFixer

__all__ = [
    "PRECISION_FP32", "PRECISION_MIXED", "SOLVER_MULTIGRID", "SOLVER_REFERENCE_JACOBI", "MgsbError", "Params", "load",
    "Solver", "TetMesh", "TwoLevel", "blob_mesh", "box_mesh", "default_params", "extract_surface", "params_dict", "read_msh",
    "value_noise", "PDSolver", "SphereCollider", "SphereFixer",
]

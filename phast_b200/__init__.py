"""B200 backend for PhAST's matrix-free phase-field hot path.

Host code mirrors PhAST's operator/solver interfaces; every numerical step runs
in the sm_100a library ``phast_b200/_lib/libphastb.so`` (C ABI: include/phastb.h).
"""
from . import _lib
from .damage2d import PhaseFieldDamageSolver
from .fem2d import FEMMesh, FEMOperators, Material, structured_q4_mesh
from .mechanics2d import ExplicitDynamics, QuasiStaticSolver
from .staggered2d import BoundaryConditions, SolverConfig, StaggeredSolver

__all__ = ["FEMMesh", "FEMOperators", "Material", "structured_q4_mesh", "PhaseFieldDamageSolver",
           "ExplicitDynamics", "QuasiStaticSolver", "BoundaryConditions", "SolverConfig", "StaggeredSolver"]


def version():
    return _lib.load().phastb_version().decode()

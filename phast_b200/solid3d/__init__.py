"""Periodic voxel (H8) phase-field cells on the GPU -- the phast.solid3d hot path."""
from .model import LoadCase, PhaseMaterial, SolverConfig, VoxelGrid, isotropic_C, sphere_pore_phase
from .operator import H8DamageSystem, PeriodicVoxelPhaseFieldOperator
from .staggered import (PLAIN, MechForm, solve_constrained_form, BoxKKTResult, H8ScalarBoxKKTConvergenceError, IncrementRecord, PCGBreakdownError, PCGInfo,
                        SolverState, StaggerConvergenceError, StaggeredSolver, solve_constrained,
                        solve_h8_scalar_box_kkt)

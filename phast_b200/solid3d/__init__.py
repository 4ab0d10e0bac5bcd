"""Periodic voxel (H8) phase-field cells on the GPU -- the phast.solid3d hot path.

The public names mirror ``phast.solid3d`` (model, operator, linalg, staggered and
``solvers.box_kkt_h8``) so a caller swaps the import and keeps its code.
"""
from .model import (DRIVER_FULL, DRIVER_NONE, DRIVER_SPECTRAL, PHASE_ID, PHASE_NAMES, VOIGT, ClosurePattern,
                    ElementMaterialArrays,
                    LoadCase, MaterialTable, PhaseMaterial, SolverConfig, VoxelGrid, VoxelModel, build_element_arrays,
                    isotropic_C, lame, resolve_driver, sphere_pore_model, sphere_pore_phase)
from .operator import H8DamageSystem, MechOperator, PeriodicVoxelPhaseFieldOperator, PfczmNewtonSystem
from .staggered import (PLAIN, BoxKKTFailureEvidence, BoxKKTResult, H8ScalarBoxKKTConvergenceError, IncrementRecord,
                        MechForm, PCGBreakdownError, PCGConvergenceError, PCGInfo, ProjectedAnderson, SolverState,
                        StaggerConvergenceError, StaggeredSolver, load_checkpoint, pcg, save_checkpoint,
                        solve_constrained, solve_constrained_form, solve_h8_scalar_box_kkt)

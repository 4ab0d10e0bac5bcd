"""Record the reference's public call signatures on the hot path as a JSON fixture.

Usage (where the reference sources are present)::

    python tests/golden/make_signatures.py <path-to-reference-src>

Imports the reference with the stub modules of ``make_golden.py`` and writes
``reference_signatures.json``: for every mirrored function or method its
parameters (name, kind, default as ``repr`` when the default is a plain
constant) and for every mirrored data class its field names in order.
``tests/test_signatures.py`` checks this package against the file.
"""
from __future__ import annotations

import dataclasses
import importlib
import inspect
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import make_golden as mg  # noqa: E402

# (reference module, qualified name) pairs mirrored by this package; the test maps each
# to the module of this package that implements it
FUNCTIONS = [
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.__init__"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.mech_action"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.mech_diagonal"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.degradation"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.driving_force"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.damage_action"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.damage_rhs"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.damage_diagonal"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.damage_system"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.macro_stress"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.elastic_energy"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.fracture_energy"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.hill_mandel"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.mean_strain"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.split_mech"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.pack_mech"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.mech_fixed_mask"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.mech_fixed_values"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.pfczm_damage_energy"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.pfczm_damage_gradient"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.pfczm_tangent_weights"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.pfczm_tangent_action"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.pfczm_tangent_diagonal"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.pfczm_newton_system"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.closure_pattern"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.closure_pattern_change"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.kinematic_guard"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.expand_damage"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.interface_normal_traction"),
    ("phast.solid3d.operator", "PeriodicVoxelPhaseFieldOperator.interface_opening"),
    ("phast.solid3d.staggered", "save_checkpoint"),
    ("phast.solid3d.staggered", "load_checkpoint"),
    ("phast.solid3d.linalg", "pcg"),
    ("phast.solid3d.linalg", "solve_constrained"),
    ("phast.solvers.box_kkt_h8", "solve_h8_scalar_box_kkt"),
    ("phast.solid3d.materials", "build_element_arrays"),
    ("phast.solid3d.staggered", "StaggeredSolver.__init__"),
    ("phast.solid3d.staggered", "StaggeredSolver.initial_state"),
    ("phast.solid3d.staggered", "StaggeredSolver.initial_record"),
    ("phast.solid3d.staggered", "StaggeredSolver.advance"),
    ("phast.solid3d.staggered", "StaggeredSolver.advance_increment"),
    ("phast.solid3d.staggered", "StaggeredSolver.run"),
    ("phast.solid3d.staggered", "StaggerConvergenceError.__init__"),
    ("phast.solid3d.linalg", "PCGConvergenceError.__init__"),
    ("phast.core.fem_operators", "FEMOperators.compute_strain"),
    ("phast.core.fem_operators", "FEMOperators.internal_force"),
    ("phast.core.fem_operators", "FEMOperators.internal_force_linear"),
    ("phast.core.fem_operators", "FEMOperators.compute_psi_plus"),
    ("phast.core.fem_operators", "FEMOperators.compute_driving_force"),
    ("phast.core.fem_operators", "FEMOperators.laplacian_matvec"),
    ("phast.core.fem_operators", "FEMOperators.stiffness_diagonal"),
    ("phast.core.fem_operators", "FEMOperators.compute_energy_components"),
    ("phast.core.fem_operators", "FEMOperators.compute_reaction_force"),
    ("phast.solvers.damage_solver", "PhaseFieldDamageSolver.solve"),
    ("phast.solvers.damage_solver", "PhaseFieldDamageSolver.compute_residual"),
    ("phast.solvers.mechanics_solver", "ExplicitDynamics.step"),
    ("phast.solvers.mechanics_solver", "QuasiStaticSolver.solve"),
]

DATACLASSES = [
    ("phast.solid3d.model", "VoxelGrid"),
    ("phast.solid3d.model", "PhaseMaterial"),
    ("phast.solid3d.model", "MaterialTable"),
    ("phast.solid3d.model", "VoxelModel"),
    ("phast.solid3d.model", "LoadCase"),
    ("phast.solid3d.model", "SolverConfig"),
    ("phast.solid3d.model", "IncrementRecord"),
    ("phast.solid3d.staggered", "SolverState"),
    ("phast.solid3d.linalg", "PCGInfo"),
    ("phast.solid3d.model", "ClosurePattern"),
    ("phast.physics.material", "Material"),
    ("phast.solvers.staggered_solver", "SolverConfig"),
]

PLAIN = (int, float, str, bool, type(None), tuple)


def _resolve(module, qualname):
    obj = importlib.import_module(module)
    for part in qualname.split("."):
        obj = getattr(obj, part)
    return obj


def _params(fn):
    out = []
    for p in inspect.signature(fn).parameters.values():
        entry = {"name": p.name, "kind": p.kind.name}
        if p.default is not inspect.Parameter.empty:
            entry["default"] = repr(p.default) if isinstance(p.default, PLAIN) else None
        out.append(entry)
    return out


def main(src):
    mg._import_reference(src)
    data = {"functions": {}, "dataclasses": {}}
    for module, name in FUNCTIONS:
        data["functions"][f"{module}:{name}"] = _params(_resolve(module, name))
    for module, name in DATACLASSES:
        cls = _resolve(module, name)
        data["dataclasses"][f"{module}:{name}"] = [f.name for f in dataclasses.fields(cls)]
    path = os.path.join(HERE, "reference_signatures.json")
    with open(path, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    print("wrote", path)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        raise SystemExit(__doc__)
    main(sys.argv[1])

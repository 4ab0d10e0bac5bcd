"""Writes tests/golden/closure.npz from the reference's own crack-closure code
(``crack_closure='axes'``, the isotropic group: closure axes along the cell axes).

Usage: python tests/golden/make_golden_closure.py <path to the reference's src directory>

Cases (CPU, float64, the reference's own classes):
  * operator level on a 5x4x6 pore cell at a seeded state x, damage d: the closure pattern of x,
    the elastic action and Jacobi diagonal with a fixed pattern (that of a second state) and with
    each point's own pattern, the elastic energy and macro stress, the pattern change between the
    two states, and the kinematic guard (solid3d/operator.py:770-877, 1039-1302, 1713-1770);
  * staggered increments of a 6^3 pore cell under uniaxial zz control, AT2 with the closure
    (StaggeredSolver._closure_mechanics / _energy_line_search, solid3d/staggered.py:589-751).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import _import_reference, _voxel_model, n, t  # noqa: E402


def ops_case(out):
    from phast.solid3d.model import LoadCase, SolverConfig
    from phast.solid3d.operator import PeriodicVoxelPhaseFieldOperator

    rng = np.random.default_rng(21)
    shape, h = (5, 4, 6), 1.0 / 6
    model, phase = _voxel_model(shape, h, 0.3)
    load = LoadCase(name="zz", controlled=2, targets=(0.01,), free=(), fixed_zero=(0, 1, 3, 4, 5))
    cfg = SolverConfig(device="cpu", kappa=1e-6, energy_split_isotropic="spectral", crack_closure="axes")
    op = PeriodicVoxelPhaseFieldOperator(model, load, cfg)
    x = rng.normal(size=op.n_mech) * 1e-3
    x2 = rng.normal(size=op.n_mech) * 1e-3
    x[-6:] = [-0.002, 0.001, 0.003, 0.0005, -0.001, 0.0002]
    x2[-6:] = [0.001, -0.002, -0.001, 0.0, 0.0005, -0.0003]
    d = rng.uniform(0, 1, size=op.n_red)
    g = op.degradation(t(d))
    p1 = op.closure_pattern(t(x))
    p2 = op.closure_pattern(t(x2))
    out.update({"shape": np.array(shape), "h": h, "phase": phase, "pinned": op.pinned_node, "x": x, "x2": x2, "d": d,
                "pattern": n(p1.iso), "pattern2": n(p2.iso)})
    out["act_fixed"] = n(op.mech_action(t(x), g, closure=p2))
    out["act_own"] = n(op.mech_action(t(x), g))
    out["diag_fixed"] = n(op.mech_diagonal(g, closure=p2))
    out["diag_all"] = n(op.mech_diagonal(g))
    out["energy"] = np.array([float(op.elastic_energy(t(x), g))])
    out["sigma"] = n(op.macro_stress(t(x), g))
    new, changed = op.closure_pattern_change(t(x), p2, g)
    out["change_pattern"] = n(new.iso)
    out["changed"] = np.array([bool(changed)])
    # a pattern that differs from that of x only where the flip carries no stress (undamaged: g = 1)
    _, same = op.closure_pattern_change(t(x), p1, g)
    out["unchanged"] = np.array([bool(same)])
    guard = op.kinematic_guard(t(x), t(d))
    out["guard"] = np.array([guard["min_normal_strain"], guard["min_principal_strain"], guard["min_det_F"]])


def staggered_case(out):
    from phast.solid3d.model import LoadCase, SolverConfig
    from phast.solid3d.operator import PeriodicVoxelPhaseFieldOperator
    from phast.solid3d.staggered import StaggeredSolver

    shape, h = (6, 6, 6), 1.0 / 6
    model, phase = _voxel_model(shape, h, 0.2)
    targets = (0.01, 0.02, 0.03, 0.04)
    load = LoadCase(name="zz", controlled=2, targets=targets, free=(), fixed_zero=(0, 1, 3, 4, 5))
    cfg = SolverConfig(device="cpu", kappa=1e-6, energy_split_isotropic="spectral", crack_closure="axes")
    op = PeriodicVoxelPhaseFieldOperator(model, load, cfg)
    solver = StaggeredSolver(op)
    state = solver.initial_state()
    keys = ("x", "d", "H", "sigma", "stag", "pcg_mech", "pcg_pf", "closure_solves", "guard", "frac", "elastic")
    rows = {k: [] for k in keys}
    for k in range(len(targets)):
        state, rec = solver.advance(state, targets[k])
        rows["x"].append(n(state.x))
        rows["d"].append(n(state.d))
        rows["H"].append(n(state.H))
        rows["sigma"].append(np.array(rec.macro_stress))
        rows["stag"].append(rec.stagger_iters)
        rows["pcg_mech"].append(rec.pcg_iters_mech)
        rows["pcg_pf"].append(rec.pcg_iters_pf)
        rows["closure_solves"].append(rec.closure_solves)
        rows["guard"].append(np.array([rec.min_normal_strain, rec.min_principal_strain, rec.min_det_F]))
        rows["frac"].append(rec.fracture)
        rows["elastic"].append(rec.elastic)
        print(f"increment {k + 1}: stagger {rec.stagger_iters}, closure solves {rec.closure_solves}, "
              f"pcg {rec.pcg_iters_mech}/{rec.pcg_iters_pf}, max d {float(state.d.max()):.4f}, "
              f"sigma_zz {rec.macro_stress[2]:.4f}")
    out["st_shape"], out["st_phase"], out["st_pinned"] = np.array(shape), phase, op.pinned_node
    out["st_targets"] = np.array(targets)
    for k, v in rows.items():
        out[f"st_{k}"] = np.stack(v) if isinstance(v[0], np.ndarray) else np.array(v)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        raise SystemExit(__doc__)
    _import_reference(sys.argv[1])
    import torch
    torch.set_num_threads(8)
    out = {}
    ops_case(out)
    staggered_case(out)
    np.savez_compressed(os.path.join(HERE, "closure.npz"), **out)
    print("written", os.path.join(HERE, "closure.npz"))

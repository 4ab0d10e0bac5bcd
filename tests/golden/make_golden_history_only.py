"""Writes tests/golden/history_only.npz from the reference's staggered increments with
``irreversibility='history_only'`` (the damage step a Dirichlet PCG without bounds,
solid3d/staggered.py:753-841).

Usage: python tests/golden/make_golden_history_only.py <path to the reference's src directory>
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import _import_reference, _voxel_model, n  # noqa: E402


def staggered_case(out):
    from phast.solid3d.model import LoadCase, SolverConfig
    from phast.solid3d.operator import PeriodicVoxelPhaseFieldOperator
    from phast.solid3d.staggered import StaggeredSolver

    shape, h = (6, 6, 6), 1.0 / 6
    model, phase = _voxel_model(shape, h, 0.2)
    targets = (0.01, 0.02, 0.03)
    load = LoadCase(name="zz", controlled=2, targets=targets, free=(), fixed_zero=(0, 1, 3, 4, 5))
    cfg = SolverConfig(device="cpu", kappa=1e-6, energy_split_isotropic="spectral", irreversibility="history_only")
    op = PeriodicVoxelPhaseFieldOperator(model, load, cfg)
    solver = StaggeredSolver(op)
    state = solver.initial_state()
    rows = {k: [] for k in ("x", "d", "sigma", "stag", "pcg_mech", "pcg_pf", "sets", "kkt", "viol")}
    for k in range(len(targets)):
        state, rec = solver.advance(state, targets[k])
        v = solver.last_bound_violations
        rows["x"].append(n(state.x))
        rows["d"].append(n(state.d))
        rows["sigma"].append(np.array(rec.macro_stress))
        rows["stag"].append(rec.stagger_iters)
        rows["pcg_mech"].append(rec.pcg_iters_mech)
        rows["pcg_pf"].append(rec.pcg_iters_pf)
        rows["sets"].append(rec.active_set_iters)
        rows["kkt"].append(rec.kkt_ok)
        rows["viol"].append(np.array([v["below_previous"], v["below_zero"], v["above_one"], v["max_decrease"],
                                      v["max_excess_over_one"]]))
        print(f"increment {k + 1}: stagger {rec.stagger_iters}, pcg {rec.pcg_iters_mech}/{rec.pcg_iters_pf}, "
              f"kkt_ok {rec.kkt_ok}, violations {v}")
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
    out = {"h": 1.0 / 6}
    staggered_case(out)
    np.savez_compressed(os.path.join(HERE, "history_only.npz"), **out)
    print("written", os.path.join(HERE, "history_only.npz"))

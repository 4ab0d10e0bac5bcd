"""Writes tests/golden/anderson3d.npz from the reference's own projected Anderson mixing of the
3D staggered damage fixed point (``SolverConfig.anderson_depth``).

Usage: python tests/golden/make_golden_anderson3d.py <path to the reference's src directory>

Cases (CPU, float64, the reference's own classes):
  * ProjectedAnderson alone (solid3d/staggered.py:290-376): push/mix on a seeded sequence of pairs
    of a damped affine map, with a lower-bound vector, depth 3;
  * four staggered increments of the 6^3 pore cell (AT2) with anderson_depth = 3
    (StaggeredSolver._attempt, staggered.py:1282-1400).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import _import_reference, _voxel_model, n, t  # noqa: E402


def mixer_case(out):
    from phast.solid3d.staggered import ProjectedAnderson

    rng = np.random.default_rng(41)
    N = 80
    A = rng.normal(size=(N, N)) * 0.07
    b = rng.uniform(0.2, 0.8, size=N)
    lower = np.clip(rng.uniform(-0.2, 0.4, size=N), 0, 1)
    pa = ProjectedAnderson(3)
    d = np.clip(rng.uniform(0, 0.5, size=N), 0, 1)
    ins, outs, mixes, has = [], [], [], []
    for _ in range(8):
        g = np.clip(A @ d + b, -0.5, 1.5)
        pa.push(t(d), t(g))
        m = pa.mix(t(lower))
        ins.append(d.copy())
        outs.append(g.copy())
        has.append(m is not None)
        mixes.append(n(m) if m is not None else np.full(N, np.nan))
        d = n(m) if m is not None else g
    out.update(mix_in=np.stack(ins), mix_out=np.stack(outs), mix_mix=np.stack(mixes), mix_has=np.array(has),
               mix_lower=lower)


def staggered_case(out):
    from phast.solid3d.model import LoadCase, SolverConfig
    from phast.solid3d.operator import PeriodicVoxelPhaseFieldOperator
    from phast.solid3d.staggered import StaggeredSolver

    shape, h = (6, 6, 6), 1.0 / 6
    model, phase = _voxel_model(shape, h, 0.2)
    targets = (0.01, 0.02, 0.03, 0.04)
    load = LoadCase(name="zz", controlled=2, targets=targets, free=(), fixed_zero=(0, 1, 3, 4, 5))
    cfg = SolverConfig(device="cpu", kappa=1e-6, energy_split_isotropic="spectral", anderson_depth=3)
    op = PeriodicVoxelPhaseFieldOperator(model, load, cfg)
    solver = StaggeredSolver(op)
    state = solver.initial_state()
    keys = ("x", "d", "sigma", "stag", "pcg_mech", "pcg_pf", "acc", "rej")
    rows = {k: [] for k in keys}
    for k in range(len(targets)):
        state, rec = solver.advance(state, targets[k])
        rows["x"].append(n(state.x))
        rows["d"].append(n(state.d))
        rows["sigma"].append(np.array(rec.macro_stress))
        rows["stag"].append(rec.stagger_iters)
        rows["pcg_mech"].append(rec.pcg_iters_mech)
        rows["pcg_pf"].append(rec.pcg_iters_pf)
        rows["acc"].append(rec.anderson_accepted)
        rows["rej"].append(rec.anderson_rejected)
        print(f"increment {k + 1}: stagger {rec.stagger_iters}, anderson {rec.anderson_accepted}/"
              f"{rec.anderson_rejected}, pcg {rec.pcg_iters_mech}/{rec.pcg_iters_pf}, max d {float(state.d.max()):.4f}")
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
    mixer_case(out)
    staggered_case(out)
    np.savez_compressed(os.path.join(HERE, "anderson3d.npz"), **out)
    print("written", os.path.join(HERE, "anderson3d.npz"))

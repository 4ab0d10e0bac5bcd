"""Writes tests/golden/pfczm.npz from the reference's own PF-CZM code (Wu's rational
degradation with the projected Newton damage solve of the periodic voxel cell).

Usage: python tests/golden/make_golden_pfczm.py <path to the reference's src directory>

Cases (all on the CPU, float64, with the reference's own classes):
  * operator level on a 5x4x6 cell with a soft spherical pore: the per-element a1, the
    Gauss-point degradation g, the damage energy with and without history, the unscaled
    gradient, the tangent weights, action and Jacobi diagonal, and the scaled Newton system
    (PeriodicVoxelPhaseFieldOperator.pfczm_*, solid3d/operator.py:326-606);
  * one projected Newton damage solve from a given history and lower bound
    (StaggeredSolver._damage_pfczm, solid3d/staggered.py:843-1096);
  * four staggered increments of a 6^3 pore cell under uniaxial zz control, damage_law 'pfczm'
    (StaggeredSolver.advance, solid3d/staggered.py:1215-1517).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import _import_reference, n, t  # noqa: E402

E_MATRIX, NU, GC = 3000.0, 0.35, 0.5
F_MATRIX = 30.0      # MPa: a1 = 4 E Gc / (pi ell f_t^2) = 6.4 at ell = 1/3
PORE_RATIO = 1e-6    # pore stiffness / matrix stiffness
F_PORE = F_MATRIX * PORE_RATIO ** 0.5  # keeps the pore's a1 equal to the matrix's


def pfczm_model(shape, h, pore_radius_frac, softening="linear"):
    from phast.solid3d.model import VoxelGrid, VoxelModel, MaterialTable, PhaseMaterial, PHASE_ID
    nx, ny, nz = shape
    grid = VoxelGrid(shape=shape, h=(h, h, h))
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    c = np.stack([(i + 0.5) / nx - 0.5, (j + 0.5) / ny - 0.5, (k + 0.5) / nz - 0.5], -1)
    phase = np.full((nz, ny, nx), PHASE_ID["mi_matrix"], dtype=np.uint8)
    phase[np.linalg.norm(c, axis=-1) < pore_radius_frac] = PHASE_ID["pore"]
    phases = {
        "mi_matrix": PhaseMaterial(name="mi_matrix", kind="isotropic", Gc=GC, driver="spectral", E=E_MATRIX, nu=NU,
                                   tensile_strength=F_MATRIX),
        "pore": PhaseMaterial(name="pore", kind="isotropic", Gc=GC, driver="spectral", E=E_MATRIX * PORE_RATIO,
                              nu=NU, tensile_strength=F_PORE)}
    table = MaterialTable(phases=phases, length_scale=2 * h, scale="micro")
    tangent = np.zeros((nz, ny, nx, 3))
    tangent[..., 2] = 1.0
    return VoxelModel(grid=grid, phase_id=phase, tangent=tangent, materials=table), phase


def ops_case(out):
    from phast.solid3d.model import LoadCase, SolverConfig
    from phast.solid3d.operator import PeriodicVoxelPhaseFieldOperator
    from phast.solid3d.staggered import StaggeredSolver

    rng = np.random.default_rng(11)
    shape, h = (5, 4, 6), 1.0 / 6
    model, phase = pfczm_model(shape, h, 0.3)
    load = LoadCase(name="zz", controlled=2, targets=(0.01,), free=(), fixed_zero=(0, 1, 3, 4, 5))
    for softening in ("linear", "exponential"):
        p = 2 if softening == "linear" else 2.5
        cfg = SolverConfig(device="cpu", kappa=1e-6, energy_split_isotropic="spectral", damage_law="pfczm",
                           pfczm_softening=softening, pfczm_p=p)
        op = PeriodicVoxelPhaseFieldOperator(model, load, cfg)
        nr, E = op.n_red, op.n_elements
        d = np.clip(rng.uniform(-0.2, 1.1, size=nr), 0, 1)
        H = rng.uniform(0, 0.6, size=(E, 8))
        f = rng.normal(size=nr)
        tag = softening[:3]
        out[f"{tag}_d"], out[f"{tag}_H"], out[f"{tag}_f"] = d, H, f
        out[f"{tag}_a1"] = n(op._a1)
        out[f"{tag}_g"] = n(op.degradation(t(d)))
        out[f"{tag}_energy"] = np.array([float(op.pfczm_damage_energy(t(d), t(H))),
                                         float(op.pfczm_damage_energy(t(d), None))])
        out[f"{tag}_grad"] = n(op.pfczm_damage_gradient(t(d), t(H)))
        W = op.pfczm_tangent_weights(t(d), t(H))
        out[f"{tag}_W"] = n(W)
        out[f"{tag}_Kf"] = n(op.pfczm_tangent_action(t(f), W))
        out[f"{tag}_Kdiag"] = n(op.pfczm_tangent_diagonal(W))
        system, gradient = op.pfczm_newton_system(t(d), t(H))
        out[f"{tag}_rhs"] = n(system.rhs)
        out[f"{tag}_sgrad"] = n(gradient)
        out[f"{tag}_frac"] = np.array([op.fracture_energy(t(d))["total"]])
        if softening == "linear":
            out["shape"], out["h"], out["phase"], out["pinned"] = np.array(shape), h, phase, op.pinned_node
            out["damage_scale"], out["ell"] = op.damage_scale, op.ell
            # one projected Newton damage solve (history large enough to crack the cell)
            solver = StaggeredSolver(op)
            Hs = H * 4.0
            lower = np.clip(d - 0.6, 0, 1)
            ds, pcg, sets, _ = solver._damage_pfczm(t(Hs), t(lower), t(lower))
            out["newton_H"], out["newton_lower"] = Hs, lower
            out["newton_d"] = n(ds)
            out["newton_counts"] = np.array([pcg, sets, solver.last_newton_iters])
            out["newton_energies"] = np.array(solver.last_newton_energies)


def staggered_case(out):
    from phast.solid3d.model import LoadCase, SolverConfig
    from phast.solid3d.operator import PeriodicVoxelPhaseFieldOperator
    from phast.solid3d.staggered import StaggeredSolver

    shape, h = (6, 6, 6), 1.0 / 6
    model, phase = pfczm_model(shape, h, 0.2)
    targets = (0.004, 0.007, 0.009, 0.0105)
    load = LoadCase(name="zz", controlled=2, targets=targets, free=(), fixed_zero=(0, 1, 3, 4, 5))
    cfg = SolverConfig(device="cpu", kappa=1e-6, energy_split_isotropic="spectral", damage_law="pfczm")
    op = PeriodicVoxelPhaseFieldOperator(model, load, cfg)
    solver = StaggeredSolver(op)
    state = solver.initial_state()
    rows = {k: [] for k in ("x", "d", "H", "sigma", "stag", "pcg_mech", "pcg_pf", "sets", "newton", "frac")}
    for k in range(len(targets)):
        state, rec = solver.advance(state, targets[k])
        rows["x"].append(n(state.x))
        rows["d"].append(n(state.d))
        rows["H"].append(n(state.H))
        rows["sigma"].append(np.array(rec.macro_stress))
        rows["stag"].append(rec.stagger_iters)
        rows["pcg_mech"].append(rec.pcg_iters_mech)
        rows["pcg_pf"].append(rec.pcg_iters_pf)
        rows["sets"].append(rec.active_set_iters)
        rows["newton"].append(rec.newton_iters_pf)
        rows["frac"].append(rec.fracture)
        print(f"increment {k + 1}: stagger {rec.stagger_iters}, newton {rec.newton_iters_pf}, "
              f"max d {float(state.d.max()):.4f}, sigma_zz {rec.macro_stress[2]:.4f}")
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
    out = {"E": E_MATRIX, "nu": NU, "Gc": GC, "f_matrix": F_MATRIX, "f_pore": F_PORE, "pore_ratio": PORE_RATIO}
    ops_case(out)
    staggered_case(out)
    np.savez_compressed(os.path.join(HERE, "pfczm.npz"), **out)
    print("written", os.path.join(HERE, "pfczm.npz"))

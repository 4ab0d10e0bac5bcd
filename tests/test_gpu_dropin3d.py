"""The 3D drop-in boundary on the GPU: PhAST's own calling code with this package bound.

``phast.solid3d.api.Problem.run`` builds the operator and the solver with two
lines (solid3d/api.py:203-204)::

    op = PeriodicVoxelPhaseFieldOperator(model, load, cfg, materials=build_element_arrays(model, cfg, device=device))
    solver = StaggeredSolver(op)

and then follows the load path with ``solver.run(max_increments=..., on_increment=...)``
(api.py:221-233).  These tests run exactly those calls against the names of
``phast_b200.solid3d`` and compare the records with the reference's golden
increments; then they check the cutback contract of ``advance_increment``.
"""
import numpy as np
import pytest
import torch

from conftest import golden, rel

pytestmark = pytest.mark.gpu


def _inputs(n=6, **cfg_kw):
    from phast_b200.solid3d import LoadCase, SolverConfig, sphere_pore_model
    model = sphere_pore_model((n, n, n), 0.2, E=3000.0, nu=0.35, Gc=0.5, ell_voxels=2.0, pore_stiffness=1e-6)
    load = LoadCase(name="zz", controlled=2, targets=tuple(0.02 * k / 50 for k in range(1, 51)), free=(),
                    fixed_zero=(0, 1, 3, 4, 5))
    cfg = SolverConfig(device="cuda", kappa=1e-6, energy_split_isotropic="spectral", damage_law="at2",
                       on_stagger_failure="cutback", final_mechanics_resolve=True, **cfg_kw)
    return model, load, cfg


def test_problem_run_lines_unchanged():
    from phast_b200.solid3d import PeriodicVoxelPhaseFieldOperator, StaggeredSolver, build_element_arrays
    g = golden("h8_staggered")
    model, load, cfg = _inputs()
    device = "cuda"
    # solid3d/api.py:203-204, unchanged
    op = PeriodicVoxelPhaseFieldOperator(model, load, cfg, materials=build_element_arrays(model, cfg, device=device))
    solver = StaggeredSolver(op)
    seen = []
    records = solver.run(max_increments=3, on_increment=lambda state, rec: seen.append((state.increment, rec.step)))
    assert seen == [(1, 1), (2, 2), (3, 3)]
    assert [r.increment for r in records] == [1, 2, 3]
    state = solver.last_state
    for k, rec in enumerate(records):
        assert rec.stagger_iters == int(g["stag"][k])
        assert rec.pcg_iters_mech == int(g["pcg_mech"][k]) and rec.pcg_iters_pf == int(g["pcg_pf"][k])
        assert rel(np.array(rec.macro_stress), g["sigma"][k]) < 1e-7
    assert rel(state.x.cpu(), g["x"][2]) < 1e-7 and rel(state.d.cpu(), g["d"][2]) < 1e-7
    assert state.increment == 3 and state.step == 3
    # the record's energies and damage statistics against the same quantities of the state
    rec = records[-1]
    assert rec.elastic == pytest.approx(float(op.elastic_energy(state.x, op.degradation(state.d))), rel=1e-12)
    fr = op.fracture_energy(state.d)
    assert rec.fracture == pytest.approx(fr["total"], rel=1e-12)
    assert set(rec.fracture_by_phase) == {"mi_matrix", "pore"}
    assert rec.max_damage == pytest.approx(float(state.d.max()), rel=0, abs=0)
    assert rec.max_H == pytest.approx(float(state.H.max()), rel=0, abs=0)
    assert rec.macro_strain[2] == pytest.approx(0.02 * 3 / 50, rel=1e-15)
    assert abs(rec.balance_residual_rel) < 0.5


def test_fracture_energy_against_oracle():
    from oracle import h8
    from phast_b200.solid3d import PeriodicVoxelPhaseFieldOperator
    model, load, cfg = _inputs(n=7)
    op = PeriodicVoxelPhaseFieldOperator(model, load, cfg)
    d = np.random.default_rng(3).uniform(0, 1, op.n_red)
    C = [h8.isotropic_C(float(p.E), float(p.nu)) for p in op.phases]
    ref = h8.VoxelOperator(op.shape, op.h, op.slot_np, np.stack([c[0] for c in C]), np.array([c[1] for c in C]),
                           np.array([c[2] for c in C]), np.array([float(p.Gc) for p in op.phases]),
                           np.array([2, 0]), op.ell, op.kappa, op.pinned_node, 2, (0, 1, 3, 4, 5))
    want = ref.fracture_energy(d)
    got = op.fracture_energy(torch.as_tensor(d, device="cuda"))
    assert got["total"] == pytest.approx(want, rel=1e-12)
    assert got["local"] + got["gradient"] == pytest.approx(want, rel=1e-12)
    assert sum(got["by_phase"].values()) == pytest.approx(want, rel=1e-12)


def test_advance_increment_cuts_back_then_reports_the_last_accepted_state():
    """A mechanics PCG capped far below what the increment needs fails every attempt: one
    halving (max_cutbacks = 1), then StaggerConvergenceError carrying the start state."""
    from phast_b200.solid3d import PeriodicVoxelPhaseFieldOperator, StaggerConvergenceError, StaggeredSolver
    model, load, cfg = _inputs(pcg_maxit_mech=3, max_cutbacks=1)
    op = PeriodicVoxelPhaseFieldOperator(model, load, cfg)
    solver = StaggeredSolver(op)
    start = solver.initial_state()
    with pytest.raises(StaggerConvergenceError) as info:
        solver.advance_increment(start, load.targets[0])
    exc = info.value
    assert exc.cutbacks == 1 and exc.attempts == 2 and exc.increment == 1
    assert exc.state is start and exc.records == ()
    assert exc.target == pytest.approx(0.5 * load.targets[0])
    assert "did not converge" in exc.reason
    assert solver.n_attempts == 2 and solver.n_failed_attempts == 2


def test_on_stagger_failure_raise_makes_one_attempt():
    from phast_b200.solid3d import PeriodicVoxelPhaseFieldOperator, SolverConfig, StaggerConvergenceError, StaggeredSolver
    model, load, _ = _inputs()
    cfg = SolverConfig(device="cuda", kappa=1e-6, pcg_maxit_mech=3, on_stagger_failure="raise")
    op = PeriodicVoxelPhaseFieldOperator(model, load, cfg)
    solver = StaggeredSolver(op)
    with pytest.raises(StaggerConvergenceError) as info:
        solver.run(max_increments=2)
    assert info.value.attempts == 1 and info.value.cutbacks == 0 and info.value.records == ()
    assert solver.last_state.increment == 0

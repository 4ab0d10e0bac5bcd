"""Crack closure (``crack_closure='axes'``, isotropic group) on the GPU against fixtures the
reference wrote (``tests/golden/make_golden_closure.py``): the pattern, the elastic action,
diagonal, energy and stress with the (1 - g) add-back, the pattern change, the kinematic guard
and four staggered increments with the line-searched pattern iteration (needs a B200)."""
import numpy as np
import pytest
import torch

from conftest import golden, rel

pytestmark = pytest.mark.gpu


def _op(shape, radius, targets=(0.01,)):
    from phast_b200.solid3d import LoadCase, PeriodicVoxelPhaseFieldOperator, SolverConfig, sphere_pore_model
    model = sphere_pore_model(tuple(int(v) for v in shape), radius)
    load = LoadCase(name="zz", controlled=2, targets=tuple(targets), free=(), fixed_zero=(0, 1, 3, 4, 5))
    cfg = SolverConfig(device="cuda", kappa=1e-6, energy_split_isotropic="spectral", crack_closure="axes")
    return PeriodicVoxelPhaseFieldOperator(model, load, cfg)


def _t(a):
    return torch.as_tensor(np.asarray(a), device="cuda")


def test_closure_operators():
    from phast_b200.solid3d import ClosurePattern
    g = golden("closure")
    op = _op(g["shape"], 0.3)
    assert op.has_closure and op.pinned_node == int(g["pinned"])
    x, x2, d = _t(g["x"]), _t(g["x2"]), _t(g["d"])
    gq = op.degradation(d)
    p1 = op.closure_pattern(x)
    assert np.array_equal(p1.iso.cpu().numpy(), g["pattern"])
    p2 = ClosurePattern(iso=_t(g["pattern2"]))
    assert rel(op.mech_action(x, gq, closure=p2).cpu(), g["act_fixed"]) < 1e-12
    assert rel(op.mech_action(x, gq).cpu(), g["act_own"]) < 1e-12
    assert rel(op.mech_action(x, d=d).cpu(), g["act_own"]) < 1e-12
    assert rel(op.mech_diagonal(gq, closure=p2).cpu(), g["diag_fixed"]) < 1e-12
    assert rel(op.mech_diagonal(gq).cpu(), g["diag_all"]) < 1e-12
    assert abs(float(op.elastic_energy(x, gq)) - float(g["energy"][0])) <= 1e-12 * abs(float(g["energy"][0]))
    assert rel(op.macro_stress(x, gq).cpu(), g["sigma"]) < 1e-12
    new, changed = op.closure_pattern_change(x, p2, gq)
    assert np.array_equal(new.iso.cpu().numpy(), g["change_pattern"]) and changed == bool(g["changed"][0])
    assert op.closure_pattern_change(x, p1, gq)[1] == bool(g["unchanged"][0])
    guard = op.kinematic_guard(x, d)
    assert rel(np.array([guard["min_normal_strain"], guard["min_principal_strain"], guard["min_det_F"]]),
               g["guard"]) < 1e-12
    # the damaged_* minima: none without damage, the overall minima when every element is damaged
    none = op.kinematic_guard(x, torch.zeros_like(d))
    assert none["damaged_min_det_F"] is None and none["damaged_min_normal_strain"] is None
    full = op.kinematic_guard(x, torch.ones_like(d))
    for key in ("min_normal_strain", "min_principal_strain", "min_det_F"):
        assert full["damaged_" + key] == full[key]
    # a pattern is refused without the closure
    from phast_b200.solid3d import LoadCase, PeriodicVoxelPhaseFieldOperator, SolverConfig, sphere_pore_model
    plain = PeriodicVoxelPhaseFieldOperator(sphere_pore_model((5, 4, 6), 0.3),
                                            LoadCase(name="zz", controlled=2, targets=(0.01,), free=(),
                                                     fixed_zero=(0, 1, 3, 4, 5)),
                                            SolverConfig(device="cuda"))
    with pytest.raises(ValueError):
        plain.mech_action(x, gq, closure=p2)


def test_closure_staggered_increments():
    """Four increments of the 6^3 pore cell through PhAST's solver API: stagger passes, closure
    solves and damage PCG counts equal to the reference's, the mechanics PCG total within the
    stopping-point round-off, fields and guard within the solve tolerance."""
    from phast_b200.solid3d import StaggeredSolver
    g = golden("closure")
    op = _op(g["st_shape"], 0.2, targets=tuple(float(v) for v in g["st_targets"]))
    assert op.pinned_node == int(g["st_pinned"])
    solver = StaggeredSolver(op)
    state = solver.initial_state()
    for k, target in enumerate(g["st_targets"]):
        state, rec = solver.advance(state, float(target))
        assert rec.stagger_iters == int(g["st_stag"][k]), k
        assert rec.closure_solves == int(g["st_closure_solves"][k]), k
        assert rec.pcg_iters_pf == int(g["st_pcg_pf"][k]), k
        assert abs(rec.pcg_iters_mech - int(g["st_pcg_mech"][k])) <= 2, k
        assert rel(np.array(rec.macro_stress), g["st_sigma"][k]) < 1e-8
        assert abs(rec.elastic - float(g["st_elastic"][k])) <= 1e-8 * abs(float(g["st_elastic"][k]))
        assert rel(state.d.cpu(), g["st_d"][k]) < 1e-6
        assert rel(state.x.cpu(), g["st_x"][k]) < (1e-8 if k < 3 else 1e-5)
        assert rel(np.array([rec.min_normal_strain, rec.min_principal_strain, rec.min_det_F]), g["st_guard"][k]) < 1e-6
        assert np.array_equal(state.d.cpu().numpy() > 0.5, g["st_d"][k] > 0.5)

"""PF-CZM damage law of the voxel cell on the GPU against fixtures the reference wrote
(``tests/golden/make_golden_pfczm.py``): the operators, one projected Newton damage solve and
four staggered increments, two of them cracking (needs a B200)."""
import numpy as np
import pytest
import torch

from conftest import golden, rel

pytestmark = pytest.mark.gpu


def _op(g, shape_key="shape", softening="linear", radius=0.3, targets=(0.01,)):
    from phast_b200.solid3d import LoadCase, PeriodicVoxelPhaseFieldOperator, SolverConfig, sphere_pore_model
    from phast_b200.solid3d.model import sphere_pore_phase
    shape = tuple(int(v) for v in g[shape_key])
    model = sphere_pore_model(shape, radius, E=float(g["E"]), nu=float(g["nu"]), Gc=float(g["Gc"]),
                              pore_stiffness=float(g["pore_ratio"]), tensile_strength=float(g["f_matrix"]),
                              pore_tensile_strength=float(g["f_pore"]))
    phase_key = "phase" if shape_key == "shape" else "st_phase"
    assert np.array_equal(sphere_pore_phase(shape, radius), g[phase_key])
    load = LoadCase(name="zz", controlled=2, targets=tuple(targets), free=(), fixed_zero=(0, 1, 3, 4, 5))
    cfg = SolverConfig(device="cuda", kappa=1e-6, energy_split_isotropic="spectral", damage_law="pfczm",
                       pfczm_softening=softening, pfczm_p=2 if softening == "linear" else 2.5)
    return PeriodicVoxelPhaseFieldOperator(model, load, cfg), cfg


def _t(a):
    return torch.as_tensor(np.asarray(a), dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("softening", ["linear", "exponential"])
def test_pfczm_operators(softening):
    g = golden("pfczm")
    op, _ = _op(g, softening=softening)
    tag = softening[:3]
    d, H, f = _t(g[f"{tag}_d"]), _t(g[f"{tag}_H"]), _t(g[f"{tag}_f"])
    assert op.is_pfczm and op.pinned_node == int(g["pinned"])
    assert torch.equal(op._a1.cpu(), torch.as_tensor(g[f"{tag}_a1"]))
    assert rel(op.degradation(d).cpu(), g[f"{tag}_g"]) < 1e-13
    e_h, e_0 = (float(v) for v in g[f"{tag}_energy"])
    assert abs(float(op.pfczm_damage_energy(d, H)) - e_h) <= 1e-12 * abs(e_h)
    assert abs(float(op.pfczm_damage_energy(d, None)) - e_0) <= 1e-12 * abs(e_0)
    assert abs(op.fracture_energy(d)["total"] - float(g[f"{tag}_frac"][0])) <= 1e-12 * abs(float(g[f"{tag}_frac"][0]))
    assert rel(op.pfczm_damage_gradient(d, H).cpu(), g[f"{tag}_grad"]) < 1e-12
    W = op.pfczm_tangent_weights(d, H)
    assert rel(W.cpu(), g[f"{tag}_W"]) < 1e-12
    assert rel(op.pfczm_tangent_action(f, W).cpu(), g[f"{tag}_Kf"]) < 1e-12
    assert rel(op.pfczm_tangent_diagonal(W).cpu(), g[f"{tag}_Kdiag"]) < 1e-12
    system, grad = op.pfczm_newton_system(d, H)
    assert rel(system.rhs.cpu(), g[f"{tag}_rhs"]) < 1e-12 and rel(grad.cpu(), g[f"{tag}_sgrad"]) < 1e-12


def test_pfczm_elastic_action_uses_the_law():
    """The elastic action and solve take the PF-CZM g whether given g or d."""
    g = golden("pfczm")
    op, _ = _op(g)
    rng = np.random.default_rng(3)
    d = _t(g["lin_d"])
    x = _t(rng.normal(size=op.n_mech) * 1e-3)
    gq = op.degradation(d)
    assert torch.equal(op.mech_action(x, gq), op.mech_action(x, d=d))
    assert torch.equal(op.mech_diagonal(gq), op.mech_diagonal(d=d))


def test_pfczm_newton_solve():
    """One projected Newton damage solve: iterate and every count against the reference's."""
    from phast_b200.solid3d import StaggeredSolver
    g = golden("pfczm")
    op, _ = _op(g)
    solver = StaggeredSolver(op)
    lower = _t(g["newton_lower"])
    d, pcg, sets, ok = solver._damage(_t(g["newton_H"]), lower, lower)
    assert ok and [pcg, sets, solver.last_newton_iters] == [int(v) for v in g["newton_counts"]]
    assert rel(d.cpu(), g["newton_d"]) < 1e-10
    assert bool((d >= lower).all()) and bool((d <= 1.0).all())
    # the energy sequence ends at the reference's last energy
    e = float(op.pfczm_damage_energy(d, _t(g["newton_H"])))
    assert abs(e - float(g["newton_energies"][-1])) <= 1e-11 * abs(e)


def test_pfczm_staggered_increments():
    """Four increments of the 6^3 pore cell through PhAST's solver API: every decision (stagger,
    Newton, PCG and active-set counts) and the fields against the reference's run."""
    from phast_b200.solid3d import StaggeredSolver
    g = golden("pfczm")
    op, cfg = _op(g, "st_shape", radius=0.2, targets=tuple(float(v) for v in g["st_targets"]))
    assert op.pinned_node == int(g["st_pinned"])
    solver = StaggeredSolver(op)
    state = solver.initial_state()
    for k, target in enumerate(g["st_targets"]):
        state, rec = solver.advance(state, float(target))
        assert rec.stagger_iters == int(g["st_stag"][k]), k
        assert rec.newton_iters_pf == int(g["st_newton"][k]), k
        assert rec.pcg_iters_mech == int(g["st_pcg_mech"][k]) and rec.pcg_iters_pf == int(g["st_pcg_pf"][k]), k
        assert rec.active_set_iters == int(g["st_sets"][k]), k
        assert rel(np.array(rec.macro_stress), g["st_sigma"][k]) < 1e-9
        assert abs(rec.fracture - float(g["st_frac"][k])) <= 1e-8 * max(abs(float(g["st_frac"][k])), 1e-300)
        assert rel(state.x.cpu(), g["st_x"][k]) < 1e-8
        if g["st_d"][k].any():
            assert rel(state.d.cpu(), g["st_d"][k]) < 1e-8
            # same cracked support
            assert np.array_equal(state.d.cpu().numpy() > 0.05, g["st_d"][k] > 0.05)
        else:
            assert not bool(state.d.any())


def test_pfczm_refuses_what_it_does_not_run():
    from phast_b200.solid3d import StaggeredSolver
    from phast_b200.solid3d.staggered import MechForm
    g = golden("pfczm")
    op, _ = _op(g)
    with pytest.raises(NotImplementedError):
        StaggeredSolver(op, form=MechForm(precond="gmg"))
    with pytest.raises(ValueError, match="onset condition"):
        from phast_b200.solid3d import LoadCase, PeriodicVoxelPhaseFieldOperator, SolverConfig, sphere_pore_model
        model = sphere_pore_model((6, 6, 6), 0.2, tensile_strength=200.0, pore_tensile_strength=0.03)
        PeriodicVoxelPhaseFieldOperator(model, LoadCase(name="zz", controlled=2, targets=(0.01,), free=(),
                                                        fixed_zero=(0, 1, 3, 4, 5)),
                                        SolverConfig(device="cuda", damage_law="pfczm"))

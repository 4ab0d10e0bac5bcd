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
    with pytest.raises(ValueError, match="onset condition"):
        from phast_b200.solid3d import LoadCase, PeriodicVoxelPhaseFieldOperator, SolverConfig, sphere_pore_model
        model = sphere_pore_model((6, 6, 6), 0.2, tensile_strength=200.0, pore_tensile_strength=0.03)
        PeriodicVoxelPhaseFieldOperator(model, LoadCase(name="zz", controlled=2, targets=(0.01,), free=(),
                                                        fixed_zero=(0, 1, 3, 4, 5)),
                                        SolverConfig(device="cuda", damage_law="pfczm"))


def _cell16():
    from phast_b200.solid3d import LoadCase, PeriodicVoxelPhaseFieldOperator, SolverConfig, sphere_pore_model
    model = sphere_pore_model((16, 16, 16), 0.2, tensile_strength=30.0, pore_tensile_strength=0.03)
    targets = (0.004, 0.007, 0.009)
    load = LoadCase(name="zz", controlled=2, targets=targets, free=(), fixed_zero=(0, 1, 3, 4, 5))
    cfg = SolverConfig(device="cuda", kappa=1e-6, energy_split_isotropic="spectral", damage_law="pfczm",
                       pcg_rtol_mech=1e-12, damage_linear_tol=1e-12)
    return PeriodicVoxelPhaseFieldOperator(model, load, cfg), cfg, targets


def test_pfczm_multigrid_and_fp32_forms_match_plain():
    """The multigrid and FP32 forms take the PF-CZM g in every operator (fine action, smoother,
    diagonal, coarse moduli): the same FP64 solution as the plain Jacobi solve."""
    from phast_b200.solid3d.staggered import MechForm, _solve_fused, solve_constrained_form
    op, _, _ = _cell16()
    rng = np.random.default_rng(5)
    d = _t(np.clip(rng.uniform(-0.3, 0.9, size=op.n_red), 0, 1))
    mask = op.mech_fixed_mask().to(torch.uint8).contiguous()
    vals = op.mech_fixed_values(0.004)
    x1, info = _solve_fused(op, fixed_mask=mask, fixed_values=vals, g=op.degradation(d), rtol=1e-12, maxiter=20000)
    assert info.converged
    for form in (MechForm(precond="gmg", mixed=True, smooth_degree=1, coarse_degree=6, inner_rtol=1e-5),
                 MechForm(precond="gmg"), MechForm(mixed=True)):
        x, inf = solve_constrained_form(op, form, fixed_mask=mask, fixed_values=vals, d=d, rtol=1e-10, maxiter=20000)
        assert inf.converged and inf.relative_residual <= 1e-10, form
        assert rel(x.cpu(), x1.cpu()) < 1e-7, form
        if form.precond == "gmg":
            assert inf.iterations * 4 < info.iterations, (form, inf.iterations, info.iterations)


def test_pfczm_staggered_chosen_form_matches_plain():
    """Three PF-CZM increments of a 16^3 cell with FP32 + multigrid mechanics under FP64 refinement
    take the plain FP64 solver's decisions with the same fields (tight solver tolerances)."""
    from phast_b200.solid3d import StaggeredSolver
    from phast_b200.solid3d.staggered import PLAIN, MechForm
    op, cfg, targets = _cell16()
    runs = []
    for form in (PLAIN, MechForm(precond="gmg", mixed=True, smooth_degree=1, coarse_degree=6, inner_rtol=1e-5)):
        solver = StaggeredSolver(op, cfg=cfg, form=form)
        state = solver.initial_state()
        recs = []
        for t in targets:
            state, rec = solver.advance(state, t)
            recs.append(rec)
        runs.append((state, recs))
    (s0, r0), (s1, r1) = runs
    assert float(s0.d.max()) > 0.0
    for a, b in zip(r0, r1):
        assert (a.stagger_iters, a.newton_iters_pf) == (b.stagger_iters, b.newton_iters_pf)
        assert rel(np.array(b.macro_stress), np.array(a.macro_stress)) < 1e-7
    assert rel(s1.d.cpu(), s0.d.cpu()) < 1e-6 and rel(s1.x.cpu(), s0.x.cpu()) < 1e-6

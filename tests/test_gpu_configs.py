"""The CUDA path against the reference at the benchmark configurations (needs a B200).

The fixtures were written by the reference's own solvers on the full-size
inputs (``tests/golden/make_golden_configs.py``):

* cfg1: the 64^3 periodic pore cell, increments 1-3 of the eps_zz ramp, at
  PhAST's default tolerances and with the mechanics PCG and damage linear
  tolerances at 1e-12;
* cfg0: the 200 x 200 single-edge-notched tension test, load steps 1-3;
* cfg2: the 400 x 160 explicit crack-branching plate, 200 central-difference
  steps with a damage solve every step.

The plain FP64 form must reproduce the reference's fields to rel-L2 1e-10
where both sides solve to tight tolerances, the same crack support {d > 0.9},
the same staggered iteration counts and the force / macro-stress curve to 1e-6.
The chosen forms (FP32 under FP64 refinement) are held to 1e-6 against the
same FP64 fixtures.
"""
import numpy as np
import pytest
import torch

from conftest import golden, rel

pytestmark = pytest.mark.gpu


def _cell(g, **cfg_kw):
    from phast_b200 import solid3d as s3
    n = int(g["shape"][0])
    model = s3.sphere_pore_model((n, n, n), 0.2, E=3000.0, nu=0.35, Gc=0.5, ell_voxels=2.0, pore_stiffness=1e-6)
    assert np.array_equal(model.phase_id, g["phase"])
    load = s3.LoadCase.ramp("zz", 2, 0.02, 50)
    cfg = s3.SolverConfig(kappa=1e-6, energy_split_isotropic="spectral", damage_law="at2", **cfg_kw)
    op = s3.PeriodicVoxelPhaseFieldOperator(model, load, cfg)
    assert op.pinned_node == int(g["pinned"])
    return op


def _run3(op, form=None):
    from phast_b200 import solid3d as s3
    solver = s3.StaggeredSolver(op, form=form or s3.PLAIN)
    records = solver.run(max_increments=3)
    return solver.last_state, records


def _check_records(records, g, stress_tol):
    for k, rec in enumerate(records):
        assert rec.increment == k + 1 and rec.cutbacks == 0
        assert rec.stagger_iters == int(g["stag"][k])
        assert rel(np.array(rec.macro_stress), g["sigma"][k]) < stress_tol
        assert abs(rec.max_damage - g["dmax"][k]) <= 1e-6 * abs(g["dmax"][k])


def test_cfg1_pore64_tight_tolerances_plain_fp64():
    """Both sides at 1e-12 mechanics/damage tolerances: fields agree to 1e-10."""
    g = golden("cfg1_pore64_tight")
    op = _cell(g, pcg_rtol_mech=1e-12, damage_linear_tol=1e-12)
    state, records = _run3(op)
    _check_records(records, g, 1e-9)
    print("cfg1 tight: PCG mech", [r.pcg_iters_mech for r in records], "ref", list(g["pcg_mech"]),
          "pf", [r.pcg_iters_pf for r in records], "ref", list(g["pcg_pf"]))
    ex, ed = rel(state.x.cpu(), g["x"]), rel(state.d.cpu(), g["d"])
    print(f"cfg1 tight: rel-L2 x {ex:.3e}, d {ed:.3e}")
    assert ex < 1e-10 and ed < 1e-10
    assert np.array_equal(state.d.cpu().numpy() > 0.9, g["d"] > 0.9)


def test_cfg1_pore64_default_tolerances_plain_fp64():
    """PhAST's default tolerances (mechanics PCG rtol 1e-8): iteration counts and fields."""
    g = golden("cfg1_pore64")
    op = _cell(g)
    state, records = _run3(op)
    _check_records(records, g, 1e-7)
    assert [r.pcg_iters_mech for r in records] == [int(v) for v in g["pcg_mech"]]
    assert [r.pcg_iters_pf for r in records] == [int(v) for v in g["pcg_pf"]]
    assert rel(state.x.cpu(), g["x"]) < 1e-7 and rel(state.d.cpu(), g["d"]) < 1e-7
    assert np.array_equal(state.d.cpu().numpy() > 0.9, g["d"] > 0.9)


@pytest.mark.parametrize("form", ["mixed-gmg", "mixed", "gmg"])
def test_cfg1_pore64_chosen_forms_against_fp64_reference(form):
    """FP32 PCG / multigrid forms under FP64 refinement, against the reference's FP64 fields."""
    from phast_b200 import solid3d as s3
    g = golden("cfg1_pore64_tight")
    op = _cell(g)
    mf = {"mixed-gmg": s3.MechForm(precond="gmg", mixed=True), "mixed": s3.MechForm(mixed=True),
          "gmg": s3.MechForm(precond="gmg")}[form]
    state, records = _run3(op, mf)
    for k, rec in enumerate(records):
        assert rel(np.array(rec.macro_stress), g["sigma"][k]) < 1e-6
    ex, ed = rel(state.x.cpu(), g["x"]), rel(state.d.cpu(), g["d"])
    print(f"cfg1 {form}: rel-L2 x {ex:.3e}, d {ed:.3e} against the reference at 1e-12")
    assert ex < 1e-6 and ed < 1e-6
    assert np.array_equal(state.d.cpu().numpy() > 0.9, g["d"] > 0.9)


def _sent(nx, ny, width, height, mat_kw, cfg_kw, crack_y, crack_x, bc):
    import phast_b200 as pb
    sm = pb.structured_q4_mesh(width, height, nx, ny)
    mesh = pb.FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4", device="cuda")
    bcs = pb.BoundaryConditions(mesh.n_nodes, device="cuda")
    if bc:
        bcs.fix(sm.node_sets["bottom"], 0)
        bcs.fix(sm.node_sets["bottom"], 1)
        bcs.add(sm.node_sets["top"], 1, 1.0)
    nodes = sm.nodes.cpu().numpy()
    notch = np.nonzero((np.abs(nodes[:, 1] - crack_y) < 1e-9 * height) & (nodes[:, 0] < crack_x))[0]
    bcs.add_pf_dirichlet(torch.as_tensor(notch), 1.0)
    s = pb.StaggeredSolver(mesh, pb.Material(**mat_kw), bcs, pb.SolverConfig(**cfg_kw))
    s._apply_pf_dirichlet()
    return s, sm, bcs, notch


@pytest.mark.parametrize("tight", [False, True])
def test_cfg0_sent200_plain_fp64(tight):
    """At the configuration's tolerances (mechanics CG and damage projected CG at 1e-10) the
    fields agree to the size of that tolerance; with both sides at 1e-12 they agree to 1e-10."""
    g = golden("cfg0_sent200_tight" if tight else "cfg0_sent200")
    tol = float(g["tol"][0]) if "tol" in g else 1e-10
    field_tol = 1e-10 if tight else 1e-9
    mat = dict(E=210000.0, nu=0.3, Gc=2.7, l0=0.01, eta_residual=1e-8, energy_split="isotropic", rho=7.8e-9)
    cfg = dict(solver_type="quasi_static", backend="cg", static_tol=tol, damage_tol=tol,
               bounds_method="projected_cg", use_multigrid=False, stagger_tol=1e-6, max_stagger=500)
    s, sm, bcs, notch = _sent(200, 200, 1.0, 1.0, mat, cfg, 0.5, 0.5, True)
    assert np.array_equal(notch, g["notch"])
    for k in range(3):
        bcs.load_factor = 0.007 * (k + 1) / 100
        s.step_full()
        assert s._last_stagger_iter == int(g["stag"][k])
        eu, ed = rel(s.u.cpu(), g["u"][k]), rel(s.d.cpu(), g["d"][k])
        rf = s.fem.compute_reaction_force(s.u, s.d, sm.node_sets["top"], component=1)
        print(f"cfg0 (tol {tol:g}) step {k + 1}: rel-L2 u {eu:.3e}, d {ed:.3e}, "
              f"reaction {abs(rf - g['rf'][k]) / abs(g['rf'][k]):.3e}")
        assert eu < field_tol and ed < field_tol
        assert abs(rf - g["rf"][k]) <= 1e-8 * abs(g["rf"][k])
        assert np.array_equal(s.d.cpu().numpy() > 0.9, g["d"][k] > 0.9)
    assert rel(s.H_elem.cpu(), g["H"]) < field_tol


def _branch(dtype):
    mat = dict(E=32000.0, nu=0.2, Gc=3e-3, l0=0.5, rho=2.45e-9, eta_residual=1e-8, energy_split="spectral")
    cfg = dict(solver_type="explicit", dt_safety=0.5, damage_every=1, damage_tol=1e-10,
               bounds_method="projected_cg", use_multigrid=False, dtype=dtype)
    return _sent(400, 160, 100.0, 40.0, mat, cfg, 20.0, 50.0, False)


def test_cfg2_branch400_explicit_plain_fp64():
    g = golden("cfg2_branch400")
    s, sm, bcs, notch = _branch(torch.float64)
    assert np.array_equal(notch, g["notch"])
    assert abs(s.dt - g["dt"][0]) <= 1e-14 * g["dt"][0]
    s.f_ext = torch.as_tensor(g["f_ext"]).cuda()
    for k in range(1, 201):
        s.step_full()
        if k == 100:
            assert rel(s.u.cpu(), g["u100"]) < 1e-10 and rel(s.d.cpu(), g["d100"]) < 1e-10
    errs = {name: rel(getattr(s, name).cpu(), g[name]) for name in ("u", "v", "a", "d")}
    errs["H"] = rel(s.H_elem.cpu(), g["H"])
    print("cfg2 FP64 rel-L2 after 200 steps:", {k: f"{v:.3e}" for k, v in errs.items()})
    assert all(v < 1e-10 for v in errs.values())
    assert np.array_equal(s.d.cpu().numpy() > 0.9, g["d"] > 0.9)


def test_cfg2_branch400_explicit_fp32_rollout_against_fp64_reference():
    """cfg2's prescribed form: FP32 fields and kernels (FP64 damage solve) for 200 steps, against the FP64 fixture."""
    g = golden("cfg2_branch400")
    s, sm, bcs, notch = _branch(torch.float32)
    s.f_ext = torch.as_tensor(g["f_ext"]).cuda().float()
    for _ in range(200):
        s.step_full()
    assert s.u.dtype == torch.float32
    errs = {name: rel(getattr(s, name).double().cpu(), g[name]) for name in ("u", "v", "d")}
    print("cfg2 FP32 rel-L2 after 200 steps:", {k: f"{v:.3e}" for k, v in errs.items()})
    assert errs["u"] < 1e-5 and errs["v"] < 1e-4 and errs["d"] < 1e-5
    assert np.array_equal(s.d.cpu().numpy() > 0.9, g["d"] > 0.9)

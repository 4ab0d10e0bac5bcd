"""Anderson mixing of the 2D staggered damage fixed point on the GPU against fixtures the
reference wrote (``tests/golden/make_golden_anderson.py``): the accelerator alone on a seeded
sequence, and quasi-static SENT load steps with ``anderson_depth = 3`` (needs a B200)."""
import numpy as np
import pytest
import torch

from conftest import golden, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", ["floor", "nofloor"])
def test_anderson_accelerator(tag):
    from phast_b200.staggered2d import AndersonAccelerator
    g = golden("anderson")
    ins, outs, mixes = g[f"acc_{tag}_in"], g[f"acc_{tag}_out"], g[f"acc_{tag}_mix"]
    aa = AndersonAccelerator(ins.shape[1], 3, "cuda")
    floor = torch.as_tensor(g["acc_floor"], device="cuda") if tag == "floor" else None
    for k in range(ins.shape[0]):
        out = aa.step(torch.as_tensor(ins[k], device="cuda"), torch.as_tensor(outs[k], device="cuda"), floor)
        assert rel(out.cpu(), mixes[k]) < 1e-12, k
    assert aa.used > 0


def test_anderson_staggered_sent():
    """Four SENT load steps with depth-3 mixing: stagger counts, fields and reactions."""
    import phast_b200 as pb
    g = golden("anderson")
    nx = int(g["nx"])
    sm = pb.structured_q4_mesh(1.0, 1.0, nx, nx)
    mesh = pb.FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4", device="cuda")
    bcs = pb.BoundaryConditions(mesh.n_nodes, device="cuda")
    mat = pb.Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.1, eta_residual=1e-8, energy_split="isotropic", rho=7.8e-9)
    bcs.fix(sm.node_sets["bottom"], 0)
    bcs.fix(sm.node_sets["bottom"], 1)
    bcs.add(sm.node_sets["top"], 1, 1.0)
    bcs.add_pf_dirichlet(torch.as_tensor(g["notch"]), 1.0)
    cfg = pb.SolverConfig(solver_type="quasi_static", backend="cg", static_tol=1e-10, damage_tol=1e-10,
                          bounds_method="projected_cg", use_multigrid=False, stagger_tol=1e-6, max_stagger=100,
                          anderson_depth=3)
    s = pb.StaggeredSolver(mesh, mat, bcs, cfg)
    s._apply_pf_dirichlet()
    for k, lf in enumerate(g["loads"]):
        bcs.load_factor = float(lf)
        s.step_full()
        assert s._last_stagger_iter == int(g["sent_stag"][k]), k
        assert rel(s.u.cpu(), g["sent_u"][k]) < 1e-7, k
        assert rel(s.d.cpu(), g["sent_d"][k]) < 1e-7, k
        rf = s.fem.compute_reaction_force(s.u, s.d, sm.node_sets["top"], component=1)
        assert abs(rf - g["sent_rf"][k]) <= 1e-6 * abs(g["sent_rf"][k]), k
    assert ((s.d.cpu().numpy() > 0.9) == (g["sent_d"][-1] > 0.9)).all()


def test_projected_anderson_mixer():
    """ProjectedAnderson's push/mix (3D) against the reference on a seeded sequence."""
    from phast_b200.solid3d import ProjectedAnderson
    g = golden("anderson3d")
    pa = ProjectedAnderson(3)
    lower = torch.as_tensor(g["mix_lower"], device="cuda")
    for k in range(g["mix_in"].shape[0]):
        pa.push(torch.as_tensor(g["mix_in"][k], device="cuda"), torch.as_tensor(g["mix_out"][k], device="cuda"))
        m = pa.mix(lower)
        assert (m is not None) == bool(g["mix_has"][k]), k
        if m is not None:
            assert rel(m.cpu(), g["mix_mix"][k]) < 1e-12, k


def test_projected_anderson_staggered_increments():
    """Four increments of the 6^3 pore cell with anderson_depth = 3 through PhAST's solver API:
    stagger passes, accepted and rejected mixes and damage PCG counts equal to the reference's."""
    from phast_b200.solid3d import LoadCase, PeriodicVoxelPhaseFieldOperator, SolverConfig, StaggeredSolver
    from phast_b200.solid3d import sphere_pore_model
    g = golden("anderson3d")
    targets = tuple(float(v) for v in g["st_targets"])
    op = PeriodicVoxelPhaseFieldOperator(
        sphere_pore_model((6, 6, 6), 0.2),
        LoadCase(name="zz", controlled=2, targets=targets, free=(), fixed_zero=(0, 1, 3, 4, 5)),
        SolverConfig(device="cuda", kappa=1e-6, energy_split_isotropic="spectral", anderson_depth=3))
    solver = StaggeredSolver(op)
    state = solver.initial_state()
    for k, target in enumerate(targets):
        state, rec = solver.advance(state, target)
        assert rec.stagger_iters == int(g["st_stag"][k]), k
        assert (rec.anderson_accepted, rec.anderson_rejected) == (int(g["st_acc"][k]), int(g["st_rej"][k])), k
        assert rec.pcg_iters_pf == int(g["st_pcg_pf"][k]), k
        assert abs(rec.pcg_iters_mech - int(g["st_pcg_mech"][k])) <= 2, k
        assert rel(np.array(rec.macro_stress), g["st_sigma"][k]) < 1e-8
        assert rel(state.d.cpu(), g["st_d"][k]) < 1e-6
        assert rel(state.x.cpu(), g["st_x"][k]) < (1e-8 if k < 3 else 1e-5)


def test_history_only_staggered_increments():
    """irreversibility='history_only': the damage step without bounds and its violation statistics,
    three increments of the 6^3 pore cell against the reference."""
    from phast_b200.solid3d import LoadCase, PeriodicVoxelPhaseFieldOperator, SolverConfig, StaggeredSolver
    from phast_b200.solid3d import sphere_pore_model
    g = golden("history_only")
    targets = tuple(float(v) for v in g["st_targets"])
    op = PeriodicVoxelPhaseFieldOperator(
        sphere_pore_model((6, 6, 6), 0.2),
        LoadCase(name="zz", controlled=2, targets=targets, free=(), fixed_zero=(0, 1, 3, 4, 5)),
        SolverConfig(device="cuda", kappa=1e-6, energy_split_isotropic="spectral", irreversibility="history_only"))
    solver = StaggeredSolver(op)
    state = solver.initial_state()
    for k, target in enumerate(targets):
        state, rec = solver.advance(state, target)
        assert rec.stagger_iters == int(g["st_stag"][k]), k
        assert (rec.pcg_iters_pf, rec.active_set_iters) == (int(g["st_pcg_pf"][k]), int(g["st_sets"][k])), k
        assert abs(rec.pcg_iters_mech - int(g["st_pcg_mech"][k])) <= 2, k
        assert rec.kkt_ok == bool(g["st_kkt"][k])
        v = solver.last_bound_violations
        assert [v["below_previous"], v["below_zero"], v["above_one"]] == [int(a) for a in g["st_viol"][k][:3]]
        assert rel(np.array(rec.macro_stress), g["st_sigma"][k]) < 1e-8
        assert rel(state.d.cpu(), g["st_d"][k]) < 1e-7 and rel(state.x.cpu(), g["st_x"][k]) < 1e-7

"""Packed multi-cell batches: every cell of a particle-in-cube batch in one launch per operator
apply and per Krylov vector step, checked against the numpy oracle and against the single-cell
CUDA solves (needs a B200)."""
import numpy as np
import pytest
import torch

from oracle import h8
from phast_b200.solid3d import batch
from phast_b200.solid3d.model import SolverConfig
from phast_b200.solid3d.staggered import PLAIN, StaggeredSolver, _solve_fused, solve_h8_scalar_box_kkt

pytestmark = pytest.mark.gpu

DEV = "cuda"


def _setup(sizes=(8, 12, 16), n=4, seed=5, brick=(8, 8, 4)):
    cells = batch.particle_cells(seed=seed, n_cells=n, sizes=sizes)
    load = batch.batch_load()
    ops = [batch.build_operator(c, load) for c in cells]
    return cells, load, ops, batch.PackedCellBatch(ops, brick=brick)


def _oracle(op):
    C = [h8.isotropic_C(p.E, p.nu) for p in batch.BATCH_PHASES]
    return h8.VoxelOperator(op.shape, op.h, op.slot_np, np.stack([c[0] for c in C]), np.array([c[1] for c in C]),
                            np.array([c[2] for c in C]), np.array([p.Gc for p in batch.BATCH_PHASES]),
                            np.array([2, 2, 2]), op.ell, op.kappa, op.pinned_node, 0, (1, 2, 3, 4, 5))


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


def _t(a):
    return torch.as_tensor(np.asarray(a), device=DEV)


def test_packed_actions_against_oracle():
    cells, load, ops, B = _setup()
    rng = np.random.default_rng(1)
    xs = [rng.normal(size=op.n_mech) * 1e-3 for op in ops]
    ds = [rng.uniform(0, 1, size=op.n_red) for op in ops]
    Hs = [rng.uniform(0, 50, size=(op.n_elements, 8)) for op in ops]
    x, d, H = B.pack_mech([_t(v) for v in xs]), B.pack_nodes([_t(v) for v in ds]), B.pack_elems([_t(v) for v in Hs])
    y, rE = B.mech_apply(x, d)
    y32, _ = B.mech_apply(x.float(), d.float())
    yd = B.damage_apply(d, H)
    for c, op in enumerate(ops):
        ref = _oracle(op)
        g = ref.degradation(ds[c])
        y_ref = ref.mech_action(xs[c], g)
        assert _rel(B.mech_view(y, c).cpu().numpy(), y_ref) < 1e-12
        assert _rel(rE[c], y_ref[-6:]) < 1e-12
        assert _rel(B.mech_view(y32, c).double().cpu().numpy(), y_ref) < 1e-5
        yd_ref = op.damage_scale * ref.damage_action(ds[c], Hs[c])
        assert _rel(B.node_view(yd, c).cpu().numpy(), yd_ref) < 1e-12
        # the single-cell launch computes every node row the same way
        y1 = op.mech_action(B.mech_view(x, c).contiguous(), d=B.node_view(d, c).contiguous())
        assert torch.equal(y1[:-6], B.mech_view(y, c)[:-6])


def test_packed_mech_solve_matches_single_cell():
    cells, load, ops, B = _setup()
    rng = np.random.default_rng(2)
    ds = [np.clip(rng.uniform(-0.5, 0.9, size=op.n_red), 0, 1) for op in ops]
    d = B.pack_nodes([_t(v) for v in ds])
    vals = B.pack_mech([op.mech_fixed_values(0.004) for op in ops])
    x, st, its, conv, bn, rn = B.mech_solve(d, vals, rtol=1e-12)
    assert st == 0 and conv.all()
    xm, st32, its32, conv32, _, rn32 = B.mech_solve(d, vals, rtol=1e-10, mixed=True)
    assert st32 == 0 and conv32.all()
    for c, op in enumerate(ops):
        x1, info = _solve_fused(op, fixed_mask=op.mech_fixed_mask(), fixed_values=B.mech_view(vals, c).contiguous(),
                                d=B.node_view(d, c).contiguous(), rtol=1e-12)
        assert info.converged
        assert _rel(B.mech_view(x, c).cpu().numpy(), x1.cpu().numpy()) < 1e-10
        assert abs(int(its[c]) - info.iterations) <= 2
        assert rn[c] <= 1e-12 * bn[c]
        # FP32 inner solves under FP64 refinement meet the FP64 criterion
        assert rn32[c] <= 1e-10 * bn[c]
        assert _rel(B.mech_view(xm, c).cpu().numpy(), x1.cpu().numpy()) < 1e-7
    # cells left out keep their start iterate
    live = [1, 0] + [1] * (len(ops) - 2)
    x0 = torch.randn(B.n_mech, dtype=torch.float64, device=DEV)
    xl, st, its, conv, _, _ = B.mech_solve(d, vals, x0=x0, rtol=1e-10, live=live)
    assert torch.equal(B.mech_view(xl, 1), B.mech_view(x0, 1)) and its[1] == 0
    assert _rel(B.mech_view(xl, 0).cpu().numpy(), B.mech_view(x, 0).cpu().numpy()) < 1e-8


def test_packed_box_kkt_matches_single_cell():
    cells, load, ops, B = _setup()
    rng = np.random.default_rng(3)
    Hs = [rng.uniform(0, 1, size=(op.n_elements, 8)) * rng.choice([1.0, 400.0], size=(op.n_elements, 1))
          for op in ops]
    lows = [np.clip(rng.uniform(-0.3, 0.4, size=op.n_red), 0, 1) for op in ops]
    H, lower = B.pack_elems([_t(v) for v in Hs]), B.pack_nodes([_t(v) for v in lows])
    dB, st, info, _ = B.damage_box_kkt(H, lower, lower, linear_tolerance=1e-12)
    assert st == 0 and (info[:, 3] == 0).all() and info[:, 2].all()
    for c, op in enumerate(ops):
        res = solve_h8_scalar_box_kkt(op.damage_system(B.elem_view(H, c).contiguous()),
                                      lower_bound=B.node_view(lower, c).contiguous(),
                                      initial=B.node_view(lower, c).contiguous(), linear_tolerance=1e-12)
        assert res.active_set_iterations == int(info[c, 1])
        assert _rel(B.node_view(dB, c).cpu().numpy(), res.solution.cpu().numpy()) < 1e-9
        # the damage is bounded below by the previous field and above by one
        got = B.node_view(dB, c)
        assert bool((got >= B.node_view(lower, c) - 1e-15).all()) and bool((got <= 1.0).all())


@pytest.mark.parametrize("mixed", [False, True])
def test_batch_staggered_against_oracle(mixed):
    """Two load increments of every cell at once against the oracle's staggered increments."""
    cells, load, ops, B = _setup(sizes=(8, 12), n=3)
    solver = batch.BatchStaggeredSolver(B, load, SolverConfig(kappa=ops[0].kappa), mixed=mixed)
    state = solver.initial_state()
    recs = []
    for k in range(2):
        state, r = solver.advance(state, load.targets[k])
        recs.append(r)
    tol = 1e-6 if mixed else 1e-7
    for c, op in enumerate(ops):
        ref = _oracle(op)
        x = np.zeros(ref.n_mech)
        d = np.zeros(ref.n_red)
        H = np.zeros((ref.n_elements, 8))
        prev = 0.0
        for k in range(2):
            x, d, H, stag, _, _, sig = h8.increment(ref, h8.Cfg3D(), x, d, H, prev, load.targets[k])
            prev = load.targets[k]
            got = np.asarray(recs[k][c].macro_stress)
            assert _rel(got, sig) < tol, (c, k)
            assert recs[k][c].stagger_iters == stag
        assert _rel(B.node_view(state.d, c).cpu().numpy(), d) < 10 * tol
        assert _rel(B.mech_view(state.x, c).cpu().numpy(), x) < 10 * tol


def test_batch_staggered_matches_single_cell_solver():
    """The batched increment and the single-cell StaggeredSolver (plain FP64) take the same decisions."""
    cells, load, ops, B = _setup(sizes=(8, 12, 16), n=4)
    cfg = SolverConfig(kappa=ops[0].kappa, pcg_rtol_mech=1e-12, damage_linear_tol=1e-12)
    solver = batch.BatchStaggeredSolver(B, load, cfg, mixed=False)
    state = solver.initial_state()
    for k in range(2):
        state, recs = solver.advance(state, load.targets[k])
    for c, op in enumerate(ops):
        one = StaggeredSolver(op, cfg=cfg, form=PLAIN)
        s1 = one.initial_state()
        for k in range(2):
            s1, r1 = one.advance(s1, load.targets[k])
        assert recs[c].stagger_iters == r1.stagger_iters
        assert recs[c].active_set_iters == r1.active_set_iters
        assert _rel(recs[c].macro_stress, r1.macro_stress) < 1e-9
        assert _rel(B.node_view(state.d, c).cpu().numpy(), s1.d.cpu().numpy()) < 1e-9
        assert _rel(B.mech_view(state.x, c).cpu().numpy(), s1.x.cpu().numpy()) < 1e-9


def _gmg_form():
    from phast_b200.solid3d.staggered import MechForm
    return MechForm(precond="gmg", mixed=True, smooth_degree=1, coarse_degree=6, inner_rtol=1e-5)


def test_packed_multigrid_mech_solve():
    """The batched V-cycle preconditions every cell's FP32 inner solve: the same FP64 solution as
    the batched Jacobi solve, in a fraction of the iterations, and reuse of lambda_max works."""
    cells, load, ops, B = _setup(sizes=(32, 40), n=3, brick=(8, 8, 8))
    rng = np.random.default_rng(9)
    d = B.pack_nodes([_t(np.clip(rng.uniform(-0.5, 0.9, size=op.n_red), 0, 1)) for op in ops])
    vals = B.pack_mech([op.mech_fixed_values(0.004) for op in ops])
    xj, st, itj, conv, bn, rn = B.mech_solve(d, vals, rtol=1e-12)
    assert st == 0 and conv.all()
    for reuse in (False, True):
        xg, st, itg, conv, bng, rng_ = B.mech_solve(d, vals, rtol=1e-10, mixed=True, form=_gmg_form(),
                                                    reuse_lmax=reuse)
        assert st == 0 and conv.all()
        assert (rng_ <= 1e-10 * bng).all()
        for c in range(len(ops)):
            assert _rel(B.mech_view(xg, c).cpu().numpy(), B.mech_view(xj, c).cpu().numpy()) < 1e-7
        assert itg.sum() * 4 < itj.sum(), (itg, itj)


def test_batch_staggered_multigrid_matches_single_cell_solver():
    """At tight solver tolerances (so both sides stop on the same side of the staggered threshold)
    the multigrid batch takes the plain single-cell solver's decisions with the same fields."""
    cells, load, ops, B = _setup(sizes=(32, 40), n=3, brick=(8, 8, 8))
    cfg = SolverConfig(kappa=ops[0].kappa, pcg_rtol_mech=1e-12, damage_linear_tol=1e-12)
    solver = batch.BatchStaggeredSolver(B, load, cfg, mixed=True, form=_gmg_form())
    state = solver.initial_state()
    for k in range(2):
        state, recs = solver.advance(state, load.targets[k])
    for c, op in enumerate(ops):
        one = StaggeredSolver(op, cfg=cfg, form=PLAIN)
        s1 = one.initial_state()
        for k in range(2):
            s1, r1 = one.advance(s1, load.targets[k])
        assert recs[c].stagger_iters == r1.stagger_iters
        assert _rel(recs[c].macro_stress, r1.macro_stress) < 1e-6
        assert _rel(B.node_view(state.d, c).cpu().numpy(), s1.d.cpu().numpy()) < 1e-6

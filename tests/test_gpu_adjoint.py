"""Adjoint gradients of the Q4 AT2 damage solve against central finite differences
(needs a B200).

L = sum_i w_i d_i(H, d_prev, Gc, l0) for the bound-projected solve; the adjoint
(one device PCG on the frozen active set plus the per-element sensitivity
kernel) must agree with central differences of the forward solve at 1e-4
relative, element by element.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

FD_TOL = 1e-4


def setup(seed=0, nx=14, ny=10):
    import phast_b200 as pb
    sm = pb.structured_q4_mesh(1.0, 0.8, nx, ny)
    mesh = pb.FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4", device="cuda")
    mat = pb.Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.08, eta_residual=1e-8, energy_split="isotropic")
    fem = pb.FEMOperators(mesh, mat)
    solver = pb.PhaseFieldDamageSolver(fem, tol=1e-13, max_iter=20000, bounds_method="projected_cg")
    rng = np.random.default_rng(seed)
    E, N = fem.n_elems, fem.n_nodes
    H = torch.as_tensor(rng.uniform(5.0, 60.0, (E, 4)), device="cuda")
    d_prev = torch.as_tensor(rng.uniform(0.0, 0.05, N), device="cuda")
    # a band of nodes held above the unconstrained solution: irreversibility is active there
    d_prev[: nx + 1] = 0.95
    w = torch.as_tensor(rng.normal(size=N), device="cuda")
    gc = torch.as_tensor(2.7 * np.exp(0.2 * rng.normal(size=E)), device="cuda")
    return solver, H, d_prev, w, gc, rng


def loss(solver, H, d_prev, w, **kw):
    with torch.no_grad():
        return float((w * solver.solve(H, d_prev, **kw)).sum())


def rel_close(a, b, tol):
    return abs(a - b) <= tol * max(abs(a), abs(b), 1e-300)


def test_adjoint_gc_field_and_h_match_central_differences():
    solver, H, d_prev, w, gc, rng = setup()
    Hg = H.clone().requires_grad_(True)
    gcg = gc.clone().requires_grad_(True)
    d = solver.solve(Hg, d_prev, Gc_field=gcg)
    (w * d).sum().backward()
    lower = (d.detach() <= d_prev + 1e-12)
    assert int(lower.sum()) > 0  # the active set is exercised
    for e in rng.choice(solver.fem.n_elems, 8, replace=False):
        eps = 1e-4 * float(gc[e])
        gp, gm = gc.clone(), gc.clone()
        gp[e] += eps
        gm[e] -= eps
        fd = (loss(solver, H, d_prev, w, Gc_field=gp) - loss(solver, H, d_prev, w, Gc_field=gm)) / (2 * eps)
        assert rel_close(float(gcg.grad[e]), fd, FD_TOL), (e, float(gcg.grad[e]), fd)
    for e, q in zip(rng.choice(solver.fem.n_elems, 6, replace=False), rng.integers(0, 4, 6)):
        eps = 1e-4 * float(H[e, q])
        hp, hm = H.clone(), H.clone()
        hp[e, q] += eps
        hm[e, q] -= eps
        fd = (loss(solver, hp, d_prev, w, Gc_field=gc) - loss(solver, hm, d_prev, w, Gc_field=gc)) / (2 * eps)
        assert rel_close(float(Hg.grad[e, q]), fd, FD_TOL), (e, q, float(Hg.grad[e, q]), fd)


def test_adjoint_scalar_gc_l0_and_d_prev():
    solver, H, d_prev, w, _, rng = setup(seed=1)
    Gc = torch.tensor(2.7, dtype=torch.float64, device="cuda", requires_grad=True)
    l0 = torch.tensor(0.08, dtype=torch.float64, device="cuda", requires_grad=True)
    dp = d_prev.clone().requires_grad_(True)
    d = solver.solve(H, dp, Gc=Gc, l0=l0)
    (w * d).sum().backward()
    for name, t, base in (("Gc", Gc, 2.7), ("l0", l0, 0.08)):
        eps = 1e-4 * base
        kw_p = {name: base + eps}
        kw_m = {name: base - eps}
        fd = (loss(solver, H, d_prev, w, **kw_p) - loss(solver, H, d_prev, w, **kw_m)) / (2 * eps)
        assert rel_close(float(t.grad), fd, FD_TOL), (name, float(t.grad), fd)
    lower = (d.detach() <= d_prev + 1e-12)
    # the gradient w.r.t. d_prev lives on the nodes held at their lower bound
    assert float(dp.grad[~lower].abs().max()) == 0.0
    for i in torch.nonzero(lower).flatten()[:4].tolist():
        eps = 1e-6
        pp, pm = d_prev.clone(), d_prev.clone()
        pp[i] += eps
        pm[i] -= eps
        fd = (loss(solver, H, pp, w) - loss(solver, H, pm, w)) / (2 * eps)
        assert rel_close(float(dp.grad[i]), fd, FD_TOL), (i, float(dp.grad[i]), fd)


def test_linear_solve_is_the_adjoint_system():
    """A lam = g on the free set: residual check through the operator itself."""
    solver, H, d_prev, w, gc, _ = setup(seed=2)
    fixed = torch.zeros(solver.fem.n_nodes, dtype=torch.bool, device="cuda")
    fixed[::7] = True
    lam = solver.linear_solve(H, w, Gc_field=gc, fixed=fixed, rtol=1e-12)
    assert float(lam[fixed].abs().max()) == 0.0
    solver._Gc_l0_e = (gc * solver._l0).contiguous()
    solver._Gc_over_l0_e = (gc / solver._l0).contiguous()
    try:
        r = solver.compute_residual(H, lam) + solver._prepare(H)[0] - w  # A lam - w
    finally:
        solver._Gc_l0_e = solver._Gc_over_l0_e = None
    r[fixed] = 0.0
    assert float(torch.linalg.vector_norm(r)) <= 1e-10 * float(torch.linalg.vector_norm(w))


def explicit_setup(seed=3, nx=10, ny=8):
    import phast_b200 as pb
    sm = pb.structured_q4_mesh(1.0, 0.8, nx, ny)
    mesh = pb.FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4", device="cuda")
    mat = pb.Material(E=32000.0, nu=0.2, Gc=3e-3, l0=0.1, eta_residual=1e-8, energy_split="isotropic", rho=2.45e-9)
    fem = pb.FEMOperators(mesh, mat)
    dyn = pb.ExplicitDynamics(fem, dt_safety=0.5)
    rng = np.random.default_rng(seed)
    N = fem.n_nodes
    t = lambda x: torch.as_tensor(x, device="cuda")
    u0 = t(rng.normal(size=(N, 2)) * 1e-4)
    v0 = t(rng.normal(size=(N, 2)) * 1e-2)
    a0 = torch.zeros(N, 2, dtype=torch.float64, device="cuda")
    d = t(rng.uniform(0.0, 0.6, N))
    f = t(rng.normal(size=(N, 2)) * 1e-3)
    bc = torch.zeros(N, 2, dtype=torch.bool, device="cuda")
    bc[: nx + 1] = True  # bottom row clamped
    bcv = torch.zeros(N, 2, dtype=torch.float64, device="cuda")
    wu, wv = t(rng.normal(size=(N, 2))), t(rng.normal(size=(N, 2)))
    return dyn, u0, v0, a0, d, f, bc, bcv, wu, wv, rng


def test_explicit_rollout_adjoint_matches_central_differences():
    dyn, u0, v0, a0, d, f, bc, bcv, wu, wv, rng = explicit_setup()
    n = 25

    def objective(u0_, v0_, d_, f_, k=10):
        u, v, _ = dyn.rollout(u0_, v0_, a0, d_, f_, bc, bcv, n, checkpoint_every=k)
        return (wu * u).sum() * 1e4 + (wv * v).sum()

    grads = {}
    for k in (10, 1, 25):
        leaves = [x.clone().requires_grad_(True) for x in (u0, v0, d, f)]
        objective(*leaves, k=k).backward()
        grads[k] = [x.grad.clone() for x in leaves]
    for k in (1, 25):  # the checkpoint interval changes the schedule, not the gradient
        for g10, gk in zip(grads[10], grads[k]):
            assert float((g10 - gk).abs().max()) <= 1e-12 * float(g10.abs().max()) + 1e-300
    gu, gv, gd, gf = grads[10]
    with torch.no_grad():
        def fd(which, idx, eps):
            args_p = [u0.clone(), v0.clone(), d.clone(), f.clone()]
            args_m = [u0.clone(), v0.clone(), d.clone(), f.clone()]
            args_p[which][idx] += eps
            args_m[which][idx] -= eps
            return float(objective(*args_p) - objective(*args_m)) / (2 * eps)
        free = torch.nonzero(~bc[:, 0]).flatten().tolist()
        for node in rng.choice(free, 4, replace=False):
            for c in (0, 1):
                assert rel_close(float(gf[node, c]), fd(3, (node, c), 1e-6), FD_TOL)
                assert rel_close(float(gu[node, c]), fd(0, (node, c), 1e-8), FD_TOL)
                assert rel_close(float(gv[node, c]), fd(1, (node, c), 1e-6), FD_TOL)
        for node in rng.choice(free, 5, replace=False):
            assert rel_close(float(gd[node]), fd(2, (int(node),), 1e-5), FD_TOL), (node, float(gd[node]))

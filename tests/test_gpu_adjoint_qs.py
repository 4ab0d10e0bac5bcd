"""Reverse pass of a quasi-static staggered run: d(peak reaction)/d(Gc field) (needs a B200).

A 24 x 24 single-edge-notched tension test (the cfg4 set-up at a size central
finite differences can afford) with a seeded per-element Gc field and tight
solver tolerances (so the differences are not swamped by solver noise).  The
gradient of the peak reaction force over six load steps is checked against
central differences with a relative step of 1e-4 on elements around the notch
tip and elsewhere, and must not depend on the checkpoint interval.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

NX = 24
STEPS = 6
STATIC_TOL = 1e-9


def _problem(static_tol=STATIC_TOL):
    import phast_b200 as pb
    sm = pb.structured_q4_mesh(1.0, 1.0, NX, NX)
    mesh = pb.FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4", device="cuda")
    bcs = pb.BoundaryConditions(mesh.n_nodes, device="cuda")
    bcs.fix(sm.node_sets["bottom"], 0)
    bcs.fix(sm.node_sets["bottom"], 1)
    bcs.add(sm.node_sets["top"], 1, 1.0)
    nodes = sm.nodes.cpu().numpy()
    notch = np.nonzero((np.abs(nodes[:, 1] - 0.5) < 1e-12) & (nodes[:, 0] < 0.5))[0]
    bcs.add_pf_dirichlet(torch.as_tensor(notch), 1.0)
    mat = pb.Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.05, eta_residual=1e-8, energy_split="isotropic", rho=7.8e-9)
    cfg = pb.SolverConfig(solver_type="quasi_static", backend="cg", static_tol=static_tol, static_max_iter=50,
                          damage_tol=1e-12,
                          bounds_method="projected_cg", use_multigrid=False, stagger_tol=1e-10, max_stagger=500)
    s = pb.StaggeredSolver(mesh, mat, bcs, cfg)
    s._apply_pf_dirichlet()
    return s, sm


def _gradient(checkpoint_every):
    from phast_b200.adjoint2d import PeakReactionGradient
    s, sm = _problem()
    rng = np.random.default_rng(7)
    gc = torch.as_tensor(2.7 * np.exp(0.2 * rng.standard_normal(NX * NX) - 0.02), device="cuda")
    pr = PeakReactionGradient(s, sm.node_sets["top"], lambda k: 0.0012 * k, STEPS, checkpoint_every=checkpoint_every)
    return pr, gc, pr.gradient(gc)


def test_peak_reaction_gradient_against_central_differences():
    pr, gc, res = _gradient(2)
    assert res.peak_step >= 1 and res.objective > 0
    g = res.grad.cpu().numpy()
    # elements around the notch tip (x = 0.5, y = 0.5) and a few others, seeded
    tip = [(j * NX + i) for j in (NX // 2 - 2, NX // 2 - 1, NX // 2, NX // 2 + 1) for i in (NX // 2 - 1, NX // 2, NX // 2 + 1)]
    others = list(np.random.default_rng(3).choice(NX * NX, 5, replace=False))
    scale = float(np.abs(g).max())
    worst = 0.0
    for e in tip + others:
        eps = 1e-4 * float(gc[e])
        vals = []
        for sgn in (1.0, -1.0):
            gp = gc.clone()
            gp[e] += sgn * eps
            vals.append(float(pr.forward(gp).max()))
        fd = (vals[0] - vals[1]) / (2 * eps)
        err = abs(fd - g[e]) / max(abs(fd), 1e-3 * scale)
        worst = max(worst, err)
        assert err < 1e-4, (e, fd, g[e], err)
    print(f"peak reaction {res.objective:.6e} at step {res.peak_step}, passes per step {res.passes}, "
          f"worst relative FD mismatch {worst:.2e}")


def test_gradient_independent_of_checkpoint_interval():
    _, _, a = _gradient(1)
    _, _, b = _gradient(10)
    assert a.peak_step == b.peak_step
    assert float(torch.linalg.vector_norm(a.grad - b.grad) / torch.linalg.vector_norm(b.grad)) < 1e-12


# ---------------------------------------------------------------------------------------------
# T3 twin against PhAST's own autograd gradient (tests/golden/make_golden_adjoint.py)
# ---------------------------------------------------------------------------------------------

def _t3_problem():
    import phast_b200 as pb
    from conftest import golden
    g = golden("t3_qs_adjoint")
    mesh = pb.FEMMesh.from_tensors(torch.as_tensor(g["nodes"]), torch.as_tensor(g["tris"]), element_type="T3",
                                   device="cuda")
    bcs = pb.BoundaryConditions(mesh.n_nodes, device="cuda")
    bot, top = torch.as_tensor(g["bottom"]), torch.as_tensor(g["top"])
    bcs.fix(bot, 0)
    bcs.fix(bot, 1)
    bcs.add(top, 1, 1.0)
    bcs.add_pf_dirichlet(torch.as_tensor(g["notch"]), 1.0)
    mat = pb.Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.125, eta_residual=1e-8, energy_split="isotropic", rho=7.8e-9,
                      gamma_correction=True)
    cfg = pb.SolverConfig(solver_type="quasi_static", backend="cg", static_tol=STATIC_TOL, static_max_iter=50,
                          damage_tol=1e-12, damage_max_iter=5000, bounds_method="projected_cg", use_multigrid=False,
                          stagger_tol=1e-10, max_stagger=400)
    s = pb.StaggeredSolver(mesh, mat, bcs, cfg)
    s._apply_pf_dirichlet()
    return s, g


def _t3_gradient(past_peak=1):
    from phast_b200.adjoint2d import PeakReactionGradient
    s, g = _t3_problem()
    load = float(g["load"][0])
    kstar = int(g["peak_step"][0])
    pr = PeakReactionGradient(s, g["top"], lambda k: load * k, kstar + past_peak, checkpoint_every=2)
    return pr, g, pr.gradient(torch.as_tensor(g["gc"], device="cuda"))


def test_t3_peak_reaction_gradient_against_reference_autograd():
    """The reference's J.backward() through its staggered loop (SuperLU mechanics with the
    stiffness values differentiated, the field adjoint of the damage solve, torch.maximum
    history) against this reverse pass, to 1e-6; the forward reactions and pass counts too."""
    pr, g, res = _t3_gradient()
    kstar = int(g["peak_step"][0])
    assert res.peak_step == kstar
    assert np.allclose(res.reactions[:kstar], g["reactions"][:kstar], rtol=1e-8, atol=0)
    assert res.passes == [int(v) for v in g["stag"][:kstar]]
    # the fixture saw no bound-active node up to the peak: both adjoints are the exact derivative there
    assert int(g["lower_active"][:kstar].sum()) == 0 and int(g["upper_active"][:kstar].sum()) == 0
    err = float(np.linalg.norm(res.grad.cpu().numpy() - g["grad"]) / np.linalg.norm(g["grad"]))
    print(f"T3 twin: peak reaction {res.objective:.9e} (reference {g['reactions'][kstar - 1]:.9e}), "
          f"passes {res.passes}, gradient rel-L2 against the reference autograd {err:.2e}")
    assert err < 1e-6


def test_t3_peak_reaction_gradient_against_central_differences():
    pr, g, res = _t3_gradient(past_peak=0)
    gc = torch.as_tensor(g["gc"], device="cuda")
    grad = res.grad.cpu().numpy()
    scale = float(np.abs(grad).max())
    for e in np.random.default_rng(11).choice(gc.numel(), 6, replace=False):
        eps = 1e-4 * float(gc[e])
        vals = []
        for sgn in (1.0, -1.0):
            gp = gc.clone()
            gp[e] += sgn * eps
            vals.append(float(pr.forward(gp).max()))
        fd = (vals[0] - vals[1]) / (2 * eps)
        assert abs(fd - grad[e]) / max(abs(fd), 1e-3 * scale) < 1e-4, (e, fd, grad[e])

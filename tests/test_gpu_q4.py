"""CUDA Q4 path against the reference's golden vectors and the oracle (needs a B200)."""
import numpy as np
import pytest
import torch

from conftest import golden, rel

pytestmark = pytest.mark.gpu

TOL = 1e-12  # FP64 kernels vs FP64 reference: summation-order differences only


def cuda(x, dtype=torch.float64):
    return torch.as_tensor(np.asarray(x)).to("cuda", dtype)


def ops(g, split="isotropic", ps=False, **kw):
    import phast_b200 as pb
    sm = pb.structured_q4_mesh(float(g["width"]), float(g["height"]), int(g["nx"]), int(g["ny"]))
    mesh = pb.FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4", device="cuda")
    mat = pb.Material(E=kw.get("E", 210000.0), nu=kw.get("nu", 0.3), Gc=kw.get("Gc", 2.7), l0=kw.get("l0", 0.01),
                      eta_residual=1e-8, energy_split=split, plane_stress=ps, rho=kw.get("rho", 2.45e-9))
    return pb.FEMOperators(mesh, mat), sm


@pytest.mark.parametrize("split", ["isotropic", "amor", "spectral", "star_convex", "spectral_stress"])
@pytest.mark.parametrize("ps", [False, True])
def test_q4_force_psi_golden(split, ps):
    if ps and split.startswith("spectral"):
        pytest.skip("plane-strain only")
    g = golden("q4_ops")
    fem, _ = ops(g, split, ps)
    key = f"{split}_{'ps' if ps else 'pe'}"
    u, d = cuda(g["u"]), cuda(g["d"])
    assert rel(fem.internal_force(u, d).cpu(), g["f_" + key]) < TOL
    assert rel(fem.compute_psi_plus(u).cpu(), g["psi_" + key]) < TOL


def test_q4_misc_golden():
    g = golden("q4_ops")
    fem, sm = ops(g)
    u, d, v = cuda(g["u"]), cuda(g["d"]), cuda(g["v"])
    exx, eyy, gxy = fem.compute_strain(u)
    assert rel(exx.cpu(), g["exx"]) < TOL and rel(eyy.cpu(), g["eyy"]) < TOL and rel(gxy.cpu(), g["gxy"]) < TOL
    assert rel(fem.internal_force_linear(u).cpu(), g["f_linear"]) < TOL
    assert rel(fem.stiffness_diagonal(d).cpu(), g["kdiag"]) < TOL
    assert rel(fem.stiffness_diagonal().cpu(), g["kdiag0"]) < TOL
    assert rel(fem.laplacian_matvec(d).cpu(), g["lap"]) < TOL
    assert rel(fem._q4_mass_matvec(d).cpu(), g["mass"]) < TOL
    assert rel(fem.M_scalar.cpu(), g["M_scalar"]) < TOL
    ec = fem.compute_energy_components(u, d, v=v)
    assert rel([ec["elastic"], ec["kinetic"], ec["fracture"], ec["total"]], g["energy"]) < TOL
    r = fem.compute_reaction_force(u, d, sm.node_sets["top"], component=1)
    assert abs(r - g["reaction"][0]) <= 1e-12 * abs(g["reaction"][0])
    assert abs(fem.dt_cfl - g["dt_cfl"][0]) <= 1e-12 * g["dt_cfl"][0]


def test_q4_float32_force_close():
    g = golden("q4_ops")
    fem, _ = ops(g, "spectral")
    u, d = cuda(g["u"], torch.float32), cuda(g["d"], torch.float32)
    assert rel(fem.internal_force(u, d).double().cpu(), g["f_spectral_pe"]) < 1e-5


def test_q4_damage_apply_prepare_solve_golden():
    import phast_b200 as pb
    g = golden("q4_damage")
    fem, _ = ops(g, Gc=float(g["Gc"]), l0=float(g["l0"]))
    ds = pb.PhaseFieldDamageSolver(fem, tol=1e-10, max_iter=2000, use_multigrid=False, bounds_method="projected_cg")
    H = cuda(g["H"])
    rd = 2 * H + float(g["Gc"]) / float(g["l0"])
    assert rel(ds._Ax_q4(cuda(g["x"]), rd).cpu(), g["Ax"]) < TOL
    b, m_inv = ds._prepare(H)
    assert rel(b.cpu(), g["b"]) < TOL and rel(m_inv.cpu(), g["M_inv"]) < TOL
    d = ds.solve(H, cuda(g["d_prev"]))
    assert rel(d.cpu(), g["d_solve"]) < 1e-10
    assert ds.last_iter == int(g["iters_solve"][0])
    d = ds.solve(H, cuda(g["d_prev"]), initial_guess=cuda(g["guess"]))
    assert rel(d.cpu(), g["d_solve_guess"]) < 1e-10
    assert ds.last_iter == int(g["iters_solve_guess"][0])
    m = torch.as_tensor(g["pf_mask"]).cuda()
    d = ds.solve(H, cuda(g["d_prev"]), pf_dirichlet_mask=m, pf_dirichlet_values=m.double())
    assert rel(d.cpu(), g["d_solve_pf"]) < 1e-10
    assert ds.last_iter == int(g["iters_solve_pf"][0])
    assert float(d.min()) >= 0.0 and float(d.max()) <= 1.0


def test_q4_explicit_steps_golden():
    import phast_b200 as pb
    g = golden("q4_dynamics")
    fem, _ = ops(g, "spectral", E=32000.0, nu=0.2, Gc=3e-3, l0=0.5, rho=2.45e-9)
    ex = pb.ExplicitDynamics(fem, dt_safety=0.5)
    assert abs(ex.dt - g["dt"][0]) <= 1e-12 * g["dt"][0]
    u, v, a = cuda(g["u"]), cuda(g["v"]), cuda(g["a"])
    m = torch.as_tensor(g["bc_mask"]).cuda()
    for _ in range(3):
        u, v, a = ex.step(u, v, a, cuda(g["d"]), cuda(g["f_ext"]), m, torch.zeros_like(u))
    assert rel(u.cpu(), g["u3"]) < TOL and rel(v.cpu(), g["v3"]) < TOL and rel(a.cpu(), g["a3"]) < 1e-11


def test_q4_quasi_static_golden():
    import phast_b200 as pb
    g = golden("q4_dynamics")
    fem, _ = ops(g)
    qs = pb.QuasiStaticSolver(fem, tol=1e-10, max_iter=50, backend="cg")
    N = fem.n_nodes
    u, conv, nit = qs.solve(cuda(g["d"]), torch.zeros(N, 2, dtype=torch.float64, device="cuda"),
                            torch.as_tensor(g["qs_bc_mask"]).cuda(), cuda(g["qs_bc_vals"]))
    assert conv == bool(g["qs_conv"][0]) and nit == int(g["qs_nit"][0])
    assert rel(u.cpu(), g["qs_u"]) < 1e-10


def _sent(g, solver_type):
    import phast_b200 as pb
    nx = int(g["nx"])
    sm = pb.structured_q4_mesh(1.0, 1.0, nx, nx)
    mesh = pb.FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4", device="cuda")
    N = mesh.n_nodes
    bcs = pb.BoundaryConditions(N, device="cuda")
    if solver_type == "quasi_static":
        mat = pb.Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.1, eta_residual=1e-8, energy_split="isotropic", rho=7.8e-9)
        bcs.fix(sm.node_sets["bottom"], 0)
        bcs.fix(sm.node_sets["bottom"], 1)
        bcs.add(sm.node_sets["top"], 1, 1.0)
        cfg = pb.SolverConfig(solver_type="quasi_static", backend="cg", static_tol=1e-10, damage_tol=1e-10,
                              bounds_method="projected_cg", use_multigrid=False, stagger_tol=1e-6, max_stagger=100)
    else:
        mat = pb.Material(E=32000.0, nu=0.2, Gc=3e-3, l0=0.15, rho=2.45e-9, eta_residual=1e-8,
                          energy_split="spectral")
        cfg = pb.SolverConfig(solver_type="explicit", dt_safety=0.5, damage_every=1, damage_tol=1e-10,
                              bounds_method="projected_cg", use_multigrid=False)
    bcs.add_pf_dirichlet(torch.as_tensor(g["notch"]), 1.0)
    s = pb.StaggeredSolver(mesh, mat, bcs, cfg)
    s._apply_pf_dirichlet()
    return s, sm, bcs


def test_q4_staggered_quasi_static_golden():
    g = golden("q4_staggered")
    s, sm, bcs = _sent(g, "quasi_static")
    for k in range(3):
        bcs.load_factor = 0.004 * (k + 1)
        s.step_full()
        assert s._last_stagger_iter == int(g["qs_stag"][k])
        assert rel(s.u.cpu(), g["qs_u"][k]) < 1e-9
        assert rel(s.d.cpu(), g["qs_d"][k]) < 1e-9
        assert rel(s.H_elem.cpu(), g["qs_H"][k]) < 1e-9
        rf = s.fem.compute_reaction_force(s.u, s.d, sm.node_sets["top"], component=1)
        assert abs(rf - g["qs_rf"][k]) <= 1e-6 * abs(g["qs_rf"][k])
    crack = (s.d.cpu().numpy() > 0.9) == (g["qs_d"][2] > 0.9)
    assert crack.all()


def test_q4_staggered_explicit_golden():
    g = golden("q4_staggered")
    s, sm, bcs = _sent(g, "explicit")
    assert abs(s.dt - g["ex_dt"][0]) <= 1e-12 * g["ex_dt"][0]
    s.f_ext = torch.as_tensor(g["ex_f_ext"]).cuda()
    for k in range(6):
        s.step_full()
        assert rel(s.u.cpu(), g["ex_u"][k]) < 1e-10
        assert rel(s.d.cpu(), g["ex_d"][k]) < 1e-10
        assert rel(s.H_elem.cpu(), g["ex_H"][k]) < 1e-10
    assert rel(s.v.cpu(), g["ex_v"]) < 1e-10 and rel(s.a.cpu(), g["ex_a"]) < 1e-10


def test_fp32_explicit_rollout_is_reproducible():
    """The FP32 explicit step converts d, f_ext and the BC values to FP32 before its launch; two
    rollouts from the same state must give the same bits (a conversion freed before the kernel
    read it once let the allocator hand its block to the next conversion)."""
    g = golden("q4_staggered")
    runs = []
    for _ in range(2):
        import phast_b200 as pb
        nx = int(g["nx"])
        sm = pb.structured_q4_mesh(1.0, 1.0, nx, nx)
        mesh = pb.FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4", device="cuda")
        bcs = pb.BoundaryConditions(mesh.n_nodes, device="cuda")
        bcs.add_pf_dirichlet(torch.as_tensor(g["notch"]), 1.0)
        mat = pb.Material(E=32000.0, nu=0.2, Gc=3e-3, l0=0.15, rho=2.45e-9, eta_residual=1e-8,
                          energy_split="spectral")
        cfg = pb.SolverConfig(solver_type="explicit", dt_safety=0.5, damage_every=1, damage_tol=1e-10,
                              bounds_method="projected_cg", use_multigrid=False, dtype=torch.float32)
        s = pb.StaggeredSolver(mesh, mat, bcs, cfg)
        s._apply_pf_dirichlet()
        s.f_ext = torch.as_tensor(g["ex_f_ext"]).cuda().float()
        for _ in range(30):
            s.step_full()
        runs.append((s.u.clone(), s.d.clone()))
    assert torch.equal(runs[0][0], runs[1][0]) and torch.equal(runs[0][1], runs[1][1])

"""Split-aware quasi-static mechanics on unstructured T3 meshes (needs a B200): the consistent
tangent kernel against the reference's autograd JVP of internal_force, and quasi-static SENT
load steps on a triangulated mesh with the spectral and the Amor split against the reference's
StaggeredSolver (``tests/golden/make_golden_t3_splits.py``)."""
import numpy as np
import pytest
import torch

from conftest import golden, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("split", ["spectral", "amor", "star_convex"])
def test_t3_tangent_kernel_matches_reference_jvp(split):
    import phast_b200 as pb
    from phast_b200 import _lib
    g = golden("t3_qs_splits")
    mesh = pb.FEMMesh.from_tensors(g["tan_nodes"], g["tan_tris"], element_type="T3", device="cuda")
    mat = pb.Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.05, eta_residual=1e-8, energy_split=split)
    fem = pb.FEMOperators(mesh, mat)
    u, du, d = (torch.as_tensor(g[k]).cuda().contiguous() for k in ("tan_u", "tan_du", "tan_d"))
    y = torch.empty_like(u)
    _lib.call("phastb_t3_tangent_apply", fem.t3, fem._mat, _lib.ptr(u), _lib.ptr(du), _lib.ptr(d), _lib.ptr(y),
              _lib.stream())
    assert rel(y.cpu(), g[f"tan_{split}"]) < 1e-12


@pytest.mark.parametrize("split", ["spectral", "amor"])
def test_t3_quasi_static_split_steps_golden(split):
    import phast_b200 as pb
    g = golden("t3_qs_splits")
    nx = int(g["qs_nx"][0])
    sm = pb.structured_q4_mesh(1.0, 1.0, nx, nx)
    mesh = pb.FEMMesh.from_tensors(sm.nodes, g["qs_tris"], element_type="T3", device="cuda")
    bcs = pb.BoundaryConditions(mesh.n_nodes, device="cuda")
    mat = pb.Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.1, eta_residual=1e-8, energy_split=split, rho=7.8e-9)
    bcs.fix(sm.node_sets["bottom"], 0)
    bcs.fix(sm.node_sets["bottom"], 1)
    bcs.add(sm.node_sets["top"], 1, 1.0)
    bcs.add_pf_dirichlet(torch.as_tensor(g["qs_notch"]), 1.0)
    cfg = pb.SolverConfig(solver_type="quasi_static", backend="cg", static_tol=1e-10, damage_tol=1e-10,
                          bounds_method="projected_cg", use_multigrid=False, stagger_tol=1e-6, max_stagger=100)
    s = pb.StaggeredSolver(mesh, mat, bcs, cfg)
    s._apply_pf_dirichlet()
    for k in range(3):
        bcs.load_factor = 0.004 * (k + 1)
        s.step_full()
        assert s._last_stagger_iter == int(g[f"qs_{split}_stag"][k]), k
        assert rel(s.u.cpu(), g[f"qs_{split}_u"][k]) < 1e-8, k
        assert rel(s.d.cpu(), g[f"qs_{split}_d"][k]) < 1e-8, k
        rf = s.fem.compute_reaction_force(s.u, s.d, sm.node_sets["top"], component=1)
        assert abs(rf - g[f"qs_{split}_rf"][k]) <= 1e-6 * abs(g[f"qs_{split}_rf"][k]), k
    assert ((s.d.cpu().numpy() > 0.9) == (g[f"qs_{split}_d"][2] > 0.9)).all()

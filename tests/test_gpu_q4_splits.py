"""Split-aware quasi-static mechanics on structured Q4 (needs a B200): the consistent-tangent
kernel against the reference's autograd JVP of internal_force, and quasi-static SENT load steps
with the spectral and the Amor split against the reference's StaggeredSolver."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import golden, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("key,split,ps", [("tan_spectral", "spectral", False), ("tan_amor", "amor", False),
                                          ("tan_star_convex", "star_convex", False), ("tan_amor_ps", "amor", True)])
def test_q4_tangent_kernel_matches_reference_jvp(key, split, ps):
    import phast_b200 as pb
    from phast_b200 import _lib
    g = golden("q4_qs_splits")
    sm = pb.structured_q4_mesh(float(g["tan_w"][0]), float(g["tan_h"][0]), int(g["tan_nx"][0]), int(g["tan_ny"][0]))
    mesh = pb.FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4", device="cuda")
    mat = pb.Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.05, eta_residual=1e-8, energy_split=split, plane_stress=ps)
    fem = pb.FEMOperators(mesh, mat)
    u, du, d = (torch.as_tensor(g[k]).cuda().contiguous() for k in ("tan_u", "tan_du", "tan_d"))
    y = torch.empty_like(u)
    _lib.call("phastb_q4_tangent_apply", C.byref(fem.grid), fem.mat(torch.float64), _lib.ptr(u), _lib.ptr(du),
              _lib.ptr(d), _lib.ptr(y), _lib.stream())
    assert rel(y.cpu(), g[key]) < 1e-12
    # the force at u is the split's (the tangent differentiates the same stress)
    assert rel(fem.internal_force(u, d).cpu(), g[key + "_f"]) < 1e-12


@pytest.mark.parametrize("split", ["spectral", "amor"])
def test_q4_quasi_static_split_steps_golden(split):
    import phast_b200 as pb
    g = golden("q4_qs_splits")
    nx = int(g["qs_nx"][0])
    sm = pb.structured_q4_mesh(1.0, 1.0, nx, nx)
    mesh = pb.FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4", device="cuda")
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
        assert s._last_stagger_iter == int(g[f"qs_{split}_stag"][k])
        assert rel(s.u.cpu(), g[f"qs_{split}_u"][k]) < 1e-8
        assert rel(s.d.cpu(), g[f"qs_{split}_d"][k]) < 1e-8
        assert rel(s.H_elem.cpu(), g[f"qs_{split}_H"][k]) < 1e-8
        rf = s.fem.compute_reaction_force(s.u, s.d, sm.node_sets["top"], component=1)
        assert abs(rf - g[f"qs_{split}_rf"][k]) <= 1e-6 * abs(g[f"qs_{split}_rf"][k])
    assert ((s.d.cpu().numpy() > 0.9) == (g[f"qs_{split}_d"][2] > 0.9)).all()

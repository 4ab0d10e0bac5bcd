"""Unstructured T3 operators with the coloured scatter against the reference's
golden vectors (needs a B200)."""
import numpy as np
import pytest
import torch

from conftest import golden, rel

pytestmark = pytest.mark.gpu

TOL = 1e-12


def ops(g, split="isotropic", ps=False):
    import phast_b200 as pb
    mesh = pb.FEMMesh.from_tensors(g["nodes"], g["tris"], element_type="T3", device="cuda")
    mat = pb.Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.05, eta_residual=1e-8, energy_split=split, plane_stress=ps,
                      rho=2.45e-9)
    return pb.FEMOperators(mesh, mat)


def cuda(x):
    return torch.as_tensor(np.asarray(x), device="cuda", dtype=torch.float64)


@pytest.mark.parametrize("split", ["isotropic", "amor", "spectral", "star_convex", "spectral_stress"])
@pytest.mark.parametrize("ps", [False, True])
def test_t3_force_psi_golden(split, ps):
    if ps and split.startswith("spectral"):
        pytest.skip("plane-strain only")
    g = golden("t3_ops")
    fem = ops(g, split, ps)
    assert fem.n_colors >= 3
    key = f"{split}_{'ps' if ps else 'pe'}"
    assert rel(fem.internal_force(cuda(g["u"]), cuda(g["d"])).cpu(), g["f_" + key]) < TOL
    assert rel(fem.compute_psi_plus(cuda(g["u"])).cpu(), g["psi_" + key]) < TOL


def test_t3_geometry_damage_and_solve_golden():
    import phast_b200 as pb
    g = golden("t3_ops")
    fem = ops(g)
    assert rel(fem.grad_phi.cpu(), g["grad_phi"]) < TOL and rel(fem.M_scalar.cpu(), g["M_scalar"]) < TOL
    assert rel(fem.internal_force_linear(cuda(g["u"])).cpu(), g["f_linear"]) < TOL
    ds = pb.PhaseFieldDamageSolver(fem, tol=1e-10, max_iter=3000, bounds_method="projected_cg")
    H = cuda(g["H"])
    b, m_inv = ds.prepare(H)
    assert rel(b.cpu(), g["b"]) < TOL and rel(m_inv.cpu(), g["M_inv"]) < TOL
    assert rel(ds._Ax(cuda(g["x"]), H).cpu(), g["Ax"]) < TOL
    d = ds.solve(H, cuda(g["d_prev"]))
    assert rel(d.cpu(), g["d_solve"]) < 1e-10
    assert abs(ds.last_iter - int(g["iters_solve"][0])) <= 1
    H2 = ds.fem.psi_history(cuda(g["u"]), H)
    assert torch.equal(H2, torch.maximum(H, fem.compute_psi_plus(cuda(g["u"]))))

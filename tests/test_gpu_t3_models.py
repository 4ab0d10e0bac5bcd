"""T3 damage models beyond element-history AT2 (needs a B200): AT1 with element history and AT2
with nodal history, through PhaseFieldDamageSolver on the coloured T3 kernels, against the
reference's golden vectors (prepared system, one action, the bound-projected solve)."""
import numpy as np
import pytest
import torch

from conftest import golden, rel

pytestmark = pytest.mark.gpu


def _solver(g, model, nodal):
    import phast_b200 as pb
    mesh = pb.FEMMesh.from_tensors(g["nodes"], g["tris"], element_type="T3", device="cuda")
    mat = pb.Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.05, eta_residual=1e-8, energy_split="isotropic",
                      rho=2.45e-9, pf_model=model)
    fem = pb.FEMOperators(mesh, mat)
    return pb.PhaseFieldDamageSolver(fem, tol=1e-10, max_iter=3000, use_multigrid=False,
                                     bounds_method="projected_cg", nodal_H=nodal)


def cuda(x):
    return torch.as_tensor(np.asarray(x), device="cuda", dtype=torch.float64)


@pytest.mark.parametrize("key,model,nodal", [("at1", "AT1", False), ("nodal", "AT2", True)])
def test_t3_damage_model_golden(key, model, nodal):
    g = golden("t3_models")
    ds = _solver(g, model, nodal)
    H = cuda(g[f"{key}_H"])
    b, mi = ds.prepare(H)
    assert rel(b.cpu(), g[f"{key}_b"]) < 1e-12
    assert rel(mi.cpu(), g[f"{key}_M_inv"]) < 1e-12
    assert rel(ds._Ax(cuda(g["x"]), H).cpu(), g[f"{key}_Ax"]) < 1e-12
    d = ds.solve(H, cuda(g["d_prev"]))
    assert rel(d.cpu(), g[f"{key}_d_solve"]) < 1e-10
    assert ds.last_iter == int(g[f"{key}_iters"][0])
    assert bool((d >= cuda(g["d_prev"]) - 1e-14).all()) and bool((d <= 1.0).all())


def test_t3_damage_models_refused_where_the_reference_refuses():
    g = golden("t3_models")
    with pytest.raises(NotImplementedError):
        _solver(g, "AT1", True)

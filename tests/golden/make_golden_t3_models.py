"""Golden vectors of the T3 damage models beyond element-history AT2, written by the PhAST reference.

Run in a container where the reference sources are present, passing the reference's
``src`` directory::

    python tests/golden/make_golden_t3_models.py <path-to-reference-src>

Writes ``t3_models.npz`` on the perturbed ``q4_to_triangles`` twin of ``make_golden.py``'s
T3 case: for AT1 with element history and for AT2 with nodal history
(``PhaseFieldDamageSolver(..., nodal_H=True)``), the prepared right-hand side and Jacobi
inverse, one operator action, and a bound-projected solve with its iteration count.
The script reuses the stub import of ``make_golden.py``; it is never run by the tests.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import _import_reference, n, t  # noqa: E402


def main(out):
    from phast.core.fem_operators import FEMOperators
    from phast.core.mesh import FEMMesh
    from phast.core.quad_elements import q4_to_triangles, structured_q4_mesh
    from phast.physics.material import Material
    from phast.solvers.damage_solver import PhaseFieldDamageSolver

    rng = np.random.default_rng(4321)
    sm = structured_q4_mesh(1.0, 0.8, 9, 7)
    nodes = n(sm.nodes).copy()
    inner = (nodes[:, 0] > 1e-9) & (nodes[:, 0] < 1.0 - 1e-9) & (nodes[:, 1] > 1e-9) & (nodes[:, 1] < 0.8 - 1e-9)
    nodes[inner] += rng.uniform(-0.02, 0.02, size=(int(inner.sum()), 2))
    tri = q4_to_triangles(sm.quads)
    mesh = FEMMesh.from_tensors(t(nodes), tri, element_type="T3")
    N, E = mesh.n_nodes, mesh.n_elems
    out.update(nodes=nodes, tris=n(tri))
    rng = np.random.default_rng(77)
    d_prev = np.clip(rng.uniform(-0.3, 0.5, size=N), 0, 1)
    x = rng.uniform(0, 1, size=N)
    out.update(d_prev=d_prev, x=x)
    for key, model, nodal in (("at1", "AT1", False), ("nodal", "AT2", True)):
        mat = Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.05, eta_residual=1e-8, energy_split="isotropic",
                       rho=2.45e-9, pf_model=model)
        fem = FEMOperators(mesh, mat)
        # AT1 needs H above the threshold 3 Gc / (16 l0) somewhere to damage
        H = rng.uniform(0, 400.0, size=N if nodal else E)
        ds = PhaseFieldDamageSolver(fem, tol=1e-10, max_iter=3000, use_multigrid=False,
                                    bounds_method="projected_cg", nodal_H=nodal)
        prep = ds._prepare_cg(t(H), t(d_prev))
        out[f"{key}_H"] = H
        out[f"{key}_Ax"] = n(ds._Ax(t(x), prep[2]))
        out[f"{key}_b"] = n(prep[3])
        out[f"{key}_M_inv"] = n(prep[4])
        out[f"{key}_d_solve"] = n(ds.solve(t(H), t(d_prev)))
        out[f"{key}_iters"] = np.array([ds.last_iter])


if __name__ == "__main__":
    if len(sys.argv) < 2:
        raise SystemExit(__doc__)
    _import_reference(sys.argv[1])
    import torch
    torch.set_num_threads(8)
    res = {}
    main(res)
    np.savez_compressed(os.path.join(HERE, "t3_models.npz"), **res)
    print(sorted(res))

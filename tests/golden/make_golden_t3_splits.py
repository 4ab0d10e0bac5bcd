"""Golden vectors of the split-aware quasi-static mechanics on T3 meshes, written by the PhAST
reference.

Usage: python tests/golden/make_golden_t3_splits.py <path to the reference's src directory>

Writes ``t3_qs_splits.npz``:

* ``tan_<split>``: the autograd JVP of ``FEMOperators.internal_force(u, d)`` with respect to u in a
  direction du on a jittered 9 x 7 ``q4_to_triangles`` mesh (what ``QuasiStaticSolver`` uses as
  its CG operator, mechanics_solver.py:1705-1733), spectral, Amor and star-convex splits;
* ``qs_<split>_*``: three quasi-static SENT load steps of ``StaggeredSolver`` on a 12 x 12 mesh
  cut into triangles, spectral and Amor splits: u, d, the reaction force and the staggered
  iteration counts.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import _import_reference, n, t  # noqa: E402


def tangent_cases(out):
    import torch
    from phast.core.fem_operators import FEMOperators
    from phast.core.mesh import FEMMesh
    from phast.core.quad_elements import q4_to_triangles, structured_q4_mesh
    from phast.physics.material import Material

    rng = np.random.default_rng(77)
    sm = structured_q4_mesh(1.0, 0.8, 9, 7)
    nodes = n(sm.nodes).copy()
    inner = (nodes[:, 0] > 1e-9) & (nodes[:, 0] < 1.0 - 1e-9) & (nodes[:, 1] > 1e-9) & (nodes[:, 1] < 0.8 - 1e-9)
    nodes[inner] += rng.uniform(-0.02, 0.02, size=(int(inner.sum()), 2))
    tri = q4_to_triangles(sm.quads)
    mesh = FEMMesh.from_tensors(t(nodes), tri, element_type="T3")
    N = mesh.n_nodes
    u = np.stack([1e-3 * np.sin(3.0 * nodes[:, 0]) * nodes[:, 1], -8e-4 * np.cos(2.5 * nodes[:, 1]) * nodes[:, 0]], 1)
    u = u + rng.normal(size=(N, 2)) * 2e-4
    d = rng.uniform(0.0, 0.8, size=N)
    du = rng.normal(size=(N, 2)) * 1e-4
    out.update(tan_nodes=nodes, tan_tris=n(tri), tan_u=u, tan_d=d, tan_du=du)
    for split in ("spectral", "amor", "star_convex"):
        mat = Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.05, eta_residual=1e-8, energy_split=split)
        fem = FEMOperators(mesh, mat)
        _, jvp = torch.autograd.functional.jvp(lambda uu: fem.internal_force(uu, t(d)), (t(u),), (t(du),))
        out[f"tan_{split}"] = n(jvp)


def qs_cases(out):
    import torch
    from phast.core.mesh import FEMMesh
    from phast.core.quad_elements import q4_to_triangles, structured_q4_mesh
    from phast.physics.material import Material
    from phast.physics.boundary_conditions import BoundaryConditions
    from phast.solvers.staggered_solver import StaggeredSolver, SolverConfig

    nx = ny = 12
    sm = structured_q4_mesh(1.0, 1.0, nx, ny)
    tri = q4_to_triangles(sm.quads)
    mesh = FEMMesh.from_tensors(sm.nodes, tri, element_type="T3")
    N = mesh.n_nodes
    nodes = sm.nodes.numpy()
    notch = np.nonzero((np.abs(nodes[:, 1] - 0.5) < 1e-12) & (nodes[:, 0] < 0.5))[0]
    out.update(qs_nx=np.array([nx]), qs_notch=notch, qs_tris=n(tri))
    for split in ("spectral", "amor"):
        mat = Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.1, eta_residual=1e-8, energy_split=split, rho=7.8e-9)
        bcs = BoundaryConditions(N)
        bot, top = sm.node_sets["bottom"], sm.node_sets["top"]
        bcs.fix(bot, 0)
        bcs.fix(bot, 1)
        bcs.add(top, 1, 1.0)
        bcs.add_pf_dirichlet(torch.as_tensor(notch), 1.0)
        cfg = SolverConfig(solver_type="quasi_static", backend="cg", static_tol=1e-10, damage_tol=1e-10,
                           bounds_method="projected_cg", use_multigrid=False, stagger_tol=1e-6, max_stagger=100)
        s = StaggeredSolver(mesh, mat, bcs, cfg)
        pf_mask, pf_vals = bcs.get_pf_dirichlet_mask_values()
        s.d = torch.where(pf_mask, pf_vals, s.d)
        us, ds_, rf, stag = [], [], [], []
        for k in range(1, 4):
            bcs.load_factor = 0.004 * k
            s.step_full()
            us.append(n(s.u))
            ds_.append(n(s.d))
            rf.append(s.fem.compute_reaction_force(s.u, s.d, top, component=1))
            stag.append(s._last_stagger_iter)
            print(f"{split} step {k}: stagger {stag[-1]}, reaction {rf[-1]:.4f}, max d {float(s.d.max()):.4f}")
        out.update({f"qs_{split}_u": np.stack(us), f"qs_{split}_d": np.stack(ds_), f"qs_{split}_rf": np.array(rf),
                    f"qs_{split}_stag": np.array(stag)})


if __name__ == "__main__":
    if len(sys.argv) < 2:
        raise SystemExit(__doc__)
    _import_reference(sys.argv[1])
    import torch
    torch.set_num_threads(8)
    out = {}
    tangent_cases(out)
    qs_cases(out)
    np.savez_compressed(os.path.join(HERE, "t3_qs_splits.npz"), **out)
    print("written", os.path.join(HERE, "t3_qs_splits.npz"))

"""Golden vectors of the split-aware quasi-static mechanics, written by the PhAST reference.

Run in a container where the reference sources are present, passing the reference's
``src`` directory::

    python tests/golden/make_golden_splits.py <path-to-reference-src>

Writes ``q4_qs_splits.npz``:

* ``tan_<split>_*``: the consistent tangent action, i.e. the autograd JVP of
  ``FEMOperators.internal_force(u, d)`` with respect to u in a direction du (what
  ``QuasiStaticSolver`` uses as its CG operator, mechanics_solver.py:1705-1733), on a
  10 x 6 Q4 mesh with seeded u (tension and compression present), d and du, for the
  spectral, Amor and star-convex splits (plane strain) and Amor in plane stress;
* ``qs_<split>_*``: three quasi-static SENT load steps of ``StaggeredSolver`` on a 12 x 12
  mesh with the spectral and the Amor split: u, d, H, the reaction force and the staggered
  iteration counts per step.

The script reuses the stub import of ``make_golden.py``; it is never run by the tests.
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
    from phast.core.quad_elements import structured_q4_mesh
    from phast.physics.material import Material

    sm = structured_q4_mesh(2.0, 1.2, 10, 6)
    mesh = FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4")
    N = mesh.n_nodes
    rng = np.random.default_rng(21)
    nodes = sm.nodes.numpy()
    # a smooth field with tensile and compressive regions plus noise
    u = np.stack([1e-3 * np.sin(2.0 * nodes[:, 0]) * nodes[:, 1], -8e-4 * np.cos(1.5 * nodes[:, 1]) * nodes[:, 0]], 1)
    u = u + rng.normal(size=(N, 2)) * 2e-4
    d = rng.uniform(0.0, 0.8, size=N)
    du = rng.normal(size=(N, 2)) * 1e-4
    out.update(tan_nx=np.array([10]), tan_ny=np.array([6]), tan_w=np.array([2.0]), tan_h=np.array([1.2]),
               tan_u=u, tan_d=d, tan_du=du)
    for split, ps in (("spectral", False), ("amor", False), ("star_convex", False), ("amor", True)):
        mat = Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.05, eta_residual=1e-8, energy_split=split,
                       plane_stress=ps)
        fem = FEMOperators(mesh, mat)
        _, jvp = torch.autograd.functional.jvp(lambda uu: fem.internal_force(uu, t(d)), (t(u),), (t(du),))
        key = f"tan_{split}{'_ps' if ps else ''}"
        out[key] = n(jvp)
        out[key + "_f"] = n(fem.internal_force(t(u), t(d)))


def qs_cases(out):
    import torch
    from phast.core.mesh import FEMMesh
    from phast.core.quad_elements import structured_q4_mesh
    from phast.physics.boundary_conditions import BoundaryConditions
    from phast.physics.material import Material
    from phast.solvers.staggered_solver import SolverConfig, StaggeredSolver

    nx = ny = 12
    sm = structured_q4_mesh(1.0, 1.0, nx, ny)
    mesh = FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4")
    N = mesh.n_nodes
    nodes = sm.nodes.numpy()
    notch = np.nonzero((np.abs(nodes[:, 1] - 0.5) < 1e-12) & (nodes[:, 0] < 0.5))[0]
    out.update(qs_nx=np.array([nx]), qs_ny=np.array([ny]), qs_notch=notch)
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
        us, ds_, Hs, rf, stag = [], [], [], [], []
        for k in range(1, 4):
            bcs.load_factor = 0.004 * k
            s.step_full()
            us.append(n(s.u))
            ds_.append(n(s.d))
            Hs.append(n(s.H_elem))
            rf.append(s.fem.compute_reaction_force(s.u, s.d, top, component=1))
            stag.append(s._last_stagger_iter)
        out.update({f"qs_{split}_u": np.stack(us), f"qs_{split}_d": np.stack(ds_), f"qs_{split}_H": np.stack(Hs),
                    f"qs_{split}_rf": np.array(rf), f"qs_{split}_stag": np.array(stag)})


if __name__ == "__main__":
    if len(sys.argv) < 2:
        raise SystemExit(__doc__)
    _import_reference(sys.argv[1])
    import torch
    torch.set_num_threads(8)
    res = {}
    tangent_cases(res)
    qs_cases(res)
    np.savez_compressed(os.path.join(HERE, "q4_qs_splits.npz"), **res)
    print(sorted(res))

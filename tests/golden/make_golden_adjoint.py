"""Writes t3_qs_adjoint.npz: PhAST's own autograd gradient of the peak reaction force of a
quasi-static staggered run with respect to a per-element Gc field, on a small T3 mesh.

Usage: python tests/golden/make_golden_adjoint.py <path to PhAST's src directory>

The run is a single-edge-notched tension test on a jittered triangulation of the unit
square (16 x 16 quads, two triangles each; the notch row y = 0.5, the loaded top edge and
the fixed bottom edge are kept straight).  PhAST's pieces, as its differentiable workflow
assembles them:

* ``Material(..., gamma_correction=True)`` so that the damage solver routes a per-element
  ``Gc_field`` that requires grad through ``_AdjointDamageSolveField``
  (solvers/damage_solver.py:866-1037);
* ``QuasiStaticSolver`` with ``backend='scipy'``: every Newton step is a
  ``SparseSolveAutograd`` solve whose stiffness values carry the degradation g(d)
  (solvers/mechanics_solver.py:1118-1301);
* ``StaggeredSolver.step_full`` with ``diff_Gc_field`` set (staggered_solver.py:904-936),
  history by ``torch.maximum`` (staggered_solver.py:804-860);
* objective J = max_k sum over the top nodes of internal_force(u_k, d_k)[:, 1]
  (compute_reaction_force, core/fem_operators.py:1502-1530, kept as a tensor).

The load stays below crack propagation, so no damage node reaches a bound other than the
pinned notch: there PhAST's solve-then-clamp adjoint and the exact derivative of the
bound-projected solve coincide, and the file records the bound activity it saw.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from make_golden import _import_reference, n, t  # noqa: E402

NX = 16
STEPS = 5
LOAD = 0.0016          # top displacement increment per load step
GC_MEAN, GC_COV = 2.7, 0.2


def mesh_arrays():
    """Nodes (jittered off the notch row and the boundary) and triangles of the twin."""
    from phast.core.quad_elements import q4_to_triangles, structured_q4_mesh
    sm = structured_q4_mesh(1.0, 1.0, NX, NX)
    nodes = n(sm.nodes).copy()
    x, y = nodes[:, 0], nodes[:, 1]
    keep = (x < 1e-9) | (x > 1 - 1e-9) | (y < 1e-9) | (y > 1 - 1e-9) | (np.abs(y - 0.5) < 1e-9)
    rng = np.random.default_rng(2024)
    h = 1.0 / NX
    nodes[~keep] += rng.uniform(-0.15 * h, 0.15 * h, size=(int((~keep).sum()), 2))
    tri = n(q4_to_triangles(sm.quads))
    return nodes, tri, n(sm.node_sets["top"]), n(sm.node_sets["bottom"])


def main():
    import torch
    from phast.core.mesh import FEMMesh
    from phast.physics.boundary_conditions import BoundaryConditions
    from phast.physics.material import Material
    from phast.solvers.damage_solver import classify_damage_active_set
    from phast.solvers.staggered_solver import SolverConfig, StaggeredSolver

    nodes, tri, top, bot = mesh_arrays()
    mesh = FEMMesh.from_tensors(t(nodes), torch.as_tensor(tri), element_type="T3")
    N, E = mesh.n_nodes, mesh.n_elems
    notch = np.nonzero((np.abs(nodes[:, 1] - 0.5) < 1e-12) & (nodes[:, 0] < 0.5))[0]
    rng = np.random.default_rng(7)
    s2 = np.log(1 + GC_COV ** 2)
    gc = GC_MEAN * np.exp(np.sqrt(s2) * rng.standard_normal(E) - 0.5 * s2)

    mat = Material(E=210000.0, nu=0.3, Gc=GC_MEAN, l0=0.125, eta_residual=1e-8, energy_split="isotropic",
                   rho=7.8e-9, gamma_correction=True)
    bcs = BoundaryConditions(N)
    bcs.fix(torch.as_tensor(bot), 0)
    bcs.fix(torch.as_tensor(bot), 1)
    bcs.add(torch.as_tensor(top), 1, 1.0)
    bcs.add_pf_dirichlet(torch.as_tensor(notch), 1.0)
    cfg = SolverConfig(solver_type="quasi_static", backend="scipy", static_tol=1e-11, damage_tol=1e-12,
                       damage_max_iter=5000, bounds_method="projected_cg", use_multigrid=False,
                       stagger_tol=1e-10, max_stagger=200)
    s = StaggeredSolver(mesh, mat, bcs, cfg)
    pf_mask, pf_vals = bcs.get_pf_dirichlet_mask_values()
    s.d = torch.where(pf_mask, pf_vals, s.d)
    gc_t = t(gc).requires_grad_(True)
    s.diff_Gc_field = gc_t
    top_t = torch.as_tensor(top)
    R, stag, lower, upper, dmax = [], [], [], [], []
    us, ds_ = [], []
    for k in range(1, STEPS + 1):
        d_start = s.d.detach().clone()
        bcs.load_factor = LOAD * k
        s.step_full()
        R.append(s.fem.internal_force(s.u, s.d)[top_t, 1].sum())
        stag.append(s._last_stagger_iter)
        a = classify_damage_active_set(s.d.detach(), d_start, fixed=pf_mask)
        lower.append(int(a.lower.sum()))
        upper.append(int(a.upper.sum()))
        dmax.append(float(s.d.detach()[~pf_mask].max()))
        us.append(n(s.u))
        ds_.append(n(s.d))
    Rt = torch.stack(R)
    J = Rt.max()
    J.backward()
    out = dict(nodes=nodes, tris=tri, top=top, bottom=bot, notch=notch, gc=gc, load=np.array([LOAD]),
               reactions=n(Rt), stag=np.array(stag), lower_active=np.array(lower), upper_active=np.array(upper),
               d_max=np.array(dmax), u=np.stack(us), d=np.stack(ds_), grad=n(gc_t.grad),
               peak_step=np.array([int(torch.argmax(Rt)) + 1]))
    print("reactions", out["reactions"], "passes", stag, "lower/upper active", lower, upper, "d max", dmax)
    np.savez_compressed(os.path.join(HERE, "t3_qs_adjoint.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        raise SystemExit(__doc__)
    _import_reference(sys.argv[1])
    import torch
    torch.set_num_threads(8)
    main()

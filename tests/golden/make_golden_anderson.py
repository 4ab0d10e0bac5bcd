"""Writes tests/golden/anderson.npz from the reference's own Anderson mixing of the 2D staggered
damage fixed point (``SolverConfig.anderson_depth``).

Usage: python tests/golden/make_golden_anderson.py <path to the reference's src directory>

Cases (CPU, float64, the reference's own classes):
  * the accelerator alone (_AndersonAccelerator.step, solvers/staggered_solver.py:165-255) on a
    seeded sequence of (d_in, G(d_in)) pairs of a damped affine map, with and without the
    irreversibility floor, depth 3;
  * quasi-static SENT load steps through StaggeredSolver.step_full with anderson_depth = 3
    (staggered_solver.py:1229-1259).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import _import_reference, n, t  # noqa: E402


def accelerator_case(out):
    import torch
    from phast.solvers.staggered_solver import _AndersonAccelerator

    rng = np.random.default_rng(31)
    N = 64
    A = rng.normal(size=(N, N)) * 0.08
    b = rng.uniform(0.2, 0.8, size=N)
    floor = np.clip(rng.uniform(-0.2, 0.4, size=N), 0, 1)
    for tag, use_floor in (("floor", True), ("nofloor", False)):
        aa = _AndersonAccelerator(m=3)
        d = np.clip(rng.uniform(0, 0.5, size=N), 0, 1)
        ins, outs, mixed = [], [], []
        for _ in range(8):
            g = np.clip(A @ d + b, -0.5, 1.5)  # G(d), not clamped to the box
            res = aa.step(t(d), t(g), d_prev_step=t(floor) if use_floor else None)
            ins.append(d.copy())
            outs.append(g.copy())
            d = n(res)
            mixed.append(d.copy())
        out[f"acc_{tag}_in"], out[f"acc_{tag}_out"], out[f"acc_{tag}_mix"] = map(np.stack, (ins, outs, mixed))
    out["acc_floor"] = floor


def sent_case(out):
    import torch
    from phast.core.mesh import FEMMesh
    from phast.core.quad_elements import structured_q4_mesh
    from phast.physics.material import Material
    from phast.physics.boundary_conditions import BoundaryConditions
    from phast.solvers.staggered_solver import StaggeredSolver, SolverConfig

    nx = ny = 16
    sm = structured_q4_mesh(1.0, 1.0, nx, ny)
    mesh = FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4")
    N = mesh.n_nodes
    mat = Material(E=210000.0, nu=0.3, Gc=2.7, l0=0.1, eta_residual=1e-8, energy_split="isotropic", rho=7.8e-9)
    bcs = BoundaryConditions(N)
    bot, top = sm.node_sets["bottom"], sm.node_sets["top"]
    bcs.fix(bot, 0)
    bcs.fix(bot, 1)
    bcs.add(top, 1, 1.0)
    nodes = sm.nodes.numpy()
    notch = np.nonzero((np.abs(nodes[:, 1] - 0.5) < 1e-12) & (nodes[:, 0] < 0.5))[0]
    bcs.add_pf_dirichlet(torch.as_tensor(notch), 1.0)
    cfg = SolverConfig(solver_type="quasi_static", backend="cg", static_tol=1e-10, damage_tol=1e-10,
                       bounds_method="projected_cg", use_multigrid=False, stagger_tol=1e-6, max_stagger=100,
                       anderson_depth=3)
    s = StaggeredSolver(mesh, mat, bcs, cfg)
    pf_mask, pf_vals = bcs.get_pf_dirichlet_mask_values()
    s.d = torch.where(pf_mask, pf_vals, s.d)
    loads = (0.004, 0.008, 0.010, 0.011)
    us, ds_, stag, rf = [], [], [], []
    for lf in loads:
        bcs.load_factor = lf
        s.step_full()
        us.append(n(s.u))
        ds_.append(n(s.d))
        stag.append(s._last_stagger_iter)
        rf.append(s.fem.compute_reaction_force(s.u, s.d, top, component=1))
        print(f"load {lf}: stagger {s._last_stagger_iter}, max d {float(s.d.max()):.4f}, reaction {rf[-1]:.4f}")
    out.update(nx=nx, ny=ny, notch=notch, loads=np.array(loads), sent_u=np.stack(us), sent_d=np.stack(ds_),
               sent_stag=np.array(stag), sent_rf=np.array(rf))


if __name__ == "__main__":
    if len(sys.argv) < 2:
        raise SystemExit(__doc__)
    _import_reference(sys.argv[1])
    import torch
    torch.set_num_threads(8)
    out = {}
    accelerator_case(out)
    sent_case(out)
    np.savez_compressed(os.path.join(HERE, "anderson.npz"), **out)
    print("written", os.path.join(HERE, "anderson.npz"))

"""Golden fixtures at the benchmark configurations, written by the PhAST reference.

Usage (in a container where the reference sources are present)::

    python tests/golden/make_golden_configs.py <path-to-reference-src> [cfg0|cfg1|cfg1_tight|cfg2 ...]

The reference is imported with the same stub modules as ``make_golden.py``
(I/O-only dependencies the hot path never calls).  Each case runs the
reference's own solver classes on the full-size seeded inputs of one
configuration for a short window and stores the fields at the end of the
window plus per-step scalars:

* ``cfg0_sent200.npz`` / ``cfg0_sent200_tight.npz``: 2D quasi-static
  single-edge-notched tension, structured Q4 200 x 200, isotropic split; load
  steps 1-3 of the 100-step ramp to 0.007 mm
  (``phast.solvers.staggered_solver.StaggeredSolver.step_full``), once with the
  configuration's CG and projected-CG tolerances of 1e-10 and once with both at
  1e-12.
* ``cfg1_pore64.npz`` / ``cfg1_pore64_tight.npz``: 3D periodic 64^3 pore cell,
  AT2 spectral, eps_zz ramp to 0.02 in 50 increments; increments 1-3
  (``phast.solid3d.staggered.StaggeredSolver.advance``), once at PhAST's
  default tolerances and once with ``pcg_rtol_mech`` and
  ``damage_linear_tol`` at 1e-12.
* ``cfg2_branch400.npz``: 2D explicit crack branching, Q4 400 x 160 on
  100 x 40 mm, spectral split, +-1 MPa edge traction assembled on ``f_ext``
  (interior edge nodes t h, corners t h / 2), damage solved every step;
  steps 1-200.

The tests never run this script; they read the fixtures it wrote.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import make_golden as mg  # noqa: E402  (stub importer, voxel model builder)


def n(x):
    return x.detach().cpu().numpy()


def _sent_q4(nx, ny, width, height, mat_kwargs, cfg_kwargs, crack_y, crack_x_max, top_bottom_bc):
    import torch
    from phast.core.mesh import FEMMesh
    from phast.core.quad_elements import structured_q4_mesh
    from phast.physics.boundary_conditions import BoundaryConditions
    from phast.physics.material import Material
    from phast.solvers.staggered_solver import SolverConfig, StaggeredSolver

    sm = structured_q4_mesh(width, height, nx, ny)
    mesh = FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4")
    N = mesh.n_nodes
    mat = Material(**mat_kwargs)
    bcs = BoundaryConditions(N)
    bot, top = sm.node_sets["bottom"], sm.node_sets["top"]
    if top_bottom_bc:
        bcs.fix(bot, 0)
        bcs.fix(bot, 1)
        bcs.add(top, 1, 1.0)
    nodes = sm.nodes.numpy()
    notch = np.nonzero((np.abs(nodes[:, 1] - crack_y) < 1e-9 * height) & (nodes[:, 0] < crack_x_max))[0]
    bcs.add_pf_dirichlet(torch.as_tensor(notch), 1.0)
    s = StaggeredSolver(mesh, mat, bcs, SolverConfig(**cfg_kwargs))
    pf_mask, pf_vals = bcs.get_pf_dirichlet_mask_values()
    s.d = torch.where(pf_mask, pf_vals, s.d)
    return s, sm, bcs, notch, top, bot


def _cfg0(tight):
    """200 x 200 SENT, load steps 1-3 of 100 (top uy = 0.007 k / 100)."""
    mat = dict(E=210000.0, nu=0.3, Gc=2.7, l0=0.01, eta_residual=1e-8, energy_split="isotropic", rho=7.8e-9)
    tol = 1e-12 if tight else 1e-10
    cfg = dict(solver_type="quasi_static", backend="cg", static_tol=tol, damage_tol=tol,
               bounds_method="projected_cg", use_multigrid=False, stagger_tol=1e-6, max_stagger=500)
    s, sm, bcs, notch, top, bot = _sent_q4(200, 200, 1.0, 1.0, mat, cfg, 0.5, 0.5, True)
    out = {"nx": 200, "ny": 200, "notch": notch, "steps": np.arange(1, 4)}
    us, ds, rf, stag, secs = [], [], [], [], []
    for k in range(1, 4):
        bcs.load_factor = 0.007 * k / 100
        t0 = time.perf_counter()
        s.step_full()
        secs.append(time.perf_counter() - t0)
        us.append(n(s.u))
        ds.append(n(s.d))
        rf.append(s.fem.compute_reaction_force(s.u, s.d, top, component=1))
        stag.append(s._last_stagger_iter)
        print(f"cfg0 step {k}: {secs[-1]:.1f} s, stagger {stag[-1]}, reaction {rf[-1]:.9e}", flush=True)
    out.update(u=np.stack(us), d=np.stack(ds), H=n(s.H_elem), rf=np.array(rf), stag=np.array(stag),
               ref_seconds=np.array(secs), tol=np.array([tol]))
    np.savez_compressed(os.path.join(HERE, "cfg0_sent200_tight.npz" if tight else "cfg0_sent200.npz"), **out)


def cfg0():
    _cfg0(False)


def cfg0_tight():
    _cfg0(True)


def _cfg1(tight):
    from phast.solid3d.model import LoadCase, SolverConfig
    from phast.solid3d.operator import PeriodicVoxelPhaseFieldOperator
    from phast.solid3d.staggered import StaggeredSolver

    N = 64
    h = 1.0 / N
    model, phase = mg._voxel_model((N, N, N), h, 0.2)
    targets = tuple(0.02 * k / 50 for k in range(1, 51))
    load = LoadCase(name="zz", controlled=2, targets=targets, free=(), fixed_zero=(0, 1, 3, 4, 5))
    extra = dict(pcg_rtol_mech=1e-12, damage_linear_tol=1e-12) if tight else {}
    cfg = SolverConfig(device="cpu", kappa=1e-6, energy_split_isotropic="spectral", damage_law="at2", **extra)
    op = PeriodicVoxelPhaseFieldOperator(model, load, cfg)
    solver = StaggeredSolver(op)
    state = solver.initial_state()
    sig, stag, pm, pp, sets, dmax, Hsum, Hmax, secs = [], [], [], [], [], [], [], [], []
    for k in range(3):
        t0 = time.perf_counter()
        state, rec = solver.advance(state, targets[k])
        secs.append(time.perf_counter() - t0)
        sig.append(np.array(rec.macro_stress))
        stag.append(rec.stagger_iters)
        pm.append(rec.pcg_iters_mech)
        pp.append(rec.pcg_iters_pf)
        sets.append(rec.active_set_iters)
        dmax.append(float(state.d.max()))
        Hsum.append(float(state.H.sum()))
        Hmax.append(float(state.H.max()))
        print(f"cfg1{' tight' if tight else ''} increment {k + 1}: {secs[-1]:.1f} s, stagger {stag[-1]}, "
              f"pcg mech {pm[-1]}, pcg pf {pp[-1]}", flush=True)
    out = {"shape": np.array((N, N, N)), "h": h, "phase": phase, "pinned": op.pinned_node,
           "targets": np.array(targets[:3]), "rtol_mech": cfg.pcg_rtol_mech, "damage_linear_tol": cfg.damage_linear_tol,
           "x": n(state.x), "d": n(state.d), "sigma": np.stack(sig), "stag": np.array(stag), "pcg_mech": np.array(pm),
           "pcg_pf": np.array(pp), "active_sets": np.array(sets), "dmax": np.array(dmax), "H_sum": np.array(Hsum),
           "H_max": np.array(Hmax), "ref_seconds": np.array(secs)}
    name = "cfg1_pore64_tight.npz" if tight else "cfg1_pore64.npz"
    np.savez_compressed(os.path.join(HERE, name), **out)


def cfg1():
    _cfg1(False)


def cfg1_tight():
    _cfg1(True)


def cfg2():
    """400 x 160 explicit crack branching, 200 central-difference steps with a damage solve each."""
    import torch
    nx, ny, W, Hh = 400, 160, 100.0, 40.0
    mat = dict(E=32000.0, nu=0.2, Gc=3e-3, l0=0.5, rho=2.45e-9, eta_residual=1e-8, energy_split="spectral")
    cfg = dict(solver_type="explicit", dt_safety=0.5, damage_every=1, damage_tol=1e-10,
               bounds_method="projected_cg", use_multigrid=False)
    s, sm, bcs, notch, top, bot = _sent_q4(nx, ny, W, Hh, mat, cfg, 20.0, 50.0, False)
    N = s.u.shape[0]
    f_ext = np.zeros((N, 2))
    hx = W / nx
    for nodeset, sign in ((top.numpy(), 1.0), (bot.numpy(), -1.0)):
        nodeset = nodeset[np.argsort(sm.nodes.numpy()[nodeset, 0])]
        w = np.full(len(nodeset), hx)
        w[0] = w[-1] = hx / 2
        f_ext[nodeset, 1] = sign * 1.0 * w
    s.f_ext = torch.as_tensor(f_ext, dtype=torch.float64)
    out = {"nx": nx, "ny": ny, "width": W, "height": Hh, "notch": notch, "f_ext": f_ext, "dt": np.array([s.dt])}
    dmax, unorm, dsum = [], [], []
    t0 = time.perf_counter()
    for k in range(1, 201):
        s.step_full()
        dmax.append(float(s.d.max()))
        dsum.append(float(s.d.sum()))
        unorm.append(float(torch.linalg.vector_norm(s.u)))
        if k == 100:
            out.update(u100=n(s.u), d100=n(s.d))
        if k % 50 == 0:
            print(f"cfg2 step {k}: {time.perf_counter() - t0:.1f} s", flush=True)
    out.update(u=n(s.u), v=n(s.v), a=n(s.a), d=n(s.d), H=n(s.H_elem), dmax=np.array(dmax), dsum=np.array(dsum),
               unorm=np.array(unorm), ref_seconds=np.array([time.perf_counter() - t0]))
    np.savez_compressed(os.path.join(HERE, "cfg2_branch400.npz"), **out)


CASES = {"cfg0": cfg0, "cfg0_tight": cfg0_tight, "cfg1": cfg1, "cfg1_tight": cfg1_tight, "cfg2": cfg2}

if __name__ == "__main__":
    if len(sys.argv) < 2:
        raise SystemExit(__doc__)
    mg._import_reference(sys.argv[1])
    import torch
    torch.set_num_threads(int(os.environ.get("GOLDEN_THREADS", "8")))
    for name in (sys.argv[2:] or list(CASES)):
        CASES[name]()
    print("fixtures written to", HERE)

"""Benchmark: staggered load increments per second of the 3D periodic voxel pore cell.

Workload (the metric's single-GPU configuration): 64^3 periodic voxel H8 cell,
edge 1 mm, one spherical pore of radius 0.2 at the centre with E x 1e-6,
matrix E = 3 GPa, nu = 0.35, Gc = 0.5 N/mm, ell = 2 voxels, hybrid AT2 with
kappa = 1e-6, spectral driver; uniaxial macro strain eps_zz ramped 0 -> 0.02 in
50 increments.  A "step" is one staggered load increment (mechanics PCG,
driving force + history, box-KKT damage solve, until the staggered change is
below 1e-4, then the final mechanics re-solve).  Inputs are synthetic (the
geometry above, built in memory).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (torchrun, one process per GPU) every rank runs its own replica of
the cell: the workload does not shard (replicas only), the value is the total
increments of all ranks over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "staggered steps/s, chosen vs plain FP64 on 1 B200 at ≤1e-6 rel err; HBM GB/s"
UNIT = "staggered steps/s"
N_CELL = 64
N_LARGE = 192  # roofline cell: the action's working set (about 200 MB in FP32) exceeds the 126 MB L2
INCREMENTS = 50
# Wall-clock budgets of the reference's whole increments: the reference arm's
# timed region, and the CPU baseline sample inside our arm's run.
REF_BUDGET_S = 150.0
CPU_BASELINE_BUDGET_S = 30.0


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload_config():
    return {
        "workload": "3D periodic voxel H8 pore cell 64^3 (r=0.2 L, E x 1e-6), AT2 spectral, eps_zz 0->0.02 in 50 "
                    "increments; step = one staggered load increment",
        "cells": 1, "voxels": N_CELL ** 3, "mechanics": "constrained PCG, FP64 residual rtol 1e-8",
        "damage": "box-KKT active set + Dirichlet PCG (FP64)",
        "window": "load increments 1..K of the ramp from the initial state",
        "l2": "flushed (256 MB write) before every timed step", "parallelism": "replicas",
    }


def build_cell(device, n=None):
    from phast_b200 import solid3d as s3
    n = N_CELL if n is None else n
    h = 1.0 / n
    shape = (n, n, n)
    model = s3.sphere_pore_model(shape, 0.2, E=3000.0, nu=0.35, Gc=0.5, ell_voxels=2.0, pore_stiffness=1e-6)
    load = s3.LoadCase.ramp("zz", 2, 0.02, INCREMENTS)
    cfg = s3.SolverConfig(device=str(device), kappa=1e-6, energy_split_isotropic="spectral", damage_law="at2")
    op = s3.PeriodicVoxelPhaseFieldOperator(model, load, cfg)
    return op, s3.StaggeredSolver(op)


class Clocks:
    """nvidia-smi sampler over the timed region (SM clock, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # the sampler needs a moment to start: wait (at most 2 s) for its first row, so that
        # the samples cover the timed region that follows
        t0 = time.time()
        while time.time() - t0 < 2.0 and os.path.getsize(self.path) == 0:
            time.sleep(0.01)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.remove(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def flush_l2(buf):
    buf.add_(1)


# ---------------------------------------------------------------------------
# The reference: PhAST's own CPU implementation of the path, installed under
# baseline/_ref (the unmodified package), timed on whole load increments
# ---------------------------------------------------------------------------

REF_DIR = os.path.join(ROOT, "baseline", "_ref")
# I/O-only dependencies of the reference package that the solver path never calls
# (mesh files, HDF5/zarr result files, plots); they are not installed here.
REF_STUBS = ("meshio", "gmsh", "h5py", "zarr", "numcodecs", "matplotlib", "mpl_toolkits")


def import_reference():
    """Import ``phast`` from baseline/_ref with permissive stubs for its I/O-only modules."""
    import importlib.abc
    import importlib.machinery
    from unittest import mock

    if "phast" in sys.modules:
        return sys.modules["phast"]
    if not os.path.isdir(os.path.join(REF_DIR, "phast")):
        raise ImportError(f"the reference is not installed under {os.path.relpath(REF_DIR, ROOT)}")

    class _Stubs(importlib.abc.MetaPathFinder, importlib.abc.Loader):
        def find_spec(self, name, path=None, target=None):
            if name.split(".")[0] in REF_STUBS:
                return importlib.machinery.ModuleSpec(name, self, is_package=True)
            return None

        def create_module(self, spec):
            m = mock.MagicMock(name=spec.name)
            m.__path__ = []
            m.__spec__ = spec
            return m

        def exec_module(self, module):
            pass

    sys.meta_path.insert(0, _Stubs())
    sys.path.insert(0, REF_DIR)
    import phast  # noqa: F401
    return phast


def reference_solver():
    """The bench cell built with the reference's own classes (phast.solid3d)."""
    from phast.solid3d.model import (PHASE_ID, LoadCase, MaterialTable, PhaseMaterial, SolverConfig, VoxelGrid,
                                     VoxelModel)
    from phast.solid3d.operator import PeriodicVoxelPhaseFieldOperator
    from phast.solid3d.staggered import StaggeredSolver
    n = N_CELL
    h = 1.0 / n
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    c = np.stack([(i + 0.5) / n - 0.5, (j + 0.5) / n - 0.5, (k + 0.5) / n - 0.5], -1)
    phase = np.full((n, n, n), PHASE_ID["mi_matrix"], dtype=np.uint8)
    phase[np.linalg.norm(c, axis=-1) < 0.2] = PHASE_ID["pore"]
    phases = {"mi_matrix": PhaseMaterial(name="mi_matrix", kind="isotropic", Gc=0.5, driver="spectral", E=3000.0,
                                         nu=0.35),
              "pore": PhaseMaterial(name="pore", kind="isotropic", Gc=0.5, driver="spectral", E=3000.0 * 1e-6,
                                    nu=0.35)}
    tangent = np.zeros((n, n, n, 3))
    tangent[..., 2] = 1.0
    model = VoxelModel(grid=VoxelGrid(shape=(n, n, n), h=(h, h, h)), phase_id=phase, tangent=tangent,
                       materials=MaterialTable(phases=phases, length_scale=2 * h, scale="micro"))
    targets = tuple(0.02 * k / INCREMENTS for k in range(1, INCREMENTS + 1))
    load = LoadCase(name="zz", controlled=2, targets=targets, free=(), fixed_zero=(0, 1, 3, 4, 5))
    cfg = SolverConfig(device="cpu", kappa=1e-6, energy_split_isotropic="spectral", damage_law="at2")
    op = PeriodicVoxelPhaseFieldOperator(model, load, cfg)
    return op, StaggeredSolver(op)


def time_reference(max_increments, budget_s, warmup=0):
    """Whole staggered increments of the reference on the host cores, from the initial state.

    Runs ``warmup`` untimed elastic actions, then increments 1, 2, ... until
    ``max_increments`` are done or the next one would end past ``budget_s``
    (at least one).  Returns (seconds per increment, threads, records).
    """
    import torch as th
    import_reference()
    threads = os.cpu_count() or 1
    th.set_num_threads(threads)
    op, solver = reference_solver()
    state = solver.initial_state()
    for _ in range(warmup):
        op.mech_action(state.x)
    secs, recs = [], []
    for k in range(max_increments):
        t0 = time.perf_counter()
        state, rec = solver.advance(state, op.load.targets[k])
        secs.append(time.perf_counter() - t0)
        recs.append(rec)
        if sum(secs) + secs[-1] > budget_s:
            break
    return secs, th.get_num_threads(), recs


def reference_sample_note(secs, recs, threads):
    its = ", ".join(f"{r.stagger_iters}/{r.pcg_iters_mech}/{r.pcg_iters_pf}" for r in recs)
    return (f"PhAST {PHAST_VERSION} phast.solid3d.StaggeredSolver.advance (FP64, torch CPU, {threads} threads) on the "
            f"same 64^3 cell: increments 1-{len(secs)} of the load path from the initial state, whole increments "
            f"timed ({', '.join(f'{s:.1f}' for s in secs)} s; staggered/mechanics PCG/damage PCG iterations {its})")


PHAST_VERSION = "0.18.0"


# ---------------------------------------------------------------------------
# the 2D configurations: quasi-static SENT 200 x 200 (cfg0) and explicit crack
# branching 400 x 160 (cfg2), each beside the reference's own CPU time
# ---------------------------------------------------------------------------

CFG0 = dict(nx=200, ny=200, width=1.0, height=1.0, crack_y=0.5, crack_x=0.5, bc=True,
            mat=dict(E=210000.0, nu=0.3, Gc=2.7, l0=0.01, eta_residual=1e-8, energy_split="isotropic", rho=7.8e-9),
            cfg=dict(solver_type="quasi_static", backend="cg", static_tol=1e-10, damage_tol=1e-10,
                     bounds_method="projected_cg", use_multigrid=False, stagger_tol=1e-6, max_stagger=500))
CFG2 = dict(nx=400, ny=160, width=100.0, height=40.0, crack_y=20.0, crack_x=50.0, bc=False,
            mat=dict(E=32000.0, nu=0.2, Gc=3e-3, l0=0.5, rho=2.45e-9, eta_residual=1e-8, energy_split="spectral"),
            cfg=dict(solver_type="explicit", dt_safety=0.5, damage_every=1, damage_tol=1e-10,
                     bounds_method="projected_cg", use_multigrid=False))
CFG0_STEPS, CFG2_STEPS, CFG2_REF_STEPS = 3, 200, 10


def sent_problem(pkg, spec, device=None, dtype=None):
    """The structured-Q4 SENT setup of ``spec`` built with package ``pkg`` (this one or the reference):
    bottom fixed and top loaded (cfg0) or free edges with a +-1 MPa edge traction on f_ext (cfg2), the
    crack as phase-field Dirichlet d = 1 on the node line."""
    kw = {} if device is None else {"device": device}
    if pkg.__name__ == "phast":
        from phast.core.mesh import FEMMesh
        from phast.core.quad_elements import structured_q4_mesh
        from phast.physics.boundary_conditions import BoundaryConditions
        from phast.physics.material import Material
        from phast.solvers.staggered_solver import SolverConfig, StaggeredSolver
    else:
        FEMMesh, structured_q4_mesh, BoundaryConditions = pkg.FEMMesh, pkg.structured_q4_mesh, pkg.BoundaryConditions
        Material, SolverConfig, StaggeredSolver = pkg.Material, pkg.SolverConfig, pkg.StaggeredSolver
    sm = structured_q4_mesh(spec["width"], spec["height"], spec["nx"], spec["ny"])
    mesh = FEMMesh.from_tensors(sm.nodes, sm.quads, element_type="Q4", **kw)
    bcs = BoundaryConditions(mesh.n_nodes, **kw)
    if spec["bc"]:
        bcs.fix(sm.node_sets["bottom"], 0)
        bcs.fix(sm.node_sets["bottom"], 1)
        bcs.add(sm.node_sets["top"], 1, 1.0)
    nodes = sm.nodes.cpu().numpy()
    notch = np.nonzero((np.abs(nodes[:, 1] - spec["crack_y"]) < 1e-9 * spec["height"]) &
                       (nodes[:, 0] < spec["crack_x"]))[0]
    bcs.add_pf_dirichlet(torch.as_tensor(notch), 1.0)
    cfg = dict(spec["cfg"])
    if dtype is not None:
        cfg["dtype"] = dtype
    s = StaggeredSolver(mesh, Material(**spec["mat"]), bcs, SolverConfig(**cfg))
    pf_mask, pf_vals = bcs.get_pf_dirichlet_mask_values()
    s.d = torch.where(pf_mask, pf_vals.to(s.d.device), s.d)
    if not spec["bc"]:
        f_ext = np.zeros((mesh.n_nodes, 2))
        hx = spec["width"] / spec["nx"]
        for name, sign in (("top", 1.0), ("bottom", -1.0)):
            ns = sm.node_sets[name].cpu().numpy()
            ns = ns[np.argsort(nodes[ns, 0])]
            w = np.full(len(ns), hx)
            w[0] = w[-1] = hx / 2
            f_ext[ns, 1] = sign * w
        s.f_ext = torch.as_tensor(f_ext, dtype=s.u.dtype, device=s.u.device)
    return s, sm, bcs


def _time_2d(s, bcs, steps, load=None, flush=None):
    """Device time of ``steps`` staggered steps (CUDA events per step); damage PCG iterations."""
    ms, pf, stag = 0.0, 0, 0
    for k in range(steps):
        if load is not None:
            bcs.load_factor = load(k + 1)
        if flush is not None:
            flush_l2(flush)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        s.step_full()
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
        pf += s.damage_solver.last_iter
        stag += s._last_stagger_iter
    return ms, pf, stag


def _time_reference_2d(spec, steps, load=None):
    import_reference()
    import phast
    torch.set_num_threads(os.cpu_count() or 1)
    s, sm, bcs = sent_problem(phast, spec)
    secs = []
    for k in range(steps):
        if load is not None:
            bcs.load_factor = load(k + 1)
        t0 = time.perf_counter()
        s.step_full()
        secs.append(time.perf_counter() - t0)
    return secs, torch.get_num_threads()


def run_2d_configs(device, flush, with_cpu):
    """Bench lines of cfg0 and cfg2 (steps/s, DOF-updates/s, achieved GB/s of the algorithmic bytes)."""
    import phast_b200 as pb
    out = {}
    peak, _ = peaks()
    # cfg0: every load step is a full staggered solve (Newton-CG mechanics, projected-CG damage), FP64
    load0 = lambda k: 0.007 * k / 100  # noqa: E731
    s, sm, bcs = sent_problem(pb, CFG0, device=device)
    _time_2d(s, bcs, 1, load0)  # warm-up step (workspaces), then the timed window from the start
    s, sm, bcs = sent_problem(pb, CFG0, device=device)
    ms, pf, stag = _time_2d(s, bcs, CFG0_STEPS, load0, flush)
    N, E = s.fem.n_nodes, s.fem.n_elems
    line = {"workload": "2D quasi-static SENT, Q4 200x200, isotropic split, CG and projected-CG tol 1e-10; "
                        f"load steps 1..{CFG0_STEPS} of 100", "dtype": "f64",
            "value": CFG0_STEPS / (ms / 1e3), "unit": "staggered steps/s", "ms_per_step": ms / CFG0_STEPS,
            "stagger_iters_per_step": stag / CFG0_STEPS, "damage_pcg_iters_per_step": pf / CFG0_STEPS}
    if with_cpu:
        try:
            secs, threads = _time_reference_2d(CFG0, 1, load0)
            line["cpu_baseline"] = {"value": 1.0 / secs[0], "unit": "staggered steps/s", "cores": threads,
                                    "kind": "reference",
                                    "sample": f"PhAST {PHAST_VERSION} StaggeredSolver.step_full, load step 1 "
                                              f"({secs[0]:.1f} s)"}
        except ImportError as exc:
            line["cpu_baseline"] = {"value": None, "sample": f"unavailable: {exc}"}
    out["cfg0"] = line
    # cfg2: explicit steps, FP32 fields and kernels (the configuration's form) beside plain FP64
    res = {}
    for name, dt in (("fp32", torch.float32), ("fp64", torch.float64)):
        s, sm, bcs = sent_problem(pb, CFG2, device=device, dtype=dt)
        _time_2d(s, bcs, 5)
        s, sm, bcs = sent_problem(pb, CFG2, device=device, dtype=dt)
        ms, pf, _ = _time_2d(s, bcs, CFG2_STEPS)
        res[name] = (ms, pf, s)
    (ms32, pf32, s32), (ms64, pf64, s64) = res["fp32"], res["fp64"]
    N, E = s32.fem.n_nodes, s32.fem.n_elems
    # explicit step (read u, v, a, f_ext, M^-1, d; write u, v, a; H read + write) and one projected-CG
    # iteration of the damage solve (FP64) per damage PCG iteration
    bytes32 = CFG2_STEPS * ((16 * N + 8 * E) * 4) + pf32 * (8 * N + 4 * E) * 8
    bytes64 = CFG2_STEPS * ((16 * N + 8 * E) * 8) + pf64 * (8 * N + 4 * E) * 8
    rel = lambda a, b: float(torch.linalg.vector_norm(a.double() - b.double()) / torch.linalg.vector_norm(b.double()))  # noqa: E731
    line = {"workload": f"2D explicit crack branching, Q4 400x160, spectral split, damage solve every step; "
                        f"steps 1..{CFG2_STEPS}", "dtype": "f32 fields/kernels, f64 damage solve",
            "value": CFG2_STEPS / (ms32 / 1e3), "unit": "time steps/s", "ms_per_step": ms32 / CFG2_STEPS,
            "dof_updates_per_s": (2 * N * CFG2_STEPS + N * pf32) / (ms32 / 1e3),
            "achieved_GBps": bytes32 / (ms32 / 1e3) / 1e9, "hbm_frac": bytes32 / (ms32 / 1e3) / 1e9 / peak,
            "l2": "working set (about 10 MB) is L2-resident",
            "plain_fp64": {"value": CFG2_STEPS / (ms64 / 1e3), "ms_per_step": ms64 / CFG2_STEPS,
                           "achieved_GBps": bytes64 / (ms64 / 1e3) / 1e9},
            "speedup_vs_plain_fp64": ms64 / ms32,
            "rel_err_fp32_vs_fp64": {"u": rel(s32.u, s64.u), "v": rel(s32.v, s64.v), "d": rel(s32.d, s64.d),
                                     "crack_support_equal": bool(torch.equal(s32.d > 0.9, s64.d > 0.9))},
            "damage_pcg_iters_per_step": pf32 / CFG2_STEPS}
    if with_cpu:
        try:
            secs, threads = _time_reference_2d(CFG2, CFG2_REF_STEPS)
            line["cpu_baseline"] = {"value": len(secs) / sum(secs), "unit": "time steps/s", "cores": threads,
                                    "kind": "reference",
                                    "sample": f"PhAST {PHAST_VERSION} StaggeredSolver.step_full (FP64), steps "
                                              f"1..{len(secs)} ({sum(secs):.1f} s)"}
        except ImportError as exc:
            line["cpu_baseline"] = {"value": None, "sample": f"unavailable: {exc}"}
    out["cfg2"] = line
    return out


CFG3_INCREMENTS = 2
CFG4 = dict(CFG0, nx=256, ny=256)
CFG4_STEPS, CFG4_TOTAL, CFG4_CHECKPOINT = 10, 50, 10


def lognormal_gc(nx, ny, mean=2.7, cov=0.2, corr=4.0, seed=0):
    """Seeded lognormal per-element Gc field (element e = j nx + i): a Gaussian field with a
    squared-exponential correlation of length ``corr`` elements (white noise filtered in Fourier
    space), mapped to the lognormal with the given mean and coefficient of variation."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((ny, nx))
    kx, ky = np.fft.fftfreq(nx), np.fft.fftfreq(ny)
    spec = np.exp(-2.0 * np.pi ** 2 * corr ** 2 * (kx[None, :] ** 2 + ky[:, None] ** 2))
    g = np.real(np.fft.ifft2(np.fft.fft2(w) * np.sqrt(spec)))
    g = (g - g.mean()) / g.std()
    s2 = np.log1p(cov ** 2)
    return np.exp(np.log(mean) - 0.5 * s2 + np.sqrt(s2) * g).reshape(-1)


def run_cfg4(device, steps=CFG4_STEPS, with_cpu=False):
    """Bench line of cfg4: d(peak reaction)/d(Gc field) of the 256 x 256 SENT run through the
    hand-written reverse pass (checkpoint every 10 load steps), on load steps 1..steps of 50."""
    import phast_b200 as pb
    from phast_b200.adjoint2d import PeakReactionGradient
    load = lambda k: 0.007 * k / CFG4_TOTAL  # noqa: E731
    gc = torch.as_tensor(lognormal_gc(CFG4["nx"], CFG4["ny"]), device=device)
    # warm-up on two steps (workspaces), then the timed forward and gradient from the initial state
    s, sm, bcs = sent_problem(pb, CFG4, device=device)
    # adjoint stiffness and damage solves to 1e-8 relative: the cracked 256 x 256 stiffness (residual
    # stiffness 1e-8 on the notch) does not reach 1e-10 within the stiffness solve's refinement budget
    rtol = 1e-8
    PeakReactionGradient(s, sm.node_sets["top"], load, 2, checkpoint_every=CFG4_CHECKPOINT,
                         adjoint_rtol=rtol).gradient(gc)
    s, sm, bcs = sent_problem(pb, CFG4, device=device)
    pr = PeakReactionGradient(s, sm.node_sets["top"], load, steps, checkpoint_every=CFG4_CHECKPOINT,
                              adjoint_rtol=rtol)
    torch.cuda.synchronize()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record()
    pr.forward(gc)
    e1.record()
    res = pr.gradient(gc)
    e2.record()
    torch.cuda.synchronize()
    fwd_ms, grad_ms = e0.elapsed_time(e1), e1.elapsed_time(e2)
    g = res.grad
    return {"workload": f"2D quasi-static SENT, Q4 256x256, isotropic split, lognormal Gc field (mean 2.7, CoV 0.2, "
                        f"correlation 4 elements, seed 0); d(peak reaction)/d(Gc) over load steps 1..{steps} of "
                        f"{CFG4_TOTAL}, checkpoint every {CFG4_CHECKPOINT}",
            "dtype": "f64 (forward and adjoint)", "adjoint_rtol": rtol, "value": steps / (grad_ms / 1e3),
            "unit": "load steps/s (forward with checkpoints + reverse pass)", "gradient_ms": grad_ms,
            "forward_only_ms": fwd_ms, "gradient_over_forward": grad_ms / fwd_ms,
            "objective": float(res.objective), "peak_step": int(res.peak_step),
            "staggered_passes": [int(v) for v in res.passes][:steps],
            "grad_norm": float(torch.linalg.vector_norm(g)), "grad_finite": bool(torch.isfinite(g).all()),
            "check": "central differences (1e-4 relative) and PhAST's autograd gradient in tests/test_gpu_adjoint_qs.py",
            **(_cfg4_reference(load, steps, fwd_ms) if with_cpu else {})}


def _cfg4_reference(load, steps, fwd_ms):
    """The reference's forward quasi-static steps on the same 256 x 256 SENT (uniform Gc, the field's
    mean; its autograd gradient is not timed), load steps 1-2, beside this forward."""
    try:
        secs, threads = _time_reference_2d(CFG4, 2, load)
        ours = steps / (fwd_ms / 1e3)
        return {"cpu_baseline": {
                    "value": len(secs) / sum(secs), "unit": "load steps/s (forward only)", "cores": threads,
                    "kind": "reference",
                    "sample": f"PhAST {PHAST_VERSION} StaggeredSolver.step_full (FP64, torch CPU) on the same mesh "
                              f"with Gc uniform at 2.7, load steps 1-2 ({', '.join(f'{x:.1f}' for x in secs)} s)"},
                "forward_speedup_vs_reference": ours / (len(secs) / sum(secs))}
    except Exception as exc:  # noqa: BLE001
        return {"cpu_baseline": {"value": None, "sample": f"unavailable: {type(exc).__name__}: {exc}"}}


# ---------------------------------------------------------------------------
# the PF-CZM damage law (the reference's default 3D law): a 32^3 pore cell through
# the onset of cracking, beside the reference's own solver on the host cores
# ---------------------------------------------------------------------------

PFCZM_N = 32
PFCZM_TARGETS = (0.004, 0.007, 0.009, 0.0105)
PFCZM_F_MATRIX = 30.0                       # MPa
PFCZM_F_PORE = PFCZM_F_MATRIX * 1e-3        # keeps the pore's a1 equal to the matrix's (E x 1e-6)
PFCZM_CPU_BUDGET_S = 30.0


CLOSURE_TARGETS = (0.006, 0.012)


def reference_law_solver(n, targets, *, pfczm=False, closure=False):
    """The pore cell built with the reference's own classes (phast.solid3d), with the PF-CZM law
    or the crack closure."""
    from phast.solid3d.model import (PHASE_ID, LoadCase, MaterialTable, PhaseMaterial, SolverConfig, VoxelGrid,
                                     VoxelModel)
    from phast.solid3d.operator import PeriodicVoxelPhaseFieldOperator
    from phast.solid3d.staggered import StaggeredSolver
    h = 1.0 / n
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    c = np.stack([(i + 0.5) / n - 0.5, (j + 0.5) / n - 0.5, (k + 0.5) / n - 0.5], -1)
    phase = np.full((n, n, n), PHASE_ID["mi_matrix"], dtype=np.uint8)
    phase[np.linalg.norm(c, axis=-1) < 0.2] = PHASE_ID["pore"]
    fm, fp = (PFCZM_F_MATRIX, PFCZM_F_PORE) if pfczm else (None, None)
    phases = {"mi_matrix": PhaseMaterial(name="mi_matrix", kind="isotropic", Gc=0.5, driver="spectral", E=3000.0,
                                         nu=0.35, tensile_strength=fm),
              "pore": PhaseMaterial(name="pore", kind="isotropic", Gc=0.5, driver="spectral", E=3000.0 * 1e-6,
                                    nu=0.35, tensile_strength=fp)}
    tangent = np.zeros((n, n, n, 3))
    tangent[..., 2] = 1.0
    model = VoxelModel(grid=VoxelGrid(shape=(n, n, n), h=(h, h, h)), phase_id=phase, tangent=tangent,
                       materials=MaterialTable(phases=phases, length_scale=2 * h, scale="micro"))
    load = LoadCase(name="zz", controlled=2, targets=targets, free=(), fixed_zero=(0, 1, 3, 4, 5))
    cfg = SolverConfig(device="cpu", kappa=1e-6, energy_split_isotropic="spectral",
                       damage_law="pfczm" if pfczm else "at2", crack_closure="axes" if closure else "none")
    op = PeriodicVoxelPhaseFieldOperator(model, load, cfg)
    return op, StaggeredSolver(op)


_COUNT_FIELDS = ("stagger_iters", "newton_iters_pf", "closure_solves", "pcg_iters_mech", "pcg_iters_pf",
                 "active_set_iters")


def _counts(rec):
    return {f: getattr(rec, f) for f in _COUNT_FIELDS if getattr(rec, f, None) is not None}


def _run_law_line(device, with_cpu, n, targets, workload, form, *, pfczm=False, closure=False):
    """Whole staggered increments of the pore cell with the PF-CZM law or the crack closure (plain
    FP64 mechanics), and the reference's increments on the host cores with the fields compared where
    both ran."""
    from phast_b200.solid3d import LoadCase, PeriodicVoxelPhaseFieldOperator, SolverConfig, StaggeredSolver
    from phast_b200.solid3d import sphere_pore_model

    from phast_b200.solid3d.staggered import PLAIN

    def build(mech_form=PLAIN):
        model = sphere_pore_model((n, n, n), 0.2, tensile_strength=PFCZM_F_MATRIX if pfczm else None,
                                  pore_tensile_strength=PFCZM_F_PORE if pfczm else None)
        load = LoadCase(name="zz", controlled=2, targets=targets, free=(), fixed_zero=(0, 1, 3, 4, 5))
        cfg = SolverConfig(device=str(device), kappa=1e-6, energy_split_isotropic="spectral",
                           damage_law="pfczm" if pfczm else "at2", crack_closure="axes" if closure else "none")
        op = PeriodicVoxelPhaseFieldOperator(model, load, cfg)
        return op, StaggeredSolver(op, form=mech_form)

    def timed(mech_form=PLAIN):
        # warm-up on a separate solver (workspaces, library init), then the timed increments
        op, solver = build(mech_form)
        st = solver.initial_state()
        for t in targets[:2]:
            st, _ = solver.advance(st, t)
        op, solver = build(mech_form)
        state = solver.initial_state()
        states, recs, ms = [], [], []
        launches0 = _lib_launches()
        for t in targets:
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            state, rec = solver.advance(state, t)
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
            states.append(state)
            recs.append(rec)
        return states, recs, ms, _lib_launches() - launches0

    states, recs, ms, launches = timed()
    line = {"workload": workload, "dtype": "f64", "form": form, "value": len(ms) / (sum(ms) / 1e3),
            "unit": "staggered increments/s", "ms_per_increment": ms, "gpu_launches": int(launches),
            "per_increment": [dict(_counts(r), max_d=r.max_damage) for r in recs]}
    if pfczm:
        # the multigrid and FP32 forms take the PF-CZM g as a Gauss-point field
        chosen = forms()["mixed-gmg"]
        c_states, c_recs, c_ms, c_launches = timed(chosen)
        rel_ = lambda a, b: float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))  # noqa: E731
        line["chosen_form"] = {
            "form": "FP32 PCG + FP32 3-level multigrid under FP64 refinement (PF-CZM g per Gauss point in every "
                    "level), projected Newton damage solve",
            "value": len(c_ms) / (sum(c_ms) / 1e3), "ms_per_increment": c_ms, "gpu_launches": int(c_launches),
            "speedup_vs_plain_fp64": sum(ms) / sum(c_ms),
            "rel_err_vs_plain_fp64": {"x": rel_(c_states[-1].x, states[-1].x), "d": rel_(c_states[-1].d, states[-1].d)},
            "per_increment": [_counts(r) for r in c_recs]}
    if with_cpu:
        try:
            import torch as th
            import_reference()
            threads = os.cpu_count() or 1
            th.set_num_threads(threads)
            rop, rsolver = reference_law_solver(n, targets, pfczm=pfczm, closure=closure)
            rstate = rsolver.initial_state()
            secs, rrecs = [], []
            for t in targets:
                t0 = time.perf_counter()
                rstate, rrec = rsolver.advance(rstate, t)
                secs.append(time.perf_counter() - t0)
                rrecs.append(rrec)
                if sum(secs) + secs[-1] > PFCZM_CPU_BUDGET_S:
                    break
            k = len(secs) - 1
            rel = lambda a, b: float(np.linalg.norm(np.asarray(a) - np.asarray(b)) /  # noqa: E731
                                     max(np.linalg.norm(np.asarray(b)), 1e-300))
            ours_ms = sum(ms[:len(secs)])
            line["cpu_baseline"] = {
                "value": len(secs) / sum(secs), "unit": "staggered increments/s", "cores": th.get_num_threads(),
                "kind": "reference",
                "sample": f"PhAST {PHAST_VERSION} phast.solid3d.StaggeredSolver.advance (FP64, torch CPU) on the same "
                          f"cell, increments 1-{len(secs)} ({', '.join(f'{s:.1f}' for s in secs)} s)"}
            line["speedup_vs_reference_same_increments"] = sum(secs) / (ours_ms / 1e3)
            line["parity_vs_reference"] = {
                "increments": len(secs),
                "reference_per_increment": [_counts(r) for r in rrecs],
                "same_counts": all(_counts(a) == _counts(b) for a, b in zip(recs, rrecs)),
                "rel_err_x": rel(states[k].x.cpu().numpy(), rstate.x.numpy()),
                "rel_err_d": rel(states[k].d.cpu().numpy(), rstate.d.numpy()) if float(rstate.d.abs().max()) > 0
                else float(states[k].d.abs().max()),
                "rel_err_macro_stress": max(rel(a.macro_stress, b.macro_stress) for a, b in zip(recs, rrecs))}
        except Exception as exc:  # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "sample": f"unavailable: {type(exc).__name__}: {exc}"}
    return line


def run_pfczm(device, with_cpu, n=PFCZM_N):
    """Bench line of the PF-CZM law: increments 1-4 of the pore cell through the onset of cracking."""
    return _run_law_line(
        device, with_cpu, n, PFCZM_TARGETS,
        f"3D periodic pore cell {n}^3 (E 3000, nu 0.35, Gc 0.5, ell 2h, pore E x 1e-6), damage_law 'pfczm' "
        f"(linear softening, f_t {PFCZM_F_MATRIX:g} MPa), spectral split, uniaxial zz strain increments "
        f"{PFCZM_TARGETS}",
        "plain FP64 mechanics (Jacobi PCG, PF-CZM g per Gauss point) + projected Newton damage solve (box-KKT QP "
        "per step)", pfczm=True)


def run_closure(device, with_cpu, n=PFCZM_N):
    """Bench line of the crack closure: AT2 increments of the pore cell with crack_closure 'axes'."""
    return _run_law_line(
        device, with_cpu, n, CLOSURE_TARGETS,
        f"3D periodic pore cell {n}^3 (E 3000, nu 0.35, Gc 0.5, ell 2h, pore E x 1e-6), AT2, spectral split, "
        f"crack_closure 'axes', uniaxial zz strain increments {CLOSURE_TARGETS}",
        "plain FP64 mechanics with the closure add-back (line-searched pattern iteration) + box-KKT damage",
        closure=True)


def _lib_launches():
    from phast_b200 import _lib
    return int(_lib.load().phastb_launch_count())


def run_cfg3_action(device, flush, n_cells=16, brick=(16, 8, 8)):
    """Profiling case of the packed batch: the batched FP32 elastic action of the seeded cells alone,
    beside the same cells' single-cell actions (device time per launch, L2 flushed before each)."""
    from phast_b200.solid3d import batch as bt
    cells = bt.particle_cells(seed=0, n_cells=n_cells)
    load = bt.batch_load()
    ops = [bt.build_operator(c, load, device=device) for c in cells]
    B = bt.PackedCellBatch(ops, brick=brick)
    rng = np.random.default_rng(1)
    x = torch.as_tensor(rng.normal(size=B.n_mech) * 1e-3, device=device).float()
    d = torch.as_tensor(rng.uniform(0, 0.9, size=B.n_nodes), device=device).float()

    def timed(fn, n=5):
        for _ in range(3):
            fn()
        ms = 0.0
        for _ in range(n):
            flush_l2(flush)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1) / n
        return ms

    yb = torch.empty_like(x)
    batched = timed(lambda: B.mech_apply(x, d, out=yb, macro_rows=False))
    xs = [B.mech_view(x, c).clone() for c in range(n_cells)]
    dsv = [B.node_view(d, c).clone() for c in range(n_cells)]
    ys = [torch.empty_like(v) for v in xs]

    def singles():
        for op, xv, dv, yv in zip(ops, xs, dsv, ys):
            op.mech_action(xv, d=dv, out=yv)

    single = timed(singles)
    peak, _ = peaks()
    nbytes = sum(7 * op.n_red * 4 + op.n_elements for op in ops)
    return {"workload": f"batched FP32 elastic action of {n_cells} particle-in-cube cells "
                        f"({sum(op.n_elements for op in ops)} voxels), bricks {brick}",
            "batched_ms": batched, "one_launch_per_cell_ms": single, "algorithmic_bytes": nbytes,
            "batched_GBps": nbytes / (batched / 1e3) / 1e9, "hbm_frac": nbytes / (batched / 1e3) / 1e9 / peak,
            "blocks": B.n_blocks}


def _batch_increments(B, load, cfg, flush, increments, mixed, form, profile=False):
    """Timed load increments 1..K of every cell of a packed batch, after one warm-up increment from a
    separate initial state; returns (ms, records per increment)."""
    from phast_b200.solid3d import batch as bt
    solver = bt.BatchStaggeredSolver(B, load, cfg, mixed=mixed, form=form)
    solver.advance(solver.initial_state(), load.targets[0])
    torch.cuda.synchronize()
    solver = bt.BatchStaggeredSolver(B, load, cfg, mixed=mixed, form=form)
    state = solver.initial_state()
    total_ms, recs = 0.0, []
    if profile:  # brackets the timed increments for a profiler started with --profile-from-start off
        torch.cuda.profiler.start()
    for k in range(increments):
        flush_l2(flush)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        state, r = solver.advance(state, load.targets[k])
        e1.record()
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1)
        recs.append(r)
    if profile:
        torch.cuda.profiler.stop()
    return total_ms, recs, state


def _one_cell_at_a_time(ops, load, cfg, form, increments):
    """The same increments with the single-cell solver, one cell after the other (each cell warmed up
    on its own first increment); returns (ms, last record per cell)."""
    from phast_b200.solid3d.staggered import StaggeredSolver
    ms, last = 0.0, []
    for op in ops:
        sv = StaggeredSolver(op, cfg=cfg, form=form)
        sv.advance(sv.initial_state(), load.targets[0])
        sv = StaggeredSolver(op, cfg=cfg, form=form)
        st1 = sv.initial_state()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in range(increments):
            st1, r1 = sv.advance(st1, load.targets[k])
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
        last.append(r1)
    return ms, last


CFG3_CPU_BUDGET_S = 40.0


def reference_cfg3_cells(cells, load, increments, budget_s):
    """The reference's solid3d solver on one batch cell per edge size (smallest first), whole
    increments 1..K, until the budget is spent.  Returns [(N, seconds per increment)]."""
    import torch as th
    import_reference()
    from phast.solid3d.model import (PHASE_ID, LoadCase, MaterialTable, PhaseMaterial, SolverConfig, VoxelGrid,
                                     VoxelModel)
    from phast.solid3d.operator import PeriodicVoxelPhaseFieldOperator
    from phast.solid3d.staggered import StaggeredSolver
    from phast_b200.solid3d import batch as bt
    th.set_num_threads(os.cpu_count() or 1)
    names = [p.name for p in bt.BATCH_PHASES]
    ids = np.array([PHASE_ID[nm] for nm in names], dtype=np.uint8)
    phases = {p.name: PhaseMaterial(name=p.name, kind="isotropic", Gc=p.Gc, driver="spectral", E=p.E, nu=p.nu)
              for p in bt.BATCH_PHASES}
    ref_load = LoadCase(name=load.name, controlled=load.controlled, targets=tuple(load.targets),
                        free=tuple(load.free), fixed_zero=tuple(load.fixed_zero))
    out, spent = [], 0.0
    for n in sorted({c.n for c in cells}):
        cell = next(c for c in cells if c.n == n)
        h = 1.0 / n
        tangent = np.zeros((n, n, n, 3))
        tangent[..., 2] = 1.0
        model = VoxelModel(grid=VoxelGrid(shape=(n, n, n), h=(h, h, h)), phase_id=ids[cell.phase], tangent=tangent,
                           materials=MaterialTable(phases=phases, length_scale=2 * h, scale="micro"))
        cfg = SolverConfig(device="cpu", kappa=1e-6, energy_split_isotropic="spectral")
        solver = StaggeredSolver(PeriodicVoxelPhaseFieldOperator(model, ref_load, cfg))
        state = solver.initial_state()
        secs = []
        for k in range(increments):
            t0 = time.perf_counter()
            state, _ = solver.advance(state, ref_load.targets[k])
            secs.append(time.perf_counter() - t0)
        out.append((n, sum(secs) / len(secs)))
        spent += sum(secs)
        if spent + 8.0 * out[-1][1] * increments > budget_s:  # the next size takes about twice as long
            break
    return out, th.get_num_threads()


def run_cfg3(device, flush, n_cells=128, increments=CFG3_INCREMENTS, per_cell=True, with_cpu=False):
    """Bench line of cfg3: the seeded particle-in-cube batch advanced as one packed batch (every
    cell in one launch per operator apply, per multigrid step and per Krylov vector step), load
    increments 1..K of every cell from the initial state; beside the batch with Jacobi PCG and
    the same cells advanced one at a time by the single-cell solver (same multigrid form, and the
    plain FP64 form)."""
    from phast_b200.solid3d import batch as bt
    from phast_b200.solid3d.model import SolverConfig
    from phast_b200.solid3d.staggered import PLAIN
    peak, _ = peaks()
    cells = bt.particle_cells(seed=0, n_cells=n_cells)
    load = bt.batch_load()
    ops = [bt.build_operator(c, load, device=device) for c in cells]
    B = bt.PackedCellBatch(ops, brick=(16, 8, 8))
    cfg = SolverConfig(kappa=ops[0].kappa)
    gmg = forms()["mixed-gmg"]
    total_ms, recs, state = _batch_increments(B, load, cfg, flush, increments, True, gmg, profile=True)
    jac_ms, jac_recs, _ = _batch_increments(B, load, cfg, flush, increments, True, None)
    voxels = sum(op.n_elements for op in ops)
    mech_its = sum(r.pcg_iters_mech for rr in recs for r in rr)
    pf_its = sum(r.pcg_iters_pf for rr in recs for r in rr)
    dof_updates = sum((r.pcg_iters_mech * op.n_mech + r.pcg_iters_pf * op.n_red) for rr in recs
                      for r, op in zip(rr, ops))
    # the batched FP32 elastic action alone (the dominant kernel of the batch), L2 flushed
    x32 = state.x.float().contiguous()
    d32 = state.d.float().contiguous()
    y32 = torch.empty_like(x32)
    for _ in range(3):
        B.mech_apply(x32, d32, out=y32, macro_rows=False)
    act_ms = 0.0
    for _ in range(10):
        flush_l2(flush)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        B.mech_apply(x32, d32, out=y32, macro_rows=False)
        e1.record()
        torch.cuda.synchronize()
        act_ms += e0.elapsed_time(e1) / 10
    act_bytes = sum(7 * op.n_red * 4 + op.n_elements for op in ops)
    rate = lambda ms: n_cells * increments / (ms / 1e3)  # noqa: E731

    def worst_err(a_recs, b_recs):
        w = 0.0
        for a, b in zip(a_recs, b_recs):
            a, b = np.asarray(a.macro_stress), np.asarray(b.macro_stress)
            w = max(w, float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)))
        return w

    line = {"workload": f"{n_cells} seeded periodic particle-in-cube cells (edge N in {{32,40,48,56,64}}, "
                        f"{voxels} voxels in all), eps_xx ramp 0 -> 0.015 over 40 steps; increments 1..{increments} "
                        "of every cell as one packed batch: FP32 PCG with the batched 3-level multigrid V-cycle "
                        "(FP64 dots) under FP64 refinement, FP64 box-KKT damage",
            "dtype": "f32 mechanics (f64 dots, f64 refinement), f64 damage",
            "value": rate(total_ms), "unit": "cell increments/s",
            "ms_per_batch_increment": total_ms / increments,
            "dof_updates_per_s": dof_updates / (total_ms / 1e3),
            "mech_iters_per_cell_increment": mech_its / (n_cells * increments),
            "damage_pcg_iters_per_cell_increment": pf_its / (n_cells * increments),
            "batched_jacobi": {"value": rate(jac_ms), "ms_per_batch_increment": jac_ms / increments,
                               "mech_iters_per_cell_increment":
                                   sum(r.pcg_iters_mech for rr in jac_recs for r in rr) / (n_cells * increments)},
            "batched_action": {"kernel": "h8_tile_batch_kernel<float> (every cell in one launch)",
                               "launch_ms": act_ms, "algorithmic_bytes": act_bytes,
                               "achieved_GBps": act_bytes / (act_ms / 1e3) / 1e9,
                               "hbm_frac": act_bytes / (act_ms / 1e3) / 1e9 / peak,
                               "l2": "working set beyond the 126 MB L2"}}
    if per_cell:
        one_ms, one_last = _one_cell_at_a_time(ops, load, cfg, gmg, increments)
        plain_ms, plain_last = _one_cell_at_a_time(ops, load, cfg, PLAIN, increments)
        line["one_cell_at_a_time"] = {"form": "the same multigrid form, single-cell solver", "value": rate(one_ms),
                                      "ms_per_batch_increment": one_ms / increments}
        line["plain_fp64_one_cell_at_a_time"] = {"form": "plain FP64 (Jacobi PCG), single-cell solver",
                                                 "value": rate(plain_ms), "ms_per_batch_increment": plain_ms / increments}
        line["speedup_vs_one_cell_at_a_time"] = one_ms / total_ms
        line["speedup_vs_plain_fp64"] = plain_ms / total_ms
        line["rel_err_macro_stress_vs_plain_fp64"] = worst_err(recs[-1], plain_last)
        line["rel_err_macro_stress_jacobi_vs_plain_fp64"] = worst_err(jac_recs[-1], plain_last)
    if with_cpu:
        try:
            per_size, threads = reference_cfg3_cells(cells, load, increments, CFG3_CPU_BUDGET_S)
            ref_rate = len(per_size) / sum(t for _, t in per_size)  # cell increments/s over the sampled cells
            line["cpu_baseline"] = {
                "value": ref_rate, "unit": "cell increments/s", "cores": threads, "kind": "reference",
                "sample": f"PhAST {PHAST_VERSION} phast.solid3d.StaggeredSolver.advance (FP64, torch CPU) on one "
                          f"batch cell per edge size, smallest first, increments 1-{increments}: "
                          + ", ".join(f"N={n}: {t:.1f} s per increment" for n, t in per_size)
                          + " (the larger cells are slower, so the batch's true reference rate is lower)"}
            line["speedup_vs_reference_lower_bound"] = line["value"] / ref_rate
        except Exception as exc:  # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "sample": f"unavailable: {type(exc).__name__}: {exc}"}
    return line


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def forms():
    from phast_b200.solid3d import MechForm
    # the chosen form's V-cycle (one Chebyshev step per smoothing on the fine and middle levels,
    # degree 6 on the coarsest) and inner tolerance came from a sweep on increments 1-20 of this cell
    return {"plain": MechForm(), "gmg": MechForm(precond="gmg"), "mixed": MechForm(mixed=True),
            "mixed-gmg": MechForm(precond="gmg", mixed=True, smooth_degree=1, coarse_degree=6, inner_rtol=1e-5)}


FORM_LABEL = {
    "plain": "plain FP64: Jacobi PCG (PhAST's algorithm), FP64 box-KKT damage",
    "gmg": "FP64 PCG with a 3-level voxel multigrid V-cycle (Chebyshev deg 2, coarse deg 8)",
    "mixed": "FP32 Jacobi PCG (FP64 dots) under FP64 iterative refinement",
    "mixed-gmg": "FP32 PCG with an FP32 3-level multigrid V-cycle (Chebyshev degree 1 / coarse 6; FP64 dots) under "
                 "FP64 iterative refinement; FP64 box-KKT damage",
}


def run_steps(op, form, steps, flush, clocks=None):
    """Timed staggered increments 1..steps from the initial state; device time per step with CUDA events."""
    from phast_b200.solid3d import StaggeredSolver
    solver = StaggeredSolver(op, form=form)
    state = solver.initial_state()
    torch.cuda.synchronize()
    if clocks is not None:
        clocks.start()
    total_ms, counts = 0.0, []
    for _ in range(steps):
        flush_l2(flush)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        state, rec = solver.advance(state, op.load.targets[state.increment])
        e1.record()
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1)
        counts.append((rec.pcg_iters_mech, rec.pcg_iters_pf, rec.stagger_iters))
    clk = clocks.stop() if clocks is not None else None
    return total_ms, state, counts, clk


def run_ours(args, rank, world, device):
    from phast_b200 import _lib
    from phast_b200.solid3d import SolverState, StaggeredSolver
    fm = forms()
    chosen = fm[args.form]
    op, solver = build_cell(device)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=device)  # 256 MB > 126 MB L2
    # warm-up: W increments of the plain FP64 form and one of the chosen form, each from the
    # initial state (workspaces, graphs and kernels); the timed runs start from the initial
    # state again, so every arm times load increments 1..K of the same path
    state = solver.initial_state()
    for _ in range(args.warmup):
        state, _ = solver.advance(state, op.load.targets[state.increment])
    torch.cuda.synchronize()
    run_steps(op, chosen, 1, flush)

    # ---- chosen form, device-resident timed region -----------------------------------
    lib = _lib.load()
    if world > 1:
        torch.distributed.barrier()
    lib.phastb_launch_count_reset()
    clocks = Clocks(torch.cuda.current_device())
    # brackets the timed steps for a profiler started with --profile-from-start off (no-op otherwise)
    torch.cuda.profiler.start()
    total_ms, st_c, counts, clk = run_steps(op, chosen, args.steps, flush, clocks)
    torch.cuda.profiler.stop()
    launches = lib.phastb_launch_count()
    t = torch.tensor([total_ms], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.barrier()
    max_ms = float(t.item())
    value = args.steps * world / (max_ms / 1e3)

    # ---- plain FP64 form on the same increments (the comparison of the metric) --------
    plain_ms, st_p, counts_p, _ = run_steps(op, fm["plain"], args.steps, flush)
    tp = torch.tensor([plain_ms], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(tp, op=torch.distributed.ReduceOp.MAX)
    plain_value = args.steps * world / (float(tp.item()) / 1e3)

    def relerr(a, b):
        nb = float(torch.linalg.vector_norm(b))
        return float(torch.linalg.vector_norm(a - b)) / (nb if nb > 0 else 1.0)

    err = {"x": relerr(st_c.x, st_p.x), "d": relerr(st_c.d, st_p.d),
           "macro_stress": float(np.linalg.norm((st_c.macro_stress - st_p.macro_stress).numpy()) /
                                 max(float(np.linalg.norm(st_p.macro_stress.numpy())), 1e-300)),
           "crack_support_equal": bool(torch.equal(st_c.d > 0.9, st_p.d > 0.9))}

    # ---- end to end through the public API with host buffers ---------------------------
    # every step copies the state in from pinned host memory, advances one increment and
    # copies the new state out (x, d, H; the lower bound d_prev_step is the incoming d)
    solver_c = StaggeredSolver(op, form=chosen)
    init = solver_c.initial_state()
    host_state = {k: getattr(init, k).detach().cpu().pin_memory() for k in ("x", "d", "H")}
    pinned_out = {k: torch.empty_like(v).pin_memory() for k, v in host_state.items()}
    dev_in = {k: torch.empty(v.shape, dtype=v.dtype, device=device) for k, v in host_state.items()}
    h2d = sum(v.numel() * v.element_size() for v in host_state.values())
    meta = (init.step, init.macro_strain, init.macro_stress, init.external_work, init.increment)
    e2e_ms = 0.0
    for _ in range(args.steps):
        flush_l2(flush)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in dev_in:
            dev_in[k].copy_(host_state[k], non_blocking=True)
        s_in = SolverState(meta[0], dev_in["x"].clone(), dev_in["d"].clone(), dev_in["H"].clone(), meta[1].clone(),
                           meta[2].clone(), meta[3], dev_in["d"].clone(), meta[4])
        s_out, _ = solver_c.advance(s_in, op.load.targets[s_in.increment])
        for k in pinned_out:
            pinned_out[k].copy_(getattr(s_out, k), non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        e2e_ms += e0.elapsed_time(e1)
        host_state = {k: v.clone().pin_memory() for k, v in pinned_out.items()}
        meta = (s_out.step, s_out.macro_strain, s_out.macro_stress, s_out.external_work, s_out.increment)
    te = torch.tensor([e2e_ms], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(te, op=torch.distributed.ReduceOp.MAX)
    e2e_value = args.steps * world / (float(te.item()) / 1e3)

    # ---- dominant kernel: the elastic action (element kernel + node gather) ------------
    mixed = chosen.mixed
    kdt = torch.float32 if mixed else torch.float64
    x, d = st_c.x.to(kdt).contiguous(), st_c.d.to(kdt).contiguous()
    apply_s = time_action(op, x, d, flush)
    wsz = 4 if mixed else 8
    alg_bytes = 7 * op.n_red * wsz + op.n_elements * 1  # read u~ 3n, d n; write 3n; slot id per voxel
    peak, peak_src = peaks()
    achieved = alg_bytes / apply_s / 1e9
    # the same kernel on a cell whose working set exceeds L2 (HBM-bound regime)
    big, _ = build_cell(device, N_LARGE)
    xb = torch.as_tensor(np.random.default_rng(1).normal(size=big.n_mech) * 1e-3, device=device).to(kdt)
    db = torch.as_tensor(np.random.default_rng(2).uniform(0, 0.9, size=big.n_red), device=device).to(kdt)
    big_s = time_action(big, xb, db, flush)
    big_bytes = 7 * big.n_red * wsz + big.n_elements
    del big, xb, db
    mech = float(np.mean([c[0] for c in counts]))
    pf = float(np.mean([c[1] for c in counts]))
    stag = float(np.mean([c[2] for c in counts]))
    mech_p = float(np.mean([c[0] for c in counts_p]))
    dof_updates = (mech * op.n_mech + pf * op.n_red) * args.steps * world / (max_ms / 1e3)
    cfg = workload_config()
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (f64 dots, f64 refinement)" if mixed else "f64", "data": "synthetic", "config": cfg,
        "form": FORM_LABEL[args.form],
        "plain_fp64": {"value": plain_value, "unit": UNIT, "ms_per_step": float(tp.item()) / args.steps,
                       "mech_iters_per_step": mech_p},
        "speedup_vs_plain_fp64": value / plain_value,
        "rel_err_vs_plain_fp64": err,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": profile_traffic(mixed),
                     "kernel": f"h8 elastic action (tiled z-marching, fused g(d)), {'FP32' if mixed else 'FP64'}",
                     "note": "64^3 working set is L2-resident; HBM fraction of the large cell in roofline_large",
                     "algorithmic_bytes": alg_bytes, "launch_ms": apply_s * 1e3, "peak_source": peak_src},
        "roofline_large": {"bound": "hbm", "cell": f"{N_LARGE}^3", "achieved": big_bytes / big_s / 1e9, "peak": peak,
                           "unit": "GB/s", "frac": big_bytes / big_s / 1e9 / peak, "algorithmic_bytes": big_bytes,
                           "launch_ms": big_s * 1e3},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d},
        "gpu_launches": int(launches),
        "clocks": clk,
        "iterations_per_step": {"mech": mech, "pf": pf, "stagger": stag},
        "dof_updates_per_s": dof_updates,
    }
    if not args.no_2d:
        out["configs"] = run_2d_configs(device, flush, world == 1 and rank == 0 and not args.no_cpu)
    # the packed-batch (cfg3) and gradient (cfg4) lines; a failure there is reported in its line
    # and does not cost the headline
    if args.cfg3_cells > 0:
        try:
            out.setdefault("configs", {})["cfg3"] = run_cfg3(device, flush, n_cells=args.cfg3_cells,
                                                             with_cpu=world == 1 and rank == 0 and not args.no_cpu)
        except Exception as exc:  # noqa: BLE001
            out.setdefault("configs", {})["cfg3"] = {"error": f"{type(exc).__name__}: {exc}"}
    if not args.no_2d:
        try:
            out.setdefault("configs", {})["cfg4"] = run_cfg4(device, with_cpu=world == 1 and rank == 0 and not args.no_cpu)
        except Exception as exc:  # noqa: BLE001
            out.setdefault("configs", {})["cfg4"] = {"error": f"{type(exc).__name__}: {exc}"}
    if not args.no_2d:
        for key, fn in (("pfczm", run_pfczm), ("closure", run_closure)):
            try:
                out.setdefault("configs", {})[key] = fn(device, world == 1 and rank == 0 and not args.no_cpu)
            except Exception as exc:  # noqa: BLE001
                out.setdefault("configs", {})[key] = {"error": f"{type(exc).__name__}: {exc}"}
    if world == 1 and rank == 0 and not args.no_cpu:
        try:
            secs, threads, recs = time_reference(args.steps, CPU_BASELINE_BUDGET_S)
            out["cpu_baseline"] = {"value": len(secs) / sum(secs), "unit": UNIT, "cores": threads,
                                   "kind": "reference", "sample": reference_sample_note(secs, recs, threads)}
        except ImportError as exc:
            out["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                                   "sample": f"unavailable: {exc}"}
    return out


def time_action(op, x, d, flush, n_rep=20):
    """Mean device time of one elastic action (CUDA events on the launching stream, L2 flushed before each),
    with the tile shape the solver uses for this grid."""
    y = torch.empty_like(x)
    for _ in range(3):
        op.mech_action(x, d=d, out=y)
    ms = 0.0
    for _ in range(n_rep):
        flush_l2(flush)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        op.mech_action(x, d=d, out=y)
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
    return ms / n_rep / 1e3


def profile_traffic(fp32):
    """DRAM bytes per 64^3 launch of the elastic action from the committed ncu summary, if any."""
    key = "traffic_bytes_per_apply_64_fp32:" if fp32 else "traffic_bytes_per_apply_64_fp64:"
    try:
        for name in sorted(os.listdir(os.path.join(ROOT, "profiles"))):
            with open(os.path.join(ROOT, "profiles", name)) as f:
                for line in f:
                    if line.startswith(key):
                        return float(line.split(":")[1])
    except OSError:
        pass
    return None


def run_reference(args, rank, world):
    """PhAST's own solver on the host cores: whole increments 1..m (m <= K within the budget)."""
    try:
        secs, threads, recs = time_reference(args.steps, REF_BUDGET_S, warmup=args.warmup)
    except ImportError as exc:
        return {"impl": "reference", "unavailable": str(exc)}
    total = sum(secs)
    value = len(secs) / total
    cfg = workload_config()
    sample = reference_sample_note(secs, recs, threads)
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": len(secs),
        "warmup": args.warmup, "ms_per_step": total * 1e3 / len(secs), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
        "impl": "reference", "form": "PhAST's own solver: FP64 Jacobi PCG mechanics, FP64 box-KKT damage (torch CPU)",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "timed_increments": {"requested": args.steps, "timed": len(secs), "budget_s": REF_BUDGET_S,
                             "seconds": secs},
    }


def run_damage_cg_only(args, device):
    """Box-KKT damage solves only (the persistent damage CG), on an N^3 cell with a
    seeded history field: the profiling case of h8_damage_pcg_kernel."""
    from phast_b200 import solid3d as s3
    op, _ = build_cell(device, args.cell)
    gen = torch.Generator(device="cpu").manual_seed(0)
    H = (torch.rand(op.n_elements, 8, generator=gen, dtype=torch.float64) * 50.0).to(device)
    lower = torch.zeros(op.n_red, dtype=torch.float64, device=device)
    system = op.damage_system(H)

    def solve():
        return s3.solve_h8_scalar_box_kkt(system, lower_bound=lower, upper_bound=1.0, initial=lower,
                                          linear_tolerance=1e-10, kkt_tolerance=1e-8, check_bounds=False)
    for _ in range(args.warmup):
        res = solve()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        res = solve()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    its = res.total_pcg_iterations
    # per CG iteration: z, p read and Ap, p written (action), x, p, r, Ap, 1/diag read and x, r, z
    # written (update): 12 n words, plus the history (8 words) and slot byte of every element
    alg = (12 * op.n_red + 8 * op.n_elements) * 8 + op.n_elements
    print(json.dumps({"kernel": "persistent damage CG (box-KKT)", "cell": args.cell, "ms_per_solve": ms,
                      "cg_iterations": its, "active_set_iterations": res.active_set_iterations,
                      "us_per_cg_iteration": 1e3 * ms / max(its, 1),
                      "algorithmic_GBps": alg * its / ms / 1e6}), flush=True)


def run_kernel_only(args, device):
    """Elastic-action launches only, on an N^3 cell (the profiling case for ncu)."""
    op, _ = build_cell(device, args.cell)
    rng = np.random.default_rng(0)
    x = torch.as_tensor(rng.normal(size=op.n_mech) * 1e-3, device=device)
    d = torch.as_tensor(rng.uniform(0, 1, size=op.n_red), device=device)
    dt = torch.float32 if args.fp32 else torch.float64
    x, d = x.to(dt), d.to(dt)
    if args.tile:
        op.tile_shape(dt, tuple(int(v) for v in args.tile.split(",")))  # pinned shape
    for _ in range(args.warmup):
        op.mech_action(x, d=d)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        op.mech_action(x, d=d)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    w = 4 if args.fp32 else 8
    alg = 7 * op.n_red * w + op.n_elements
    print(json.dumps({"kernel": "h8 elastic action (tiled)", "cell": args.cell, "dtype": str(dt),
                      "tile": op.tile_shape(dt), "ms_per_apply": ms, "algorithmic_GBps": alg / ms / 1e6}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-2d", action="store_true", help="skip the 2D configuration lines (cfg0, cfg2)")
    ap.add_argument("--form", default="mixed-gmg", choices=["plain", "gmg", "mixed", "mixed-gmg"],
                    help="mechanics form of the timed value (the plain FP64 form is timed beside it)")
    ap.add_argument("--kernel-only", action="store_true", help="time the elastic action alone (profiling case)")
    ap.add_argument("--cell", type=int, default=N_CELL, help="cell edge in voxels for --kernel-only")
    ap.add_argument("--fp32", action="store_true", help="FP32 storage/arithmetic for --kernel-only")
    ap.add_argument("--damage-cg", action="store_true", help="with --kernel-only: time box-KKT damage solves instead")
    ap.add_argument("--tile", default="", help="pin the tile shape ox,oy,kz for --kernel-only (else the solver's shape)")
    ap.add_argument("--cfg3-cells", type=int, default=128, help="cells of the packed-batch line (0: skip it)")
    ap.add_argument("--cfg3-only", action="store_true", help="print the packed-batch line alone")
    ap.add_argument("--cfg3-action", action="store_true", help="time the packed batch's elastic action alone")
    ap.add_argument("--cfg4-only", action="store_true", help="print the gradient line (cfg4) alone")
    ap.add_argument("--pfczm-only", action="store_true", help="print the PF-CZM line alone")
    ap.add_argument("--closure-only", action="store_true", help="print the crack-closure line alone")
    ap.add_argument("--brick", default="16,8,8", help="brick ox,oy,kz of --cfg3-action")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    if args.steps > INCREMENTS or args.warmup > INCREMENTS:
        raise SystemExit(f"steps and warmup must not exceed the {INCREMENTS} increments of the load path")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, rank, world)), flush=True)
        return
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if args.pfczm_only:
        print(json.dumps(run_pfczm(device, not args.no_cpu)), flush=True)
        return
    if args.closure_only:
        print(json.dumps(run_closure(device, not args.no_cpu)), flush=True)
        return
    if args.cfg4_only:
        print(json.dumps(run_cfg4(device, with_cpu=not args.no_cpu)), flush=True)
        return
    if args.cfg3_action:
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=device)
        brick = tuple(int(v) for v in args.brick.split(","))
        print(json.dumps(run_cfg3_action(device, flush, n_cells=args.cfg3_cells, brick=brick)), flush=True)
        return
    if args.cfg3_only:
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=device)
        print(json.dumps(run_cfg3(device, flush, n_cells=args.cfg3_cells, with_cpu=not args.no_cpu)), flush=True)
        return
    if args.kernel_only:
        if args.damage_cg:
            run_damage_cg_only(args, device)
        else:
            run_kernel_only(args, device)
        return
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=device)
    try:
        out = run_ours(args, rank, world, device)
        if rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()

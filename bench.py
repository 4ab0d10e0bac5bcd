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
# Mean per-increment iteration counts of this workload over increments 4..5
# (the default timed window), measured with this repository's CUDA solver on a
# B200; the CPU reference arm scales its timed per-iteration samples by them.
REF_COUNTS = {"mech": 232.5, "pf": 83.0, "stag": 3.0}


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
        "damage": "box-KKT active set + Dirichlet PCG (FP64)", "form": "",
        "l2": "flushed (256 MB write) before every timed step", "parallelism": "replicas",
    }


def build_cell(device, n=None):
    from phast_b200 import solid3d as s3
    n = N_CELL if n is None else n
    h = 1.0 / n
    shape = (n, n, n)
    phase = s3.sphere_pore_phase(shape, 0.2)
    phases = [s3.PhaseMaterial("mi_matrix", 3000.0, 0.35, 0.5), s3.PhaseMaterial("pore", 3000.0 * 1e-6, 0.35, 0.5)]
    load = s3.LoadCase.ramp("zz", 2, 0.02, INCREMENTS)
    op = s3.PeriodicVoxelPhaseFieldOperator(s3.VoxelGrid(shape, (h, h, h)), phase, phases, 2 * h, 1e-6, load,
                                            device=device)
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
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

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
# CPU baseline: the numpy oracle timed on bounded samples of the same cell
# ---------------------------------------------------------------------------

def cpu_per_iteration_costs(threads_note=True):
    """Seconds per mechanics PCG iteration, per damage PCG iteration and per staggered pass
    of the oracle at full size (64^3); ~10-20 s of CPU work."""
    from oracle import h8
    shape, h = (N_CELL,) * 3, 1.0 / N_CELL
    k, j, i = np.meshgrid(*(np.arange(N_CELL),) * 3, indexing="ij")
    c = np.stack([(i + 0.5) / N_CELL - 0.5, (j + 0.5) / N_CELL - 0.5, (k + 0.5) / N_CELL - 0.5], -1)
    slot = (np.linalg.norm(c, axis=-1) < 0.2).astype(np.int64).reshape(-1)
    C0, l0, m0 = h8.isotropic_C(3000.0, 0.35)
    C1, l1, m1 = h8.isotropic_C(3e-3, 0.35)
    op = h8.VoxelOperator(shape, (h, h, h), slot, np.stack([C0, C1]), np.array([l0, l1]), np.array([m0, m1]),
                          np.array([0.5, 0.5]), np.array([2, 0]), 2 * h, 1e-6, 0, 2, (0, 1, 3, 4, 5))
    rng = np.random.default_rng(0)
    d = rng.uniform(0, 0.5, op.n_red)
    g = op.degradation(d)
    x = rng.normal(size=op.n_mech) * 1e-4
    H = rng.uniform(0, 1, (op.n_elements, 8))
    dg = op.mech_diagonal(g)
    free = ~op.fixed_mask()
    n_it = 4
    t0 = time.perf_counter()
    _, its, _, _, _ = h8.pcg(lambda v: np.where(free, op.mech_action(v, g), 0.0), np.where(free, x, 0.0),
                             np.where(free, dg, 1.0), rtol=1e-30, atol=1e-300, maxiter=n_it, check_every=n_it)
    t_mech = (time.perf_counter() - t0) / n_it
    s = op.damage_scale
    n_it = 10
    t0 = time.perf_counter()
    h8.dirichlet_pcg(lambda v: s * op.damage_action(v, H), s * op.damage_rhs(H), s * op.damage_diagonal(H),
                     np.zeros(op.n_red, bool), np.zeros(op.n_red), None, 1e-300, n_it)
    t_pf = (time.perf_counter() - t0) / n_it
    t0 = time.perf_counter()
    op.degradation(d)
    op.mech_diagonal(g)
    op.driving_force(x)
    op.damage_rhs(H)
    op.damage_diagonal(H)
    t_pass = time.perf_counter() - t0
    return t_mech, t_pf, t_pass


def cpu_step_estimate(counts):
    t_mech, t_pf, t_pass = cpu_per_iteration_costs()
    sec = counts["mech"] * t_mech + counts["pf"] * t_pf + (counts["stag"] + 1) * t_pass
    sample = (f"numpy oracle on the full 64^3 cell: 4 mechanics PCG iterations ({t_mech:.3f} s each), 10 damage "
              f"PCG iterations ({t_pf:.4f} s each), one staggered pass of diagonal/driving/rhs ({t_pass:.2f} s); "
              f"scaled to one step with {counts['mech']:.0f} mechanics + {counts['pf']:.0f} damage iterations "
              f"and {counts['stag']:.1f} staggered passes per increment")
    return sec, sample


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def forms():
    from phast_b200.solid3d import MechForm
    return {"plain": MechForm(), "gmg": MechForm(precond="gmg"), "mixed": MechForm(mixed=True),
            "mixed-gmg": MechForm(precond="gmg", mixed=True)}


FORM_LABEL = {
    "plain": "plain FP64: Jacobi PCG (PhAST's algorithm), FP64 box-KKT damage",
    "gmg": "FP64 PCG with a 3-level voxel multigrid V-cycle (Chebyshev deg 2, coarse deg 8)",
    "mixed": "FP32 Jacobi PCG (FP64 dots) under FP64 iterative refinement",
    "mixed-gmg": "FP32 PCG with an FP32 3-level multigrid V-cycle (FP64 dots) under FP64 iterative refinement; "
                 "FP64 box-KKT damage",
}


def run_steps(op, form, snap, meta, steps, flush, device, clocks=None):
    """Timed staggered increments from a host snapshot; device time per step with CUDA events."""
    from phast_b200.solid3d import SolverState, StaggeredSolver
    solver = StaggeredSolver(op, form=form)
    state = SolverState(meta[0], snap["x"].to(device), snap["d"].to(device), snap["H"].to(device), meta[1].copy(),
                        meta[2].copy(), meta[3])
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
    state = solver.initial_state()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=device)  # 256 MB > 126 MB L2
    for _ in range(args.warmup):  # warm-up increments with the plain FP64 form (same start for both forms)
        state, _ = solver.advance(state, op.load.targets[state.increment])
    torch.cuda.synchronize()
    snap = {k: getattr(state, k).detach().cpu().pin_memory() for k in ("x", "d", "H")}
    meta = (state.step, state.macro_strain.copy(), state.macro_stress.copy(), state.increment)
    # one untimed increment of the chosen form warms its workspaces and kernels
    run_steps(op, chosen, snap, meta, 1, flush, device)

    # ---- chosen form, device-resident timed region -----------------------------------
    lib = _lib.load()
    if world > 1:
        torch.distributed.barrier()
    lib.phastb_launch_count_reset()
    clocks = Clocks(torch.cuda.current_device())
    # brackets the timed steps for a profiler started with --profile-from-start off (no-op otherwise)
    torch.cuda.profiler.start()
    total_ms, st_c, counts, clk = run_steps(op, chosen, snap, meta, args.steps, flush, device, clocks)
    torch.cuda.profiler.stop()
    launches = lib.phastb_launch_count()
    t = torch.tensor([total_ms], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.barrier()
    max_ms = float(t.item())
    value = args.steps * world / (max_ms / 1e3)

    # ---- plain FP64 form on the same increments (the comparison of the metric) --------
    plain_ms, st_p, counts_p, _ = run_steps(op, fm["plain"], snap, meta, args.steps, flush, device)
    tp = torch.tensor([plain_ms], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(tp, op=torch.distributed.ReduceOp.MAX)
    plain_value = args.steps * world / (float(tp.item()) / 1e3)

    def relerr(a, b):
        nb = float(torch.linalg.vector_norm(b))
        return float(torch.linalg.vector_norm(a - b)) / (nb if nb > 0 else 1.0)

    err = {"x": relerr(st_c.x, st_p.x), "d": relerr(st_c.d, st_p.d),
           "macro_stress": float(np.linalg.norm(st_c.macro_stress - st_p.macro_stress) /
                                 max(np.linalg.norm(st_p.macro_stress), 1e-300)),
           "crack_support_equal": bool(torch.equal(st_c.d > 0.9, st_p.d > 0.9))}

    # ---- end to end through the public API with host buffers ---------------------------
    solver_c = StaggeredSolver(op, form=chosen)
    pinned_out = {k: torch.empty_like(v).pin_memory() for k, v in snap.items()}
    dev_in = {k: torch.empty(v.shape, dtype=v.dtype, device=device) for k, v in snap.items()}
    h2d = sum(v.numel() * v.element_size() for v in snap.values())
    st_meta = meta
    e2e_ms = 0.0
    host_state = dict(snap)
    for _ in range(args.steps):
        flush_l2(flush)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in dev_in:
            dev_in[k].copy_(host_state[k], non_blocking=True)
        s_in = SolverState(st_meta[0], dev_in["x"].clone(), dev_in["d"].clone(), dev_in["H"].clone(),
                           st_meta[1].copy(), st_meta[2].copy(), st_meta[3])
        s_out, _ = solver_c.advance(s_in, op.load.targets[s_in.increment])
        for k in pinned_out:
            pinned_out[k].copy_(getattr(s_out, k), non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        e2e_ms += e0.elapsed_time(e1)
        host_state = {k: v.clone().pin_memory() for k, v in pinned_out.items()}
        st_meta = (s_out.step, s_out.macro_strain, s_out.macro_stress, s_out.increment)
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
    cfg["form"] = FORM_LABEL[args.form]
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (f64 dots, f64 refinement)" if mixed else "f64", "data": "synthetic", "config": cfg,
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
    if world == 1 and rank == 0 and not args.no_cpu:
        sec, sample = cpu_step_estimate({"mech": mech_p, "pf": pf, "stag": stag})
        out["cpu_baseline"] = {"value": 1.0 / sec, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                               "sample": sample}
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
    torch.set_num_threads(os.cpu_count() or 1)
    times = []
    sample = ""
    for _ in range(args.warmup):
        pass
    for _ in range(max(1, min(args.steps, 2))):
        sec, sample = cpu_step_estimate(REF_COUNTS)
        times.append(sec)
    sec = float(np.mean(times))
    value = 1.0 / sec
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(), "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
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
    ap.add_argument("--form", default="mixed-gmg", choices=["plain", "gmg", "mixed", "mixed-gmg"],
                    help="mechanics form of the timed value (the plain FP64 form is timed beside it)")
    ap.add_argument("--kernel-only", action="store_true", help="time the elastic action alone (profiling case)")
    ap.add_argument("--cell", type=int, default=N_CELL, help="cell edge in voxels for --kernel-only")
    ap.add_argument("--fp32", action="store_true", help="FP32 storage/arithmetic for --kernel-only")
    ap.add_argument("--damage-cg", action="store_true", help="with --kernel-only: time box-KKT damage solves instead")
    ap.add_argument("--tile", default="", help="pin the tile shape ox,oy,kz for --kernel-only (else the solver's shape)")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    if args.warmup + args.steps > INCREMENTS:
        raise SystemExit(f"warmup + steps must not exceed the {INCREMENTS} increments of the load path")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, rank, world)), flush=True)
        return
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
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

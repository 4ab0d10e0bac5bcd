"""Many periodic particle-in-matrix cells: seeded microstructures, cost-balanced
sharding across ranks, and the per-rank driver.

The cells are independent units of work, so a multi-GPU run partitions them by
cost (voxel count, greedy longest-processing-time bin packing) and every rank
advances its own cells with no collective on the data path; only the per-cell
records are gathered at the end (``gather_records``).

Microstructure: random sequential addition of spheres in a periodic box with
minimum-image distances, an inclusion core and an interface shell straddling
the particle surface (phast.solid3d.geometry.place_particles / particles,
src/phast/solid3d/geometry.py:30-80), here with one radius per sphere.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .model import LoadCase, PhaseMaterial, SolverConfig, VoxelGrid

MATRIX, INCLUSION, INTERFACE = 0, 1, 2
#: matrix, particle ('fibre') and interface shell ('bn_band') phases of the
#: particle-in-cube batch: E (MPa), nu, Gc (N/mm).  The shell carries 0.3 x the
#: matrix Gc and the matrix stiffness; the particle keeps the matrix Gc.
BATCH_PHASES = (PhaseMaterial("mi_matrix", "isotropic", 0.5, "spectral", 3000.0, 0.3),
                PhaseMaterial("fibre", "isotropic", 0.5, "spectral", 70000.0, 0.3),
                PhaseMaterial("bn_band", "isotropic", 0.15, "spectral", 3000.0, 0.3))


@dataclass
class CellSpec:
    """One cell of the batch: edge ``n`` voxels (edge length 1 mm), phase ids (nz, ny, nx)."""
    index: int
    n: int
    phase: np.ndarray
    centres: np.ndarray = field(repr=False)
    radii: np.ndarray = field(repr=False)

    @property
    def voxels(self):
        return self.n ** 3


def place_spheres(n, radii, rng, max_tries=200000):
    """Random sequential addition of spheres with the given radii (voxel units) in a periodic n^3 box.

    Returns (k, 3) centres in voxel units; a sphere is accepted when its
    minimum-image distance to every placed sphere is at least the sum of the radii.
    """
    box = float(n)
    centres, placed = [], []
    for r in radii:
        for _ in range(max_tries):
            c = rng.random(3) * box
            ok = True
            for o, ro in zip(centres, placed):
                dv = np.abs(c - o)
                dv = np.minimum(dv, box - dv)
                if math.sqrt(float((dv * dv).sum())) < r + ro:
                    ok = False
                    break
            if ok:
                centres.append(c)
                placed.append(r)
                break
        else:
            raise RuntimeError(f"could not place {len(radii)} spheres in a {n}^3 cell")
    return np.array(centres).reshape(-1, 3)


def particle_phase(n, centres, radii, shell=1.0):
    """Phase ids (nz, ny, nx): inclusion inside r - shell/2, interface shell up to r + shell/2."""
    x = np.arange(n) + 0.5
    phase = np.full((n, n, n), MATRIX, dtype=np.uint8)
    best = np.full((n, n, n), np.inf)  # distance to the nearest sphere surface (negative inside)
    for c, r in zip(centres, radii):
        dx = x - c[0]
        dx -= n * np.round(dx / n)
        dy = x - c[1]
        dy -= n * np.round(dy / n)
        dz = x - c[2]
        dz -= n * np.round(dz / n)
        d = np.sqrt(dx[None, None, :] ** 2 + dy[None, :, None] ** 2 + dz[:, None, None] ** 2)
        best = np.minimum(best, d - r)
    phase[best < 0.5 * shell] = INTERFACE
    phase[best < -0.5 * shell] = INCLUSION
    return phase


def particle_cells(seed=0, n_cells=128, sizes=(32, 40, 48, 56, 64), k_range=(4, 12), r_range=(0.08, 0.15)):
    """The seeded particle-in-cube batch: edge N ~ U(sizes), 4-12 spheres of radius U(0.08, 0.15) N voxels."""
    rng = np.random.default_rng(seed)
    cells = []
    for i in range(n_cells):
        n = int(rng.choice(np.asarray(sizes)))
        k = int(rng.integers(k_range[0], k_range[1] + 1))
        radii = np.sort(rng.uniform(r_range[0], r_range[1], k) * n)[::-1]  # large spheres first
        centres = place_spheres(n, radii + 0.5, rng)  # +0.5: the shell half-thickness
        cells.append(CellSpec(i, n, particle_phase(n, centres, radii), centres, radii))
    return cells


def shard_cells(costs, world):
    """Greedy longest-processing-time partition of cells (by cost) over ``world`` ranks.

    Returns a list of index lists, one per rank, each in ascending order.  The
    largest rank load is at most 4/3 of the optimum (Graham's LPT bound).
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += costs[i]
    return [sorted(p) for p in parts]


def batch_load(increments=40, target=0.015):
    """Uniaxial macro strain eps_xx ramped 0 -> target over ``increments`` steps, other components fixed at zero."""
    return LoadCase.ramp("xx", 0, target, increments)


def build_operator(cell, load, device="cuda", phases=BATCH_PHASES, kappa=1e-6):
    """The periodic voxel operator of one batch cell (edge 1 mm, ell = 2 voxels)."""
    from .operator import PeriodicVoxelPhaseFieldOperator
    h = 1.0 / cell.n
    grid = VoxelGrid((cell.n, cell.n, cell.n), (h, h, h))
    return PeriodicVoxelPhaseFieldOperator.from_slots(grid, cell.phase, list(phases), 2 * h, kappa, load,
                                                      device=device)


@dataclass
class CellRecord:
    """What a rank reports for one cell: macro stress per increment and solver counts."""
    index: int
    n: int
    increments: int
    sigma: list
    max_damage: float
    pcg_iters_mech: int
    pcg_iters_pf: int
    seconds: float


def _run_one(cell, increments, device, form, cfg):
    import time

    from .staggered import PLAIN, StaggeredSolver
    load = batch_load()
    t0 = time.perf_counter()
    op = build_operator(cell, load, device=device)
    solver = StaggeredSolver(op, cfg=cfg or SolverConfig(kappa=op.kappa), form=form or PLAIN)
    state = solver.initial_state()
    sig, pm, pp = [], 0, 0
    for _ in range(min(increments, load.n_increments)):
        state, rec = solver.advance(state, load.targets[state.increment])
        sig.append(list(rec.macro_stress))
        pm += rec.pcg_iters_mech
        pp += rec.pcg_iters_pf
    dmax = float(state.d.max())
    return CellRecord(cell.index, cell.n, len(sig), sig, dmax, pm, pp, time.perf_counter() - t0)


def run_cells(cells, indices, increments, *, device="cuda", form=None, cfg=None, streams=1, on_cell=None):
    """Advance the cells ``indices`` (this rank's shard) through ``increments`` load steps; returns records.

    With ``streams`` > 1 that many host threads each own a CUDA stream and take
    the next cell (largest first) from a shared queue, so the small-cell solves,
    which leave most SMs idle on their own, run concurrently on the GPU.
    """
    import queue
    import threading

    import torch
    order = sorted(indices, key=lambda i: (-cells[i].voxels, i))
    if streams <= 1:
        out = []
        for i in order:
            r = _run_one(cells[i], increments, device, form, cfg)
            out.append(r)
            if on_cell is not None:
                on_cell(r)
        return sorted(out, key=lambda r: r.index)
    work = queue.Queue()
    for i in order:
        work.put(i)
    out, errors, lock = [], [], threading.Lock()
    dev = torch.device(device)

    def worker():
        s = torch.cuda.Stream(device=dev)
        with torch.cuda.device(dev), torch.cuda.stream(s):
            while True:
                try:
                    i = work.get_nowait()
                except queue.Empty:
                    break
                try:
                    r = _run_one(cells[i], increments, device, form, cfg)
                except BaseException as exc:  # reported after the other workers drain the queue
                    with lock:
                        errors.append(exc)
                    break
                with lock:
                    out.append(r)
                    if on_cell is not None:
                        on_cell(r)
            s.synchronize()

    threads = [threading.Thread(target=worker, daemon=True) for _ in range(int(streams))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    return sorted(out, key=lambda r: r.index)


def gather_records(local, rank, world, dst=0):
    """Collect every rank's records on ``dst`` (one gather after the solves; None on other ranks)."""
    if world == 1:
        return sorted(local, key=lambda r: r.index)
    import torch.distributed as dist
    got = [None] * world if rank == dst else None
    dist.gather_object(local, got, dst=dst)
    if rank != dst:
        return None
    return sorted((r for part in got for r in part), key=lambda r: r.index)

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


# ----------------------------------------------------------------------------- packed batches

class PackedCellBatch:
    """Cells packed into shared device arrays, with the plan of the batched launches.

    Cell c's reduced nodes, mechanics unknowns ``[u~ (3 n_red), E (6)]`` and elements
    follow those of cells 0..c-1 (``node_off``, ``mech_off``, ``elem_off``).  Every
    elastic or damage action runs all cells in one launch (one block per brick of a cell)
    and every Krylov vector step in one launch (one block per chunk of a cell's vector),
    with each cell's solver state on the device.  The cells share their material slots'
    constants and ``kappa``; grid sizes, ``ell`` and the damage-system scale differ per cell.

    ``brick = (ox, oy, kz)``: nodes per block in x and y (16 x 8 or 8 x 8) and node layers
    per block in z.
    """

    def __init__(self, ops, *, brick=(16, 8, 8)):
        import ctypes as C

        import torch

        from .. import _lib
        if not ops:
            raise ValueError("a batch needs at least one cell")
        ref = ops[0]
        for op in ops[1:]:
            if op.device != ref.device or op.kappa != ref.kappa or op.mat.n_slots != ref.mat.n_slots:
                raise ValueError("batch cells must share device, kappa and material slots")
            for s in range(ref.mat.n_slots):
                if (op.mat.lam[s], op.mat.mu[s], op.mat.Gc[s], op.mat.driver[s]) != \
                        (ref.mat.lam[s], ref.mat.mu[s], ref.mat.Gc[s], ref.mat.driver[s]):
                    raise ValueError("batch cells must share their material slots' constants")
        self.ops = list(ops)
        self.device = ref.device
        self.mat = ref.mat
        self.n_cells = n = len(ops)
        grids = (_lib.VoxelGrid * n)(*[op.vgrid for op in ops])
        ell = (C.c_double * n)(*[op.ell for op in ops])
        dscale = (C.c_double * n)(*[op.damage_scale for op in ops])
        lib = _lib.load()
        self._lib = lib
        self.brick = tuple(int(v) for v in brick)
        h = lib.phastb_batch_create(n, grids, ell, dscale, *self.brick)
        if not h:
            raise ValueError(f"cannot plan a batch with bricks {self.brick} for these grids")
        self._h = C.c_void_p(h)
        out = (C.c_longlong * (7 + 3 * n))()
        _lib.check(lib.phastb_batch_sizes(self._h, out), "phastb_batch_sizes")
        self.n_nodes, self.n_mech, self.n_elem, self.n_blocks = int(out[0]), int(out[1]), int(out[2]), int(out[3])
        self.node_off = [int(out[7 + 3 * c]) for c in range(n)]
        self.mech_off = [int(out[8 + 3 * c]) for c in range(n)]
        self.elem_off = [int(out[9 + 3 * c]) for c in range(n)]
        self._tables = torch.empty(max(int(out[4]), 1), dtype=torch.uint8, device=self.device)
        _lib.check(lib.phastb_batch_bind(self._h, C.c_void_p(self._tables.data_ptr()), C.c_size_t(int(out[4])),
                                         _lib.stream(self.device)), "phastb_batch_bind")
        self.slot = torch.cat([op.slot for op in ops]).contiguous()
        self.fixed = torch.cat([op.mech_fixed_mask().to(torch.uint8) for op in ops]).contiguous()
        self._ws = {}

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and getattr(self, "_lib", None) is not None:
            self._lib.phastb_batch_destroy(h)
            self._h = None

    def workspace(self, key, nbytes):
        """A grow-only device buffer per purpose (stable pointers keep captured graphs valid)."""
        from .. import _lib
        ws = self._ws.get(key)
        if ws is None:
            ws = self._ws[key] = _lib.Workspace(self.device)
        return ws.get(nbytes)

    # -- packing -----------------------------------------------------------------------------
    def pack_nodes(self, parts):
        import torch
        return torch.cat([p.reshape(-1) for p in parts]).contiguous()

    def pack_mech(self, parts):
        import torch
        return torch.cat([p.reshape(-1) for p in parts]).contiguous()

    def pack_elems(self, parts):
        import torch
        return torch.cat([p.reshape(-1, 8) for p in parts]).contiguous()

    def node_view(self, t, c):
        return t[self.node_off[c]:self.node_off[c] + self.ops[c].n_red]

    def mech_view(self, t, c):
        return t[self.mech_off[c]:self.mech_off[c] + self.ops[c].n_mech]

    def elem_view(self, t, c):
        return t[self.elem_off[c]:self.elem_off[c] + self.ops[c].n_elements]

    # -- batched operators and solves --------------------------------------------------------
    def mech_apply(self, x, d=None, *, mask=None, out=None, macro_rows=True):
        """y = A(d) x of every cell in one launch (FP64 or FP32, like ``x``); returns (y, rE (C, 6)),
        rE the per-cell macro-stress row sums (None with ``macro_rows=False``, which skips their
        host read).  ``out`` receives y."""
        import ctypes as C

        import numpy as np
        import torch

        from .. import _lib
        y = torch.empty_like(x) if out is None else out
        rE = (C.c_double * (6 * self.n_cells))() if macro_rows else None
        dt = _lib.F64 if x.dtype == torch.float64 else _lib.F32
        wp, wn = self.workspace("apply", self._lib.phastb_batch_apply_workspace_bytes(self._h))
        _lib.call("phastb_batch_mech_apply", self._h, self.mat, _lib.ptr(self.slot), dt, _lib.ptr(x), _lib.ptr(d),
                  _lib.ptr(mask), _lib.ptr(y), rE, wp, wn, _lib.stream(self.device))
        return y, (np.array(rE[:]).reshape(self.n_cells, 6) if macro_rows else None)

    def damage_apply(self, d, H=None, *, scaled=True, mask=None):
        """The damage action of every cell in one launch (each scaled by its damage-system scale)."""
        import torch

        from .. import _lib
        y = torch.empty_like(d)
        wp, wn = self.workspace("apply", self._lib.phastb_batch_apply_workspace_bytes(self._h))
        _lib.call("phastb_batch_damage_apply", self._h, self.mat, _lib.ptr(self.slot), _lib.ptr(d), _lib.ptr(H),
                  int(bool(scaled)), _lib.ptr(mask), _lib.ptr(y), wp, wn, _lib.stream(self.device))
        return y

    def mech_solve(self, d, fixed_values, *, x0=None, rtol=1e-8, atol=0.0, maxiter=20000, check_every=10,
                   mixed=False, inner_rtol=1e-4, max_refine=30, live=None, form=None, reuse_lmax=False):
        """Constrained mechanics solve of every cell (``live``: the cells to solve, others keep ``x0``).

        ``form``: a ``MechForm``; with ``precond='gmg'`` (and ``mixed=True``) every cell's FP32 inner
        PCG is preconditioned by the voxel multigrid V-cycle, all cells in the same launches
        (``reuse_lmax``: keep the per-cell lambda_max estimates of the previous multigrid solve).
        Returns ``(x, status, iterations (C,), converged (C,), rhs_norm (C,), residual_norm (C,))``.
        """
        if form is not None and form.precond == "gmg":
            return self._mech_solve_gmg(d, fixed_values, x0, rtol, atol, maxiter, check_every, form, live,
                                        reuse_lmax)
        import ctypes as C

        import numpy as np
        import torch

        from .. import _lib
        n = self.n_cells
        x = torch.empty(self.n_mech, dtype=torch.float64, device=self.device)
        info = (C.c_int * (2 * n))()
        rinfo = (C.c_double * (2 * n))()
        lv = None if live is None else (C.c_int * n)(*[int(bool(v)) for v in live])
        wp, wn = self.workspace(("mech", int(mixed)),
                                self._lib.phastb_batch_mech_solve_workspace_bytes(self._h, int(mixed)))
        st = _lib.raw("phastb_batch_mech_solve", self._h, self.mat, _lib.ptr(self.slot), _lib.ptr(d),
                      _lib.ptr(self.fixed), _lib.ptr(fixed_values), _lib.ptr(x0), float(rtol), float(atol),
                      int(maxiter), int(check_every), int(bool(mixed)), float(inner_rtol), int(max_refine), lv,
                      _lib.ptr(x), info, rinfo, wp, wn, _lib.stream(self.device))
        if st not in (_lib.OK, _lib.NONCONVERGED, _lib.BREAKDOWN, _lib.NONFINITE):
            _lib.check(st, "phastb_batch_mech_solve")
        inf = np.array(info[:]).reshape(n, 2)
        rin = np.array(rinfo[:]).reshape(n, 2)
        return x, st, inf[:, 0], inf[:, 1].astype(bool), rin[:, 0], rin[:, 1]

    def _mech_solve_gmg(self, d, fixed_values, x0, rtol, atol, maxiter, check_every, form, live, reuse_lmax):
        import ctypes as C

        import numpy as np
        import torch

        from .. import _lib
        if not form.mixed:
            raise NotImplementedError("the batched multigrid runs in the mixed form (FP32 V-cycle, FP64 refinement)")
        n = self.n_cells
        opts = form.struct()
        nbytes = self._lib.phastb_batch_mech_solve_ex_workspace_bytes(self._h, opts)
        if nbytes == 0:
            raise NotImplementedError("the batched multigrid needs periodic cells with edges divisible by 4 and at "
                                      "least 32 (three levels)")
        x = torch.empty(self.n_mech, dtype=torch.float64, device=self.device)
        info = (C.c_int * (2 * n))()
        rinfo = (C.c_double * (2 * n))()
        lv = None if live is None else (C.c_int * n)(*[int(bool(v)) for v in live])
        wp, wn = self.workspace("mech_gmg", nbytes)
        st = _lib.raw("phastb_batch_mech_solve_ex", self._h, self.mat, _lib.ptr(self.slot), _lib.ptr(d),
                      _lib.ptr(self.fixed), _lib.ptr(fixed_values), _lib.ptr(x0), float(rtol), float(atol),
                      int(maxiter), int(check_every), opts, int(bool(reuse_lmax)), lv, _lib.ptr(x), info, rinfo,
                      wp, wn, _lib.stream(self.device))
        if st not in (_lib.OK, _lib.NONCONVERGED, _lib.BREAKDOWN, _lib.NONFINITE):
            _lib.check(st, "phastb_batch_mech_solve_ex")
        inf = np.array(info[:]).reshape(n, 2)
        rin = np.array(rinfo[:]).reshape(n, 2)
        return x, st, inf[:, 0], inf[:, 1].astype(bool), rin[:, 0], rin[:, 1]

    def damage_box_kkt(self, H, lower, initial, *, upper=1.0, linear_tolerance=1e-10, kkt_tolerance=1e-8,
                       min_tolerance=0.0, staggered_tolerance=False, max_linear_iterations=4000,
                       max_active_set_iterations=64, live=None):
        """Box-KKT damage solve of every cell's scaled system; returns ``(d, status, info (C, 4), rinfo (C, 2))``
        with info = PCG iterations, active-set iterations, kkt_ok, status per cell."""
        import ctypes as C

        import numpy as np
        import torch

        from .. import _lib
        n = self.n_cells
        d = torch.empty(self.n_nodes, dtype=torch.float64, device=self.device)
        info = (C.c_int * (4 * n))()
        rinfo = (C.c_double * (2 * n))()
        lv = None if live is None else (C.c_int * n)(*[int(bool(v)) for v in live])
        wp, wn = self.workspace("kkt", self._lib.phastb_batch_box_kkt_workspace_bytes(self._h))
        st = _lib.raw("phastb_batch_damage_box_kkt", self._h, self.mat, _lib.ptr(self.slot), _lib.ptr(H),
                      _lib.ptr(lower), float(upper), _lib.ptr(initial), float(linear_tolerance), float(kkt_tolerance),
                      float(min_tolerance), int(bool(staggered_tolerance)), int(max_linear_iterations),
                      int(max_active_set_iterations), lv, _lib.ptr(d), info, rinfo, wp, wn, _lib.stream(self.device))
        if st not in (_lib.OK, _lib.NONCONVERGED, _lib.BREAKDOWN, _lib.NONFINITE):
            _lib.check(st, "phastb_batch_damage_box_kkt")
        return d, st, np.array(info[:]).reshape(n, 4), np.array(rinfo[:]).reshape(n, 2)

    def stagger_change(self, x_new, x_old, d_new, d_old):
        """(C, 5) staggered change parts: ||du~||, ||u~||, max|dE|, max|E|, max|dd| per cell."""
        import ctypes as C

        import numpy as np

        from .. import _lib
        out = (C.c_double * (5 * self.n_cells))()
        wp, wn = self.workspace("change", self._lib.phastb_batch_change_workspace_bytes(self._h))
        _lib.call("phastb_batch_stagger_change", self._h, _lib.ptr(x_new), _lib.ptr(x_old), _lib.ptr(d_new),
                  _lib.ptr(d_old), out, wp, wn, _lib.stream(self.device))
        return np.array(out[:]).reshape(self.n_cells, 5)


@dataclass(eq=False)
class BatchState:
    """Accepted packed state of every cell after ``step`` solves (``SolverState`` per cell, packed)."""
    step: int
    x: object
    d: object
    H: object
    macro_strain: np.ndarray  # (C, 6)
    macro_stress: np.ndarray  # (C, 6)
    external_work: np.ndarray  # (C,)
    increment: int = 0


class BatchStaggeredSolver:
    """The staggered AT2 increment of every cell of a :class:`PackedCellBatch` at once.

    Per cell the decisions of ``StaggeredSolver._attempt`` (solid3d/staggered.py:1259-1499):
    the predictor, alternate mechanics / history / box-KKT damage solves, the ``_change``
    stopping rule ``change <= stagger_tol and k >= min_stagger``, the final mechanics
    re-solve and the increment record.  A cell that has converged takes no part in the
    remaining passes of the others.  ``mixed``: FP32 mechanics PCG with FP64 dot products
    under FP64 iterative refinement to the same FP64 stopping rule.  Every cell follows the
    same load path (``load``).
    """

    def __init__(self, batch, load, cfg=None, *, mixed=True, inner_rtol=1e-4, max_refine=30, form=None):
        self.form = form
        self.lmax_every = 10
        self._gmg_solves = 0
        self.batch = batch
        self.load = load
        self.cfg = cfg or SolverConfig(kappa=batch.ops[0].kappa)
        c = self.cfg
        if (getattr(c, "irreversibility", "box_kkt") != "box_kkt" or getattr(c, "anderson_depth", 0)
                or getattr(c, "crack_closure", "none") != "none" or getattr(c, "damage_law", "at2") != "at2"
                or any(op.is_pfczm or op.has_closure for op in batch.ops)):
            raise NotImplementedError("the packed batch runs the AT2 law with box-KKT irreversibility, without "
                                      "crack closure or Anderson mixing")
        self.mixed = bool(mixed)
        self.inner_rtol = float(inner_rtol)
        self.max_refine = int(max_refine)
        self._c = int(load.controlled)
        C_ = batch.n_cells
        self._max_abs_target = max(abs(float(t)) for t in load.targets)
        self._u_floor = np.array([min(op.h) * math.sqrt(3 * op.n_red) for op in batch.ops])
        self.n_attempts = 0
        self._increments = 0

    def _mech(self, d, values, x0, live, first):
        """One batched mechanics solve of the configured form.  The multigrid's per-cell lambda_max
        estimates are refreshed at the first solve of every ``lmax_every``-th increment."""
        cfg = self.cfg
        reuse = False
        if self.form is not None and self.form.precond == "gmg":
            reuse = self._gmg_solves > 0 and not (first and self._increments % self.lmax_every == 0)
            self._gmg_solves += 1
        return self.batch.mech_solve(d, values, x0=x0, rtol=cfg.pcg_rtol_mech, maxiter=cfg.pcg_maxit_mech,
                                     check_every=cfg.check_every, mixed=self.mixed, inner_rtol=self.inner_rtol,
                                     max_refine=self.max_refine, live=live, form=self.form, reuse_lmax=reuse)

    def initial_state(self):
        import torch
        b = self.batch
        z = lambda *s: torch.zeros(*s, dtype=torch.float64, device=b.device)  # noqa: E731
        C_ = b.n_cells
        return BatchState(0, z(b.n_mech), z(b.n_nodes), z(b.n_elem, 8), np.zeros((C_, 6)), np.zeros((C_, 6)),
                          np.zeros(C_), 0)

    def _driving(self, x, H_prev, H_out, live):
        import ctypes as C

        from .. import _lib
        b = self.batch
        lib = _lib.load()
        s = _lib.stream(b.device)
        xp, hp, ho, sp = x.data_ptr(), H_prev.data_ptr(), H_out.data_ptr(), b.slot.data_ptr()
        for c, op in enumerate(b.ops):
            if not live[c]:
                continue
            st = lib.phastb_h8_driving_history(op.vgrid, op.mat, C.c_void_p(sp + b.elem_off[c]),
                                               C.c_void_p(xp + 8 * b.mech_off[c]),
                                               C.c_void_p(hp + 64 * b.elem_off[c]), None,
                                               C.c_void_p(ho + 64 * b.elem_off[c]), s)
            _lib.check(st, "phastb_h8_driving_history")

    def advance(self, state, target):
        """Solve the next load increment of every cell from ``state`` to ``E_c = target``.

        Returns ``(state, records)`` with one :class:`~phast_b200.solid3d.staggered.IncrementRecord`
        per cell; raises :class:`~phast_b200.solid3d.staggered.StaggerConvergenceError` naming the
        cells that failed.
        """
        import torch

        from time import perf_counter

        from .. import _lib
        from .staggered import _MIN_LINEAR_TOLERANCE, IncrementRecord, StaggerConvergenceError
        b, cfg = self.batch, self.cfg
        C_ = b.n_cells
        t0 = perf_counter()
        target = float(target)
        previous = float(state.macro_strain[0, self._c])
        if target == previous:
            raise ValueError(f"target {target!r} equals the current controlled strain")
        increment = state.increment + 1
        self.n_attempts += 1
        values = torch.empty(b.n_mech, dtype=torch.float64, device=b.device)
        x_old = torch.empty_like(values)
        _lib.call("phastb_batch_predictor", b._h, _lib.ptr(state.x), target / previous if previous != 0.0 else 0.0,
                  self._c, target, _lib.ptr(x_old), _lib.ptr(values), _lib.stream(b.device))
        d_old = state.d.clone()
        lower = state.d
        H = state.H.clone()
        step_size = abs(target - previous)
        live = np.ones(C_, dtype=bool)
        k_done = np.zeros(C_, dtype=np.int64)
        change_done = np.full(C_, np.inf)
        pm = np.zeros(C_, dtype=np.int64)
        pp = np.zeros(C_, dtype=np.int64)
        sets = np.zeros(C_, dtype=np.int64)
        kkt = np.ones(C_, dtype=bool)
        failed = {}

        def fail(reason):
            raise StaggerConvergenceError(f"increment {increment} to E[{self._c}] = {target:.6e} failed: {reason}",
                                          state=state, target=target, increment=increment, cutbacks=0,
                                          reason=reason)

        for k in range(1, cfg.max_stagger + 1):
            x_new, st, its, conv, _, _ = self._mech(d_old, values, x_old, live, first=(k == 1))
            pm += np.where(live, its, 0)
            bad = np.flatnonzero(live & ~conv)
            if bad.size:
                fail(f"mechanics PCG did not converge in cells {bad.tolist()}")
            self._driving(x_new, state.H, H, live)
            d_new, st, info, _ = b.damage_box_kkt(H, lower, d_old, linear_tolerance=cfg.damage_linear_tol,
                                                  kkt_tolerance=cfg.damage_kkt_tol,
                                                  min_tolerance=_MIN_LINEAR_TOLERANCE, staggered_tolerance=True,
                                                  max_linear_iterations=cfg.damage_maxit,
                                                  max_active_set_iterations=cfg.damage_max_active_set, live=live)
            pp += np.where(live, info[:, 0], 0)
            sets += np.where(live, info[:, 1], 0)
            bad = np.flatnonzero(live & (info[:, 3] != 0))
            if bad.size:
                fail(f"damage box-KKT solve failed in cells {bad.tolist()}")
            kkt &= np.where(live, info[:, 2] != 0, True)
            parts = b.stagger_change(x_new, x_old, d_new, d_old)
            du, u, dE, E_inf, dd = parts.T
            if not np.all(np.isfinite(parts[live])):
                fail("staggered iterate is not finite")
            scale_E = np.maximum(E_inf, step_size)
            u_ref = np.maximum(u, scale_E * self._u_floor)
            du_rel = np.where(u_ref > 0, du / np.where(u_ref > 0, u_ref, 1.0), 0.0)
            dE_rel = np.where(scale_E > 0, dE / np.where(scale_E > 0, scale_E, 1.0), 0.0)
            change = np.maximum(np.maximum(du_rel, dE_rel), dd)
            x_old, d_old = x_new, d_new
            stop = live & (change <= cfg.stagger_tol) & (k >= cfg.min_stagger)
            k_done[live] = k
            change_done[live] = change[live]
            live = live & ~stop
            if not live.any():
                break
        if live.any():
            fail(f"staggered iteration did not converge in {cfg.max_stagger} iterations in cells "
                 f"{np.flatnonzero(live).tolist()}")
        d = d_old
        rel = np.zeros(C_)
        if cfg.final_mechanics_resolve:
            x, st, its, conv, bn, rn = self._mech(d, values, x_old, None, first=False)
            pm += its
            if not conv.all():
                fail(f"mechanics PCG did not converge in cells {np.flatnonzero(~conv).tolist()}")
            rel = np.where(bn > 0, rn / np.where(bn > 0, bn, 1.0), 0.0)
        else:
            x = x_old
        E_all = np.zeros((C_, 6))
        S_all = np.zeros((C_, 6))
        W = np.zeros(C_)
        records = []
        wall = perf_counter() - t0
        for c, op in enumerate(b.ops):
            rec = op.increment_record(b.mech_view(x, c), b.node_view(d, c), b.elem_view(H, c), cfg.damaged_threshold)
            E = rec["E"]
            sigma = rec["rE"] / op.volume
            elastic = rec["energy"]
            fracture = rec["local"] + rec["gradient"]
            if not np.isfinite(np.concatenate([E, sigma, [elastic, fracture]])).all():
                fail(f"accepted state of cell {c} has non-finite stress, strain or energy")
            mean_work = 2.0 * elastic / op.volume
            macro_work = float(np.dot(sigma, E))
            scale = max(abs(mean_work), abs(macro_work))
            hill_rel = abs(mean_work - macro_work) / scale if scale > 0 else 0.0
            external = state.external_work[c] + op.volume * 0.5 * (sigma[self._c] + state.macro_stress[c, self._c]) * \
                (target - previous)
            residual = external - (elastic + fracture)
            E_all[c], S_all[c], W[c] = E, sigma, external
            lengths = tuple(nn * hh for nn, hh in zip(op.shape, op.h))
            axis = self._c if self._c < 3 else 0
            others = tuple(lengths[a] for a in range(3) if a != axis)
            records.append(IncrementRecord(
                step=state.step + 1, increment=increment, load_factor=target / self._max_abs_target,
                macro_strain=tuple(float(v) for v in E), macro_stress=tuple(float(v) for v in sigma),
                applied_disp=float(E[axis]) * lengths[axis], reaction_force=float(sigma[axis]) * others[0] * others[1],
                elastic=float(elastic), fracture=float(fracture), fracture_by_phase=dict(rec["by_phase"]),
                external=float(external), balance_residual=float(residual),
                balance_residual_rel=float(residual / max(abs(external), 1e-300)), max_damage=float(rec["max_d"]),
                mean_damage=float(rec["sum_element_d"] / op.n_elements),
                damaged_volume_fraction=float(rec["damaged"] / op.n_elements), max_H=float(rec["max_H"]),
                stagger_iters=int(k_done[c]), pcg_iters_mech=int(pm[c]), pcg_iters_pf=int(pp[c]),
                active_set_iters=int(sets[c]), cutbacks=0, converged=True, kkt_ok=bool(kkt[c]),
                stagger_change=float(change_done[c]), mech_relative_residual=float(rel[c]),
                hill_mandel_rel=float(hill_rel), wall_s=wall, mean_strain=tuple(float(v) for v in E)))
        new_state = BatchState(state.step + 1, x, d, H, E_all, S_all, W, increment)
        self._increments += 1
        return new_state, records

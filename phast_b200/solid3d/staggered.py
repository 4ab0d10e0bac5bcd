"""3D solvers and the staggered increment on the GPU.

* ``solve_constrained`` -- Jacobi PCG with device flags on the free set
  (solid3d/linalg.py:99-287); the whole solve is one C-ABI call.
* ``solve_h8_scalar_box_kkt`` -- primal active-set box-KKT damage solve with a
  Dirichlet PCG per set and the KKT audit (solvers/box_kkt_h8.py:256-778).
* ``StaggeredSolver`` -- alternate minimisation of one load increment with
  ``history='max'`` and ``irreversibility='box_kkt'`` (solid3d/staggered.py:1207-1517).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from time import perf_counter

import numpy as np
import torch

from .. import _lib
from .._lib import ptr, raw, stream
from .model import SolverConfig


class PCGBreakdownError(RuntimeError):
    """Non-positive curvature, non-positive diagonal or non-finite values (linalg.py:41-44)."""


class H8ScalarBoxKKTConvergenceError(RuntimeError):
    """The active set did not stabilise or a PCG did not converge (box_kkt_h8.py:239-253)."""


class StaggerConvergenceError(RuntimeError):
    """A failed increment; carries the last accepted state (staggered.py:221-263)."""

    def __init__(self, message, state=None):
        super().__init__(message)
        self.state = state


@dataclass(frozen=True)
class PCGInfo:
    iterations: int
    converged: bool
    rhs_norm: float
    residual_norm: float
    relative_residual: float


def solve_constrained(op, *, fixed_mask, fixed_values, g=None, d=None, x0=None, rtol=1e-8, atol=0.0, maxiter=5000,
                      check_every=10):
    """``A(g) x = 0`` with ``x = fixed_values`` on ``fixed_mask`` by projected Jacobi PCG (linalg.py:223-287)."""
    n = op.n_mech
    mask = fixed_mask.to(torch.uint8).contiguous()
    vals = fixed_values.to(torch.float64).contiguous()
    x0c = None if x0 is None else x0.to(torch.float64).contiguous()
    gq = None if g is None else g.to(torch.float64).contiguous()
    dd = None if d is None else d.to(torch.float64).contiguous()
    out = torch.empty(n, dtype=torch.float64, device=op.device)
    info = (C.c_int * 2)()
    rinfo = (C.c_double * 2)()
    wp, wn = op._ws.get(_lib.load().phastb_h8_mech_solve_workspace_bytes(op.vgrid, _lib.F64))
    st = raw("phastb_h8_mech_solve", op.vgrid, op.mat, ptr(op.slot), ptr(gq), ptr(dd), ptr(mask), ptr(vals),
             ptr(x0c), float(rtol), float(atol), int(maxiter), int(check_every), ptr(out), info, rinfo, wp, wn,
             stream())
    if st in (_lib.BREAKDOWN, _lib.NONFINITE):
        raise PCGBreakdownError(f"PCG breakdown (status {st})")
    if st not in (_lib.OK, _lib.NONCONVERGED):
        _lib.check(st, "phastb_h8_mech_solve")
    bn, rn = float(rinfo[0]), float(rinfo[1])
    return out, PCGInfo(int(info[0]), bool(info[1]), bn, rn, rn / bn if bn > 0 else 0.0)


@dataclass(frozen=True)
class MechForm:
    """How the mechanics system is solved.

    ``precond``: ``'jacobi'`` (PhAST's solve_constrained) or ``'gmg'`` (3-level voxel multigrid,
    Chebyshev smoothing).  ``mixed``: FP32 inner PCG with FP64 dot products under FP64 iterative
    refinement (the stopping test is always the FP64 residual).
    """
    precond: str = "jacobi"
    mixed: bool = False
    levels: int = 3
    smooth_degree: int = 2
    coarse_degree: int = 8
    power_iters: int = 30
    lmax_safety: float = 1.2
    inner_rtol: float = 1e-4
    max_refine: int = 30

    def struct(self):
        o = _lib.MechOpts()
        o.precond = 1 if self.precond == "gmg" else 0
        o.mixed = int(bool(self.mixed))
        o.levels, o.smooth_degree, o.coarse_degree = self.levels, self.smooth_degree, self.coarse_degree
        o.power_iters, o.inner_rtol, o.max_refine = self.power_iters, self.inner_rtol, self.max_refine
        o.lmax_safety = self.lmax_safety
        return o


PLAIN = MechForm()


def solve_constrained_form(op, form, *, fixed_mask, fixed_values, d=None, x0=None, rtol=1e-8, atol=0.0,
                           maxiter=5000, check_every=10, lmax_cache=None):
    """Constrained mechanics solve with a :class:`MechForm` (multigrid and/or mixed precision).

    ``lmax_cache`` (a ctypes array of 3 doubles, zero to estimate) carries the multigrid's
    lambda_max estimates from one solve to the next.
    """
    if form.precond == "jacobi" and not form.mixed:
        return solve_constrained(op, fixed_mask=fixed_mask, fixed_values=fixed_values, d=d, x0=x0, rtol=rtol,
                                 atol=atol, maxiter=maxiter, check_every=check_every)
    n = op.n_mech
    opts = form.struct()
    nbytes = _lib.load().phastb_h8_mech_solve_ex_workspace_bytes(op.vgrid, opts)
    if nbytes == 0:
        raise NotImplementedError(f"mechanics form {form} is not available for a {op.shape} grid "
                                  "(multigrid needs edges divisible by 2^(levels-1))")
    mask = fixed_mask.to(torch.uint8).contiguous()
    vals = fixed_values.to(torch.float64).contiguous()
    x0c = None if x0 is None else x0.to(torch.float64).contiguous()
    dd = (torch.zeros(op.n_red, dtype=torch.float64, device=op.device) if d is None
          else d.to(torch.float64).contiguous())
    out = torch.empty(n, dtype=torch.float64, device=op.device)
    info = (C.c_int * 2)()
    rinfo = (C.c_double * 2)()
    wp, wn = op._ws.get(nbytes)
    st = raw("phastb_h8_mech_solve_ex", op.vgrid, op.mat, ptr(op.slot), ptr(dd), ptr(mask), ptr(vals), ptr(x0c),
             float(rtol), float(atol), int(maxiter), int(check_every), opts, lmax_cache, ptr(out), info, rinfo, wp, wn,
             stream())
    if st in (_lib.BREAKDOWN, _lib.NONFINITE):
        raise PCGBreakdownError(f"PCG breakdown (status {st})")
    if st not in (_lib.OK, _lib.NONCONVERGED):
        _lib.check(st, "phastb_h8_mech_solve_ex")
    bn, rn = float(rinfo[0]), float(rinfo[1])
    return out, PCGInfo(int(info[0]), bool(info[1]), bn, rn, rn / bn if bn > 0 else 0.0)


@dataclass(frozen=True)
class BoxKKTResult:
    solution: torch.Tensor
    total_pcg_iterations: int
    active_set_iterations: int
    satisfies_kkt: bool


def solve_h8_scalar_box_kkt(system, *, lower_bound=0.0, upper_bound=1.0, initial=None, linear_tolerance=1e-10,
                            kkt_tolerance=1e-9, max_linear_iterations=4000, max_active_set_iterations=64,
                            check_bounds=True):
    """Box-constrained scalar H8 solve (box_kkt_h8.py:603-778) of ``op.damage_system(H)``.

    ``check_bounds=False`` skips the ValueError checks of the bounds and the initial
    guess (one device-to-host read) for callers whose inputs satisfy them by
    construction.
    """
    op = system.op
    n = op.n_red
    if not isinstance(upper_bound, (int, float)):
        raise NotImplementedError("the B200 box-KKT solve takes a scalar upper bound")
    lower = (torch.full((n,), float(lower_bound), dtype=torch.float64, device=op.device)
             if not isinstance(lower_bound, torch.Tensor) else lower_bound.to(torch.float64).contiguous())
    init = None if initial is None else initial.to(torch.float64).contiguous()
    if check_bounds:
        flags = [(lower > upper_bound).any()]
        if init is not None:
            flags.append(((init < lower) | (init > upper_bound)).any())
        flags = torch.stack(flags).tolist()  # one read for both checks
        if flags[0]:
            raise ValueError("lower_bound must not exceed upper_bound at any degree of freedom")
        if len(flags) > 1 and flags[1]:
            raise ValueError("initial must already satisfy the requested box bounds; it is never clipped")
    H = None if system.H is None else system.H.to(torch.float64).contiguous()
    out = torch.empty(n, dtype=torch.float64, device=op.device)
    info = (C.c_int * 3)()
    wp, wn = op._ws.get(_lib.load().phastb_h8_box_kkt_workspace_bytes(op.vgrid))
    st = raw("phastb_h8_damage_box_kkt", op.vgrid, op.mat, ptr(op.slot), ptr(H), system.scale, ptr(lower),
             float(upper_bound), ptr(init), float(linear_tolerance), float(kkt_tolerance),
             int(max_linear_iterations), int(max_active_set_iterations), ptr(out), info, wp, wn, stream())
    if st in (_lib.BREAKDOWN, _lib.NONFINITE):
        raise RuntimeError(f"PCG operator is not positive definite on the free space (status {st})")
    if st == _lib.NONCONVERGED:
        raise H8ScalarBoxKKTConvergenceError(
            f"H8 scalar box-KKT failed after {info[1]} active-set iterations ({info[0]} PCG iterations)")
    _lib.check(st, "phastb_h8_damage_box_kkt")
    return BoxKKTResult(out, int(info[0]), int(info[1]), bool(info[2]))


@dataclass
class SolverState:
    """Accepted state of the staggered solver (staggered.py:167-218)."""
    step: int
    x: torch.Tensor
    d: torch.Tensor
    H: torch.Tensor
    macro_strain: np.ndarray
    macro_stress: np.ndarray
    increment: int


@dataclass
class IncrementRecord:
    increment: int
    target: float
    macro_stress: tuple
    stagger_iters: int
    pcg_iters_mech: int
    pcg_iters_pf: int
    active_set_iters: int
    kkt_ok: bool
    max_damage: float
    wall_s: float


class _AttemptFailure(RuntimeError):
    pass


class StaggeredSolver:
    """Staggered alternate minimisation of the hybrid AT2 cell (solid3d/staggered.py)."""

    def __init__(self, op, cfg=None, form=PLAIN):
        self.op = op
        self.cfg = cfg or SolverConfig()
        self.form = form
        self._lmax = (C.c_double * 3)()
        self.lmax_every = 10
        self.load = op.load
        self._c = int(op.load.controlled)
        self._n_u = 3 * op.n_red
        self._u_floor = min(op.h) * math.sqrt(self._n_u)
        self._mask = op.mech_fixed_mask()
        self._red = _lib.Workspace(op.device)
        self._tail = torch.empty(7, dtype=torch.float64, pin_memory=True)

    def initial_state(self):
        op = self.op
        z = lambda *s: torch.zeros(*s, dtype=torch.float64, device=op.device)
        return SolverState(0, z(op.n_mech), z(op.n_red), z(op.n_elements, 8), np.zeros(6), np.zeros(6), 0)

    def _change(self, x_new, x_old, d_new, d_old, step_size):
        """max(du_rel, dE_rel, dd_inf) (staggered.py:1097-1124)."""
        out = (C.c_double * 5)()
        wp, wn = self._red.get(_lib.load().phastb_reduce_workspace_bytes())
        _lib.call("phastb_h8_stagger_change", self._n_u, ptr(x_new), ptr(x_old), self.op.n_red, ptr(d_new),
                  ptr(d_old), out, wp, wn, stream())
        du, u, dE, E_inf, dd = (float(v) for v in out)
        if not all(math.isfinite(v) for v in (du, u, dE, E_inf, dd)):
            raise _AttemptFailure("staggered iterate is not finite")
        scale_E = max(E_inf, step_size)
        u_ref = max(u, scale_E * self._u_floor)
        du_rel = du / u_ref if u_ref > 0 else 0.0
        dE_rel = dE / scale_E if scale_E > 0 else 0.0
        return max(du_rel, dE_rel, dd)

    def _mechanics(self, d, values, x0):
        cfg = self.cfg
        try:
            x, info = solve_constrained_form(self.op, self.form, fixed_mask=self._mask, fixed_values=values, d=d,
                                             x0=x0, rtol=cfg.pcg_rtol_mech, maxiter=cfg.pcg_maxit_mech,
                                             check_every=cfg.check_every, lmax_cache=self._lmax)
        except PCGBreakdownError as exc:
            raise _AttemptFailure(f"mechanics PCG breakdown: {exc}") from exc
        if not info.converged:
            raise _AttemptFailure(f"mechanics PCG did not converge in {cfg.pcg_maxit_mech} iterations")
        return x, info

    def _damage(self, H, lower, initial):
        cfg, op = self.cfg, self.op
        system = op.damage_system(H)
        r0 = float(torch.linalg.vector_norm(system.rhs - system.apply(initial)))
        if not math.isfinite(r0):
            raise _AttemptFailure("damage residual is not finite")
        tol = min(cfg.damage_linear_tol, 0.1 * cfg.damage_kkt_tol / max(r0, 1.0))
        tol = max(tol, 4.0 * float(np.finfo(np.float64).eps))
        # the bounds hold by construction: lower is the accepted damage of the last
        # increment (in [0, 1]) and initial is lower itself or a box-KKT solution
        try:
            res = solve_h8_scalar_box_kkt(system, lower_bound=lower, upper_bound=1.0, initial=initial,
                                          linear_tolerance=tol, kkt_tolerance=cfg.damage_kkt_tol,
                                          max_linear_iterations=cfg.damage_maxit,
                                          max_active_set_iterations=cfg.damage_max_active_set,
                                          check_bounds=False)
        except (H8ScalarBoxKKTConvergenceError, RuntimeError) as exc:
            raise _AttemptFailure(f"damage box-KKT solve failed: {exc}") from exc
        return res.solution, res.total_pcg_iterations, res.active_set_iterations, res.satisfies_kkt

    def _predictor(self, state, previous, target):
        x = state.x * (target / previous) if previous != 0.0 else torch.zeros_like(state.x)
        x[self._n_u + self._c] = target
        return x

    def advance(self, state, target, *, increment=None):
        """One increment to E_c = target (staggered.py:1215-1257); raises StaggerConvergenceError."""
        target = float(target)
        previous = float(state.macro_strain[self._c])
        if target == previous:
            raise ValueError(f"target {target!r} equals the current controlled strain")
        increment = state.increment + 1 if increment is None else int(increment)
        t0 = perf_counter()
        # lambda_max of the Jacobi-scaled operator barely moves with the damage
        # field; the multigrid re-estimates it every `lmax_every` increments
        if (increment - 1) % self.lmax_every == 0:
            self._lmax[0] = 0.0
        try:
            return self._attempt(state, target, previous, increment, t0)
        except _AttemptFailure as exc:
            raise StaggerConvergenceError(f"increment {increment} to E[{self._c}] = {target:.6e} failed: {exc}",
                                          state) from exc

    def _attempt(self, state, target, previous, increment, t0):
        op, cfg = self.op, self.cfg
        values = op.mech_fixed_values(target)
        step = abs(target - previous)
        x_old = self._predictor(state, previous, target)
        d_old = state.d.clone()
        lower = state.d
        pm = pp = sets = 0
        kkt = True
        H = state.H
        converged = False
        for k in range(1, cfg.max_stagger + 1):
            x_new, info = self._mechanics(d_old, values, x_old)
            pm += info.iterations
            _, H = op.driving_history(x_new, state.H)
            d_new, its, s, kkt = self._damage(H, lower, d_old)
            pp += its
            sets += s
            change = self._change(x_new, x_old, d_new, d_old, step)
            x_old, d_old = x_new, d_new
            if change <= cfg.stagger_tol and k >= cfg.min_stagger:
                converged = True
                break
        if not converged:
            raise _AttemptFailure(f"staggered iteration did not converge in {cfg.max_stagger} iterations")
        d = d_old
        if cfg.final_mechanics_resolve:
            x, info = self._mechanics(d, values, x_old)
            pm += info.iterations
        else:
            x = x_old
        g = op.degradation(d)
        # E and max(d) travel in one copy that the stress reduction's read waits for
        tail = torch.cat((op.split_mech(x)[1].detach(), d.max().reshape(1)))
        self._tail.copy_(tail, non_blocking=True)
        done = torch.cuda.Event()
        done.record()
        rE, _ = op._stress_energy(x, g)
        done.synchronize()
        sigma = rE / op.volume
        E = self._tail[:6].numpy().copy()
        d_max = float(self._tail[6])
        completes = 1 <= increment <= self.load.n_increments and target == self.load.targets[increment - 1]
        new_state = SolverState(state.step + 1, x, d, H, E.copy(), sigma,
                                increment if completes else state.increment)
        rec = IncrementRecord(increment, target, tuple(float(v) for v in sigma), k, pm, pp, sets, bool(kkt),
                              d_max, perf_counter() - t0)
        return new_state, rec

    def run(self, max_increments=None, on_increment=None, start_state=None):
        state = self.initial_state() if start_state is None else start_state
        n = self.load.n_increments if max_increments is None else min(self.load.n_increments, int(max_increments))
        records = []
        while state.increment < n:
            target = self.load.targets[state.increment]
            state, rec = self.advance(state, target)
            records.append(rec)
            if on_increment is not None:
                on_increment(state, rec)
        return state, records

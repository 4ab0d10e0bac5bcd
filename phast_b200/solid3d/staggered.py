"""3D solvers and the staggered increment on the GPU.

* ``pcg`` / ``solve_constrained`` -- Jacobi PCG with device flags on the free set
  (solid3d/linalg.py:99-287), the reference's signatures; with this backend's
  elastic action the whole constrained solve is one C-ABI call.
* ``solve_h8_scalar_box_kkt`` -- primal active-set box-KKT damage solve with a
  Dirichlet PCG per set and the KKT audit (solvers/box_kkt_h8.py:256-778).
* ``StaggeredSolver`` -- alternate minimisation of one load increment with
  ``history='max'`` and ``irreversibility='box_kkt'`` (solid3d/staggered.py:1207-1517).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math
from dataclasses import dataclass, field
from time import perf_counter

import numpy as np
import torch

from .. import _lib
from .._lib import ptr, raw, stream
from .model import unsupported_options


class PCGBreakdownError(RuntimeError):
    """Non-positive curvature, non-positive diagonal or non-finite values (linalg.py:41-42)."""


class PCGConvergenceError(RuntimeError):
    """Raised by callers that require convergence when PCG runs out of iterations (linalg.py:45-50)."""

    def __init__(self, message, info):
        super().__init__(message)
        self.info = info


@dataclass(frozen=True)
class BoxKKTFailureEvidence:
    """What a failed box-KKT solve had done (box_kkt_h8.py:226-234)."""
    reason: str
    active_set_iterations: int
    total_pcg_iterations: int


class H8ScalarBoxKKTConvergenceError(RuntimeError):
    """The active set did not stabilise or a PCG did not converge (box_kkt_h8.py:239-253)."""

    def __init__(self, reason, *, last_solution=None, last_linear_solve=None, evidence=None):
        super().__init__(reason)
        self.last_solution = last_solution
        self.last_linear_solve = last_linear_solve
        self.evidence = evidence


class StaggerConvergenceError(RuntimeError):
    """A load (sub-)increment could not be solved (solid3d/staggered.py:221-263).

    ``state`` is the last accepted state, ``target`` the controlled strain of the failed
    attempt, ``increment`` the 1-based load-case increment, ``cutbacks`` the halving depth,
    ``reason`` why the last attempt failed, ``attempts`` the attempts made for the increment
    and ``records`` the records accepted before the failure.
    """

    def __init__(self, message, *, state, target, increment, cutbacks, reason, attempts=1, records=()):
        super().__init__(message)
        self.state = state
        self.target = float(target)
        self.increment = int(increment)
        self.cutbacks = int(cutbacks)
        self.reason = str(reason)
        self.attempts = int(attempts)
        self.records = tuple(records)


@dataclass(frozen=True)
class PCGInfo:
    """Outcome of one PCG solve (linalg.py:53-68)."""
    iterations: int
    converged: bool
    rhs_norm: float
    residual_norm: float
    relative_residual: float


def _fused_target(action):
    """(op, g, d) when ``action`` is this backend's elastic action, else None.

    Recognised: the bound method ``op.mech_action`` (undamaged) and the callable of
    ``op.mech_operator(g, d=...)``.
    """
    from .operator import MechOperator, PeriodicVoxelPhaseFieldOperator
    if isinstance(action, MechOperator):
        return action.op, action.g, action.d
    if getattr(action, "__func__", None) is PeriodicVoxelPhaseFieldOperator.mech_action and \
            isinstance(getattr(action, "__self__", None), PeriodicVoxelPhaseFieldOperator):
        return action.__self__, None, None
    return None


def _check_settings(rtol, atol, maxiter, check_every):
    rtol, atol = float(rtol), float(atol)
    if not math.isfinite(rtol) or rtol < 0.0 or not math.isfinite(atol) or atol < 0.0:
        raise ValueError("rtol and atol must be finite and non-negative")
    if rtol == 0.0 and atol == 0.0:
        raise ValueError("rtol and atol must not both be zero")
    for name, value in (("maxiter", maxiter), ("check_every", check_every)):
        if isinstance(value, bool) or int(value) != value or int(value) < 1:
            raise ValueError(f"{name} must be an integer >= 1, got {value!r}")


def _vec(name, v, like=None):
    if not isinstance(v, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if v.ndim != 1:
        raise ValueError(f"{name} must be one-dimensional, got shape {tuple(v.shape)}")
    if v.dtype != torch.float64:
        raise TypeError(f"{name} must be float64, got {v.dtype}")
    if like is not None and (v.shape != like.shape or v.device != like.device):
        raise ValueError(f"{name} must have shape {tuple(like.shape)} on {like.device}")
    return v


def pcg(action, rhs, *, diag, x0=None, rtol=1.0e-8, atol=0.0, maxiter=5000, check_every=10):
    """Jacobi PCG for ``A x = rhs`` with an arbitrary matrix-free ``action`` (linalg.py:99-220).

    Stops when ``||r|| <= max(rtol ||b||, atol)``; the convergence and breakdown flags stay
    on the device and are read every ``check_every`` iterations.  Returns ``(x, PCGInfo)``;
    ``info.converged`` is False when ``maxiter`` is reached; breakdown raises
    :class:`PCGBreakdownError`.  The action is the caller's own code, so this loop drives it
    from the host with device vector updates; the staggered solver never takes this route
    (its solves are single fused C-ABI calls).
    """
    _check_settings(rtol, atol, maxiter, check_every)
    _vec("rhs", rhs)
    _vec("diag", diag, rhs)
    if x0 is not None:
        _vec("x0", x0, rhs)
    head = torch.stack((torch.linalg.vector_norm(rhs), torch.isfinite(rhs).all().double(),
                        (diag > 0).all().double(), torch.isfinite(diag).all().double())).tolist()
    b_norm = head[0]
    if head[1] < 1 or not math.isfinite(b_norm):
        raise PCGBreakdownError("PCG right-hand side contains a non-finite value")
    if head[3] < 1:
        raise PCGBreakdownError("PCG diagonal contains a non-finite value")
    if head[2] < 1:
        raise PCGBreakdownError("PCG diagonal has a non-positive entry (non-positive curvature)")
    if b_norm == 0.0:
        return torch.zeros_like(rhs), PCGInfo(0, True, 0.0, 0.0, 0.0)
    tol = max(rtol * b_norm, atol)
    if x0 is None:
        x, r, r_norm = torch.zeros_like(rhs), rhs.clone(), b_norm
    else:
        x = x0.clone()
        r = rhs - _vec("action(x0)", action(x), rhs)
        r_norm = float(torch.linalg.vector_norm(r))
        if not math.isfinite(r_norm):
            raise PCGBreakdownError("PCG initial residual is not finite")
    if r_norm <= tol:
        return x, PCGInfo(0, True, b_norm, r_norm, r_norm / b_norm)
    inv = 1.0 / diag
    z = r * inv
    p = z.clone()
    rz = torch.dot(r, z)
    tol2 = torch.tensor(tol * tol, dtype=torch.float64, device=rhs.device)
    running = torch.ones((), dtype=torch.bool, device=rhs.device)
    bad_curv = torch.zeros_like(running)
    bad_val = torch.zeros_like(running)
    steps = torch.zeros((), dtype=torch.float64, device=rhs.device)
    rr = torch.dot(r, r)
    for it in range(1, int(maxiter) + 1):
        Ap = action(p)
        pAp = torch.dot(p, Ap)
        curv = pAp > 0
        bad_curv |= running & ~curv
        bad_val |= ~torch.isfinite(pAp)
        take = running & curv
        alpha = torch.where(take, rz / torch.where(curv, pAp, torch.ones_like(pAp)), torch.zeros_like(pAp))
        x += alpha * p
        r -= alpha * Ap
        steps += take.double()
        z = r * inv
        rz_next = torch.dot(r, z)
        rr = torch.dot(r, r)
        bad_val |= ~(torch.isfinite(rz_next) & torch.isfinite(rr))
        running &= rr > tol2
        beta = torch.where(running & (rz > 0), rz_next / torch.where(rz > 0, rz, torch.ones_like(rz)),
                           torch.zeros_like(rz))
        p = z + beta * p
        rz = rz_next
        if it % int(check_every) == 0 or it == int(maxiter):
            f = torch.stack((bad_val.double(), bad_curv.double(), running.double(), rr, steps)).tolist()
            if f[0] > 0:
                raise PCGBreakdownError(f"PCG produced a non-finite value by iteration {it}")
            if f[1] > 0:
                raise PCGBreakdownError(f"PCG met non-positive curvature p.A p <= 0 by iteration {it}; "
                                        "the operator is not positive definite on the free set")
            r_norm = math.sqrt(f[3])
            if f[2] < 1:
                return x, PCGInfo(int(f[4]), True, b_norm, r_norm, r_norm / b_norm)
    return x, PCGInfo(int(maxiter), False, b_norm, r_norm, r_norm / b_norm)


def solve_constrained(action, *, diag, fixed_mask, fixed_values, rhs=None, x0=None, rtol=1.0e-8, atol=0.0,
                      maxiter=5000, check_every=10):
    """``A x = rhs`` with ``x = fixed_values`` on ``fixed_mask`` by projected Jacobi PCG (linalg.py:223-287).

    When ``action`` is this backend's elastic action (``op.mech_action`` or
    ``op.mech_operator(g, d=...)``) and ``rhs`` is None, the whole solve is one fused C-ABI
    call with the convergence flags on the device; any other action runs :func:`pcg` on the
    free set.  ``diag`` is the Jacobi diagonal (the fused solve forms its own, which is the
    same diagonal of the same operator).  Returns ``(x, PCGInfo)`` with
    ``x[fixed] == fixed_values[fixed]`` exactly.
    """
    _vec("fixed_values", fixed_values)
    n = fixed_values.shape[0]
    if not isinstance(fixed_mask, torch.Tensor) or fixed_mask.dtype != torch.bool:
        raise TypeError("fixed_mask must be a torch.bool tensor")
    if fixed_mask.shape != (n,) or fixed_mask.device != fixed_values.device:
        raise ValueError(f"fixed_mask must have shape ({n},) on {fixed_values.device}")
    _vec("diag", diag, fixed_values)
    if rhs is not None:
        _vec("rhs", rhs, fixed_values)
    if x0 is not None:
        _vec("x0", x0, fixed_values)
    _check_settings(rtol, atol, maxiter, check_every)
    target = _fused_target(action)
    if target is not None and rhs is None:
        op, g, d = target
        return _solve_fused(op, fixed_mask=fixed_mask, fixed_values=fixed_values, g=g, d=d, x0=x0, rtol=rtol,
                            atol=atol, maxiter=maxiter, check_every=check_every)
    free = ~fixed_mask
    zero = torch.zeros_like(fixed_values)
    x_c = torch.where(fixed_mask, fixed_values, zero)
    image = _vec("action(x_c)", action(x_c), fixed_values)
    b_f = torch.where(free, -image if rhs is None else rhs - image, zero)
    y, info = pcg(lambda v: torch.where(free, action(v), zero), b_f, diag=torch.where(free, diag, torch.ones_like(diag)),
                  x0=None if x0 is None else torch.where(free, x0, zero), rtol=rtol, atol=atol, maxiter=maxiter,
                  check_every=check_every)
    return torch.where(free, y, x_c), info


def _solve_fused(op, *, fixed_mask, fixed_values, g=None, d=None, x0=None, rtol=1e-8, atol=0.0, maxiter=5000,
                 check_every=10):
    """The constrained Jacobi PCG of the elastic action as one C-ABI call (FP64)."""
    n = op.n_mech
    mask = fixed_mask if fixed_mask.dtype == torch.uint8 else fixed_mask.to(torch.uint8).contiguous()
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
    plain = form.precond == "jacobi" and not form.mixed
    gq = None
    if getattr(op, "is_pfczm", False) and d is not None:
        # the PF-CZM degradation enters every operator as g (E, 8)
        gq = op.degradation(d).contiguous()
        if plain:
            return _solve_fused(op, fixed_mask=fixed_mask, fixed_values=fixed_values, g=gq, x0=x0, rtol=rtol,
                                atol=atol, maxiter=maxiter, check_every=check_every)
    if plain:
        return _solve_fused(op, fixed_mask=fixed_mask, fixed_values=fixed_values, d=d, x0=x0, rtol=rtol,
                            atol=atol, maxiter=maxiter, check_every=check_every)
    n = op.n_mech
    opts = form.struct()
    lib = _lib.load()
    nbytes = (lib.phastb_h8_mech_solve_ex_workspace_bytes(op.vgrid, opts) if gq is None
              else lib.phastb_h8_mech_solve_ex_g_workspace_bytes(op.vgrid, opts))
    if nbytes == 0:
        raise NotImplementedError(f"mechanics form {form} is not available for a {op.shape} grid "
                                  "(multigrid needs edges divisible by 2^(levels-1))")
    mask = fixed_mask if fixed_mask.dtype == torch.uint8 else fixed_mask.to(torch.uint8).contiguous()
    vals = fixed_values.to(torch.float64).contiguous()
    x0c = None if x0 is None else x0.to(torch.float64).contiguous()
    dd = (torch.zeros(op.n_red, dtype=torch.float64, device=op.device) if d is None
          else d.to(torch.float64).contiguous())
    out = torch.empty(n, dtype=torch.float64, device=op.device)
    info = (C.c_int * 2)()
    rinfo = (C.c_double * 2)()
    wp, wn = op._ws.get(nbytes)
    if gq is None:
        st = raw("phastb_h8_mech_solve_ex", op.vgrid, op.mat, ptr(op.slot), ptr(dd), ptr(mask), ptr(vals), ptr(x0c),
                 float(rtol), float(atol), int(maxiter), int(check_every), opts, lmax_cache, ptr(out), info, rinfo,
                 wp, wn, stream())
    else:
        st = raw("phastb_h8_mech_solve_ex_g", op.vgrid, op.mat, ptr(op.slot), ptr(gq), ptr(mask), ptr(vals),
                 ptr(x0c), float(rtol), float(atol), int(maxiter), int(check_every), opts, lmax_cache, ptr(out), info,
                 rinfo, wp, wn, stream())
    if st in (_lib.BREAKDOWN, _lib.NONFINITE):
        raise PCGBreakdownError(f"PCG breakdown (status {st})")
    if st not in (_lib.OK, _lib.NONCONVERGED):
        _lib.check(st, "phastb_h8_mech_solve_ex")
    bn, rn = float(rinfo[0]), float(rinfo[1])
    return out, PCGInfo(int(info[0]), bool(info[1]), bn, rn, rn / bn if bn > 0 else 0.0)


@dataclass(frozen=True)
class KKTDiagnostics:
    """The verdict of the KKT audit of a box-KKT solve (box_kkt_h8.py:165-191, ``satisfies_kkt``)."""
    satisfies_kkt: bool


@dataclass(frozen=True)
class BoxKKTResult:
    """A converged box-KKT damage field (box_kkt_h8.py:208-223): ``solution``, the iteration counts
    and the audit verdict (``satisfies_kkt``, also as ``kkt.satisfies_kkt``)."""
    solution: torch.Tensor
    total_pcg_iterations: int
    active_set_iterations: int
    satisfies_kkt: bool

    @property
    def kkt(self):
        return KKTDiagnostics(self.satisfies_kkt)


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
        reason = f"H8 scalar box-KKT failed after {info[1]} active-set iterations ({info[0]} PCG iterations)"
        raise H8ScalarBoxKKTConvergenceError(reason, last_solution=out,
                                             evidence=BoxKKTFailureEvidence(reason, int(info[1]), int(info[0])))
    _lib.check(st, "phastb_h8_damage_box_kkt")
    return BoxKKTResult(out, int(info[0]), int(info[1]), bool(info[2]))


@dataclass(eq=False)
class SolverState:
    """Accepted solution after ``step`` solves (solid3d/staggered.py:166-218).

    ``x = [u~, E]``, ``d`` the reduced nodal damage and ``H`` the (E, 8) history on the
    device; ``macro_strain`` and ``macro_stress`` (6,) float64 tensors held on the host
    (the solver reads them every increment); ``external_work`` in mJ; ``d_prev_step`` the
    lower bound that produced ``d``; ``increment`` the load-case increments completed.
    """
    step: int
    x: torch.Tensor
    d: torch.Tensor
    H: torch.Tensor
    macro_strain: torch.Tensor
    macro_stress: torch.Tensor
    external_work: float
    d_prev_step: torch.Tensor
    increment: int = 0

    def clone(self):
        return SolverState(int(self.step), self.x.clone(), self.d.clone(), self.H.clone(), self.macro_strain.clone(),
                           self.macro_stress.clone(), float(self.external_work), self.d_prev_step.clone(),
                           int(self.increment))

    def to(self, device):
        return SolverState(int(self.step), self.x.to(device), self.d.to(device), self.H.to(device),
                           self.macro_strain.clone(), self.macro_stress.clone(), float(self.external_work),
                           self.d_prev_step.to(device), int(self.increment))


CHECKPOINT_FORMAT = "phast.solid3d.checkpoint"
CHECKPOINT_VERSION = 1
_STATE_TENSORS = ("x", "d", "H", "macro_strain", "macro_stress", "d_prev_step")


def save_checkpoint(path, state, *, meta=None):
    """Write ``state`` and JSON-serialisable ``meta`` (solid3d/staggered.py:1638-1663).

    The file is the reference's checkpoint format, so either package resumes the other's
    runs: a ``torch.save`` dict with ``format``, ``version``, the state's scalars and its
    tensors on the CPU, and ``meta`` as a sorted JSON string; it is written beside the
    target and moved over it, so a crash never leaves a half-written checkpoint.
    """
    import json
    import os
    from pathlib import Path
    if not isinstance(state, SolverState):
        raise TypeError("state must be a SolverState")
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    body = {"step": int(state.step), "increment": int(state.increment), "external_work": float(state.external_work)}
    for name in _STATE_TENSORS:
        body[name] = getattr(state, name).detach().to("cpu", copy=True)
    payload = {"format": CHECKPOINT_FORMAT, "version": CHECKPOINT_VERSION, "state": body,
               "meta_json": json.dumps(dict(meta or {}), sort_keys=True)}
    tmp = path.with_name(path.name + ".tmp")
    torch.save(payload, tmp)
    os.replace(tmp, path)
    return path


def load_checkpoint(path, device="cpu"):
    """``(state, meta)`` from a checkpoint file (solid3d/staggered.py:1666-1690); the fields
    the solver keeps on the device go to ``device``, the macro strain and stress stay on the
    host as this package's states hold them."""
    import json
    from pathlib import Path
    target = torch.device(device)
    payload = torch.load(Path(path), map_location="cpu", weights_only=True)
    if not isinstance(payload, dict) or payload.get("format") != CHECKPOINT_FORMAT:
        raise ValueError(f"{path} is not a {CHECKPOINT_FORMAT} file")
    if payload.get("version") != CHECKPOINT_VERSION:
        raise ValueError(f"unsupported checkpoint version {payload.get('version')!r}")
    body = payload["state"]
    for name in _STATE_TENSORS:
        t = body.get(name)
        if not isinstance(t, torch.Tensor) or t.dtype != torch.float64:
            raise ValueError(f"checkpoint field {name!r} must be a float64 tensor")
    state = SolverState(step=int(body["step"]), x=body["x"].to(target), d=body["d"].to(target),
                        H=body["H"].to(target), macro_strain=body["macro_strain"].clone(),
                        macro_stress=body["macro_stress"].clone(), external_work=float(body["external_work"]),
                        d_prev_step=body["d_prev_step"].to(target), increment=int(body["increment"]))
    return state, json.loads(payload["meta_json"])


@dataclass(frozen=True)
class IncrementRecord:
    """Scalar record of one accepted load increment (solid3d/model.py:1234-1300), same fields.

    ``mech_s``, ``damage_s`` and ``history_s`` stay 0: the solver enqueues its device work
    asynchronously and does not stop to time the phases; ``wall_s`` is the increment's time.
    """
    step: int
    increment: int = 0
    load_factor: float = 0.0
    macro_strain: tuple = (0.0,) * 6
    macro_stress: tuple = (0.0,) * 6
    applied_disp: float = 0.0
    reaction_force: float = 0.0
    elastic: float = 0.0
    fracture: float = 0.0
    fracture_by_phase: dict = field(default_factory=dict)
    external: float = 0.0
    balance_residual: float = 0.0
    balance_residual_rel: float = 0.0
    max_damage: float = 0.0
    mean_damage: float = 0.0
    damaged_volume_fraction: float = 0.0
    max_H: float = 0.0
    stagger_iters: int = 0
    pcg_iters_mech: int = 0
    pcg_iters_pf: int = 0
    active_set_iters: int = 0
    cutbacks: int = 0
    converged: bool = True
    kkt_ok: bool = True
    stagger_change: float = 0.0
    mech_relative_residual: float = 0.0
    hill_mandel_rel: float = 0.0
    wall_s: float = 0.0
    mech_s: float = 0.0
    damage_s: float = 0.0
    history_s: float = 0.0
    mean_strain: tuple | None = None
    anderson_accepted: int | None = None
    anderson_rejected: int | None = None
    closure_solves: int | None = None
    min_normal_strain: float | None = None
    min_principal_strain: float | None = None
    min_det_F: float | None = None
    newton_iters_pf: int | None = None


class _AttemptFailure(Exception):
    """One attempt failed for a numerical reason (cut back or raise)."""


_TINY = 1.0e-300
_MIN_LINEAR_TOLERANCE = 4.0 * float(np.finfo(np.float64).eps)
_CLOSURE_MAX_SOLVES = 50            # INTERFACE_MAX_SOLVES, staggered.py:99
_CLOSURE_PATTERN_TOLERANCE = 1.0e-8  # staggered.py:105
_LS_ARMIJO = 1.0e-4                 # LINE_SEARCH_ARMIJO, staggered.py:109
_LS_ENERGY_RTOL = 1.0e-12           # staggered.py:112
_LS_MAX_HALVINGS = 30               # staggered.py:115
ANDERSON_REGULARISATION = 1.0e-10   # staggered.py:133
_ANDERSON_ENERGY_RTOL = 1.0e-12     # staggered.py:136


class ProjectedAnderson:
    """Type II Anderson mixing of the damage fixed point with a box projection (staggered.py:290-376):
    the last ``depth + 1`` pairs ``(d, G(d))`` in a device ring; a mix solves the regularised normal
    equations of the unit-norm residual differences and is clamped to ``[lower, upper]``.

    ``push(d_in, d_out)`` stores a pair, ``mix(lower, upper=1.0)`` returns the projected mix or
    ``None``; ``push_mix`` does both in one C-ABI call and also returns ``None`` for a mix equal
    to ``d_out``.
    """

    def __init__(self, depth, *, regularisation=ANDERSON_REGULARISATION, n=None, device="cuda"):
        if isinstance(depth, bool) or int(depth) != depth or not 1 <= int(depth) <= 6:
            raise ValueError(f"depth must be an integer in 1..6, got {depth!r}")
        if not (math.isfinite(regularisation) and regularisation >= 0.0):
            raise ValueError(f"regularisation must be finite and >= 0, got {regularisation!r}")
        self.depth = int(depth)
        self.regularisation = float(regularisation)
        self.device = torch.device(device)
        self._n = None if n is None else int(n)
        self._hist = None
        self._ws = _lib.Workspace(self.device)
        self.count = self.head = 0
        self._pending = None
        self._last_mix = None

    def __len__(self):
        return min(self.count + (self._pending is not None), self.depth + 1)

    def reset(self):
        """Forget every stored pair."""
        self.count = self.head = 0
        self._pending = None
        self._last_mix = None

    def _call(self, d_in, d_out, want, lower, upper):
        d_in = d_in.to(torch.float64).contiguous()
        d_out = d_out.to(torch.float64).contiguous()
        if self._hist is None:
            self._n = d_in.numel() if self._n is None else self._n
            self._hist = torch.empty(2 * (self.depth + 1) * self._n, dtype=torch.float64, device=self.device)
        if d_in.numel() != self._n or d_out.shape != d_in.shape:
            raise ValueError("d_in and d_out must be vectors of the cell's length")
        low = None
        if want:
            low = lower.to(torch.float64).contiguous() if isinstance(lower, torch.Tensor) else \
                torch.full((self._n,), float(lower), dtype=torch.float64, device=self.device)
        mixed = torch.empty_like(d_out) if want else None
        status = (C.c_int * 1)()
        wp, wn = self._ws.get(_lib.load().phastb_anderson_workspace_bytes(self.depth))
        _lib.call("phastb_anderson_projected", self._n, self.depth, self.count, self.head, ptr(self._hist),
                  ptr(d_in), ptr(d_out), int(bool(want)), ptr(low), float(upper), self.regularisation, ptr(mixed),
                  status, wp, wn, stream())
        self.head = (self.head + 1) % (self.depth + 1)
        self.count = min(self.count + 1, self.depth + 1)
        return mixed, int(status[0])

    def _flush(self):
        if self._pending is not None:
            self._call(*self._pending, False, None, 1.0)
            self._pending = None

    def push(self, d_in, d_out):
        """Store the pair ``(d_in, G(d_in))`` (copies; the oldest pair drops out at ``depth + 1``).
        The pair enters the device ring with the next ``mix`` or ``push``."""
        self._flush()
        self._pending = (d_in.detach().clone(), d_out.detach().clone())

    def mix(self, lower, upper=1.0):
        """Projected mixed iterate of the stored pairs, or ``None`` when no mix is defined (fewer than two
        pairs, every residual difference zero, a singular system or a non-finite mix)."""
        if self._pending is None:
            return self._last_mix
        mixed, status = self._call(*self._pending, True, lower, upper)
        self._pending = None
        self._last_mix = mixed if status in (1, 2) else None
        return self._last_mix

    def push_mix(self, d_in, d_out, lower, upper=1.0, *, mix=True):
        """Store the pair and return the projected mix, or ``None`` (no mix defined, or equal to d_out)."""
        self._flush()
        mixed, status = self._call(d_in, d_out, mix, lower, upper)
        return mixed if status == 1 else None


class StaggeredSolver:
    """Staggered hybrid AT2 solver of one periodic cell under mixed macro control (solid3d/staggered.py:391-1627).

    ``StaggeredSolver(op, load=None, cfg=None, *, form=PLAIN)``: ``load`` and ``cfg`` default to
    the operator's; ``form`` selects how the mechanics systems are solved (``MechForm``: the
    reference's Jacobi PCG in FP64 by default, or multigrid and/or FP32 under FP64 refinement
    to the same FP64 stopping rule).  Attributes ``op, load, cfg, last_state, n_attempts,
    n_failed_attempts`` as the reference.
    """

    def __init__(self, op, load=None, cfg=None, *, form=PLAIN):
        from .operator import PeriodicVoxelPhaseFieldOperator
        if not isinstance(op, PeriodicVoxelPhaseFieldOperator):
            raise TypeError("op must be a PeriodicVoxelPhaseFieldOperator")
        load = op.load if load is None else load
        cfg = op.cfg if cfg is None else cfg
        if (int(load.controlled), set(load.free), set(load.fixed_zero)) != \
                (int(op.load.controlled), set(op.load.free), set(op.load.fixed_zero)):
            raise ValueError("load must control, free and fix the same components as op.load")
        for key in ("kappa", "energy_split_isotropic", "energy_split_band", "band_stress", "dtype", "crack_closure",
                    "damage_law"):
            if getattr(cfg, key, None) != getattr(op.cfg, key, None):
                raise ValueError(f"cfg.{key} must match the operator's ({getattr(op.cfg, key, None)!r})")
        bad = unsupported_options(cfg)
        if bad:
            raise NotImplementedError(f"the B200 backend does not run {', '.join(bad)}")
        if op.has_closure and cfg.anderson_depth > 0:
            raise ValueError("Anderson mixing (anderson_depth > 0) is not available with crack_closure 'axes'")
        if op.has_closure and (form.precond != "jacobi" or form.mixed):
            raise NotImplementedError("crack_closure 'axes' runs the plain FP64 mechanics form only")
        self.op = op
        self.load = load
        self.cfg = cfg
        self.form = form
        self.device = op.device
        self.dtype = torch.float64
        self.last_state = None
        self.n_attempts = 0
        self.n_failed_attempts = 0
        self._lmax = (C.c_double * 3)()
        self.lmax_every = 10
        self._c = int(load.controlled)
        self._n_u = 3 * op.n_red
        self._max_abs_target = max(abs(float(t)) for t in load.targets)
        self._u_floor = min(op.h) * math.sqrt(self._n_u)
        self._mask = op.mech_fixed_mask()
        self._mask_u8 = self._mask.to(torch.uint8).contiguous()
        self._zeros = torch.zeros(op.n_mech, dtype=torch.float64, device=op.device)
        self._red = _lib.Workspace(op.device)
        self._pfws = _lib.Workspace(op.device)
        self._clws = _lib.Workspace(op.device)
        self._neg_inf = None
        self.last_bound_violations = None
        self.last_interface_solves = 0
        self.last_line_search_steps = 0
        self._newton_count = 0
        self.last_newton_iters = None
        lengths = tuple(n * h for n, h in zip(op.shape, op.h))
        axis = self._c if self._c < 3 else 0
        others = tuple(lengths[a] for a in range(3) if a != axis)
        self._load_axis, self._load_length, self._face = axis, lengths[axis], others[0] * others[1]

    # -- states ----------------------------------------------------------------------------
    def initial_state(self):
        """Undamaged, unloaded state at step 0."""
        op = self.op
        z = lambda *s: torch.zeros(*s, dtype=torch.float64, device=op.device)  # noqa: E731
        host = lambda: torch.zeros(6, dtype=torch.float64)  # noqa: E731
        return SolverState(0, z(op.n_mech), z(op.n_red), z(op.n_elements, 8), host(), host(), 0.0, z(op.n_red), 0)

    def initial_record(self):
        """The step-0 zero row (every present phase listed with zero fracture energy)."""
        return IncrementRecord(step=0, fracture_by_phase={p.name: 0.0 for p in self.op.phases})

    def _check_state(self, state):
        if not isinstance(state, SolverState):
            raise TypeError("state must be a SolverState")
        op = self.op
        for name, shape in (("x", (op.n_mech,)), ("d", (op.n_red,)), ("H", (op.n_elements, 8)),
                            ("d_prev_step", (op.n_red,))):
            t = getattr(state, name)
            if not isinstance(t, torch.Tensor) or tuple(t.shape) != shape or t.dtype != torch.float64 or \
                    t.device != op.device:
                raise ValueError(f"state.{name} must be a float64 {shape} tensor on {op.device}")

    # -- pieces of one staggered iteration --------------------------------------------------
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
        if self.op.has_closure:
            return self._closure_mechanics(d, values, x0)
        cfg = self.cfg
        try:
            x, info = solve_constrained_form(self.op, self.form, fixed_mask=self._mask_u8, fixed_values=values, d=d,
                                             x0=x0, rtol=cfg.pcg_rtol_mech, maxiter=cfg.pcg_maxit_mech,
                                             check_every=cfg.check_every, lmax_cache=self._lmax)
        except PCGBreakdownError as exc:
            raise _AttemptFailure(f"mechanics PCG breakdown: {exc}") from exc
        if not info.converged:
            raise _AttemptFailure(f"mechanics PCG did not converge in {cfg.pcg_maxit_mech} iterations")
        return x, info

    def _linear_closure(self, g, pattern, values, x0):
        """The mechanics solve of one closure pattern (StaggeredSolver._linear_mechanics,
        staggered.py:550-587): the constrained Jacobi PCG with the add-back of ``pattern``."""
        op, cfg = self.op, self.cfg
        out = torch.empty(op.n_mech, dtype=torch.float64, device=op.device)
        info = (C.c_int * 2)()
        rinfo = (C.c_double * 2)()
        wp, wn = self._clws.get(_lib.load().phastb_h8_mech_solve_closure_workspace_bytes(op.vgrid))
        st = raw("phastb_h8_mech_solve_closure", op.vgrid, op.mat, ptr(op.slot), ptr(g), ptr(pattern),
                 ptr(self._mask_u8), ptr(values), ptr(x0), float(cfg.pcg_rtol_mech), 0.0, int(cfg.pcg_maxit_mech),
                 int(cfg.check_every), ptr(out), info, rinfo, wp, wn, stream())
        if st in (_lib.BREAKDOWN, _lib.NONFINITE):
            raise _AttemptFailure(f"mechanics PCG breakdown: PCG breakdown (status {st})")
        if st not in (_lib.OK, _lib.NONCONVERGED):
            _lib.check(st, "phastb_h8_mech_solve_closure")
        bn, rn = float(rinfo[0]), float(rinfo[1])
        pinfo = PCGInfo(int(info[0]), bool(info[1]), bn, rn, rn / bn if bn > 0 else 0.0)
        if not pinfo.converged:
            raise _AttemptFailure(f"mechanics PCG did not converge in {cfg.pcg_maxit_mech} iterations "
                                  f"(relative residual {pinfo.relative_residual:.3e} > {cfg.pcg_rtol_mech:.3e})")
        return out, pinfo

    def _energy_line_search(self, x, y, g):
        """Damped step from ``x`` towards the pattern solution ``y`` (staggered.py:589-626): alpha halved
        from 1 until the degraded energy (each point at its own signs) meets the Armijo test with the
        round-off allowance of ``|energy(x)|``; ``alpha = 1`` returns ``y`` itself."""
        op = self.op
        p = y - x
        energy0 = float(op.elastic_energy(x, g))
        force = op.mech_action(x, g)
        free = ~self._mask
        slope = min(float(torch.dot(force[free], p[free])), 0.0)
        allowance = _LS_ENERGY_RTOL * abs(energy0)
        alpha = 1.0
        for _ in range(_LS_MAX_HALVINGS + 1):
            trial = y if alpha == 1.0 else x + alpha * p
            energy = float(op.elastic_energy(trial, g))
            if not math.isfinite(energy):
                raise _AttemptFailure("mechanics energy is not finite in the line search")
            if energy <= energy0 + _LS_ARMIJO * alpha * slope + allowance:
                return trial, alpha
            alpha *= 0.5
        raise _AttemptFailure(f"the energy line search of the closure mechanics solve found no decrease in "
                              f"{_LS_MAX_HALVINGS} halvings")

    def _closure_mechanics(self, d, values, x0):
        """Line-searched active-set mechanics solve over the closure pattern (staggered.py:698-751):
        start from the pattern of ``x0``, solve the linear system of the pattern, take the energy line
        search towards it, and stop when no bit flips materially after a full step (at most
        50 solves).  ``last_interface_solves`` records the solves."""
        op = self.op
        g = op.degradation(d)
        pattern = op._closure_pattern_packed(x0)
        iterations = 0
        damped = 0
        for solve in range(1, _CLOSURE_MAX_SOLVES + 1):
            y, info = self._linear_closure(g, pattern, values, x0)
            iterations += info.iterations
            x, alpha = self._energy_line_search(x0, y, g)
            damped += int(alpha < 1.0)
            pattern, changed = op._closure_change_packed(x, pattern, g, _CLOSURE_PATTERN_TOLERANCE)
            if not changed and alpha == 1.0:
                self.last_interface_solves = solve
                self.last_line_search_steps = damped
                return x, dataclasses.replace(info, iterations=iterations)
            x0 = x
        raise _AttemptFailure("the closure pattern (crack_closure 'axes'), with the opening pattern of the interface "
                              f"elements where present, did not settle in {_CLOSURE_MAX_SOLVES} mechanics solves")

    def _damage(self, H, lower, initial):
        """(d, PCG iterations, active-set iterations, kkt_ok) of the box-KKT damage solve, or of the
        unbounded Dirichlet PCG with ``irreversibility='history_only'`` (staggered.py:753-841)."""
        if self.op.is_pfczm:
            return self._damage_pfczm(H, lower, initial)
        cfg, op = self.cfg, self.op
        r0 = op.damage_residual_norm(H, initial)
        if not math.isfinite(r0):
            raise _AttemptFailure("damage residual is not finite")
        # the PCG stops at tol * max(||r0||, 1) while the KKT audit is absolute
        tol = max(min(cfg.damage_linear_tol, 0.1 * cfg.damage_kkt_tol / max(r0, 1.0)), _MIN_LINEAR_TOLERANCE)
        if cfg.irreversibility == "history_only":
            return self._damage_history_only(H, lower, initial, tol)
        # the bounds hold by construction: lower is the accepted damage of the last
        # increment (in [0, 1]) and initial is lower itself or a box-KKT solution
        try:
            res = solve_h8_scalar_box_kkt(op.damage_system(H), lower_bound=lower, upper_bound=1.0, initial=initial,
                                          linear_tolerance=tol, kkt_tolerance=cfg.damage_kkt_tol,
                                          max_linear_iterations=cfg.damage_maxit,
                                          max_active_set_iterations=cfg.damage_max_active_set,
                                          check_bounds=False)
        except H8ScalarBoxKKTConvergenceError as exc:
            raise _AttemptFailure(f"damage box-KKT solve failed: {exc}") from exc
        except RuntimeError as exc:
            raise _AttemptFailure(f"damage PCG breakdown: {exc}") from exc
        return res.solution, res.total_pcg_iterations, res.active_set_iterations, res.satisfies_kkt

    def _damage_history_only(self, H, lower, initial, tol):
        """The damage system solved without bounds (one Dirichlet PCG with nothing fixed: the box
        solve with infinite bounds), then the bound-violation statistics (staggered.py:801-841)."""
        cfg, op = self.cfg, self.op
        if self._neg_inf is None:
            self._neg_inf = torch.full((op.n_red,), -math.inf, dtype=torch.float64, device=op.device)
        try:
            res = solve_h8_scalar_box_kkt(op.damage_system(H), lower_bound=self._neg_inf, upper_bound=math.inf,
                                          initial=initial, linear_tolerance=tol, kkt_tolerance=math.inf,
                                          max_linear_iterations=cfg.damage_maxit, max_active_set_iterations=1,
                                          check_bounds=False)
        except H8ScalarBoxKKTConvergenceError as exc:
            raise _AttemptFailure(f"damage PCG did not converge in {cfg.damage_maxit} iterations") from exc
        except RuntimeError as exc:
            raise _AttemptFailure(f"damage PCG breakdown: {exc}") from exc
        d = res.solution
        stats = torch.stack(((d < lower).sum().to(torch.float64), (d < 0.0).sum().to(torch.float64),
                             (d > 1.0).sum().to(torch.float64), torch.clamp_min(lower - d, 0.0).max(),
                             torch.clamp_min(d - 1.0, 0.0).max())).cpu()
        self.last_bound_violations = {"below_previous": int(stats[0]), "below_zero": int(stats[1]),
                                      "above_one": int(stats[2]), "max_decrease": float(stats[3]),
                                      "max_excess_over_one": float(stats[4])}
        kkt_ok = int(stats[0]) == 0 and int(stats[1]) == 0 and int(stats[2]) == 0
        return d, res.total_pcg_iterations, 0, kkt_ok

    def _damage_pfczm(self, H, lower, initial):
        """Projected Newton solve of the PF-CZM damage energy over ``lower <= d <= 1``
        (StaggeredSolver._damage_pfczm, staggered.py:843-1096), the whole loop in one C-ABI call:
        box-QP of the tangent per step (the box-KKT engine at damage_kkt_tol / 10), Armijo line
        search with step halving, projected step doubling after a full step.  Returns
        ``(d, pcg iterations, active-set iterations, True)``; failures raise ``_AttemptFailure``."""
        op, cfg = self.op, self.cfg
        out = torch.empty(op.n_red, dtype=torch.float64, device=op.device)
        info = (C.c_int * 4)()
        rinfo = (C.c_double * 2)()
        wp, wn = self._pfws.get(_lib.load().phastb_h8_pfczm_solve_workspace_bytes(op.vgrid))
        st = raw("phastb_h8_pfczm_damage_solve", op.vgrid, op.mat, C.byref(op._pf), ptr(op.slot), ptr(H),
                 float(op.damage_scale), ptr(lower), ptr(initial), float(cfg.damage_kkt_tol),
                 float(cfg.damage_linear_tol), int(cfg.damage_maxit), int(cfg.damage_max_active_set),
                 int(cfg.pfczm_max_newton), ptr(out), info, rinfo, wp, wn, stream())
        pcg, sets, its, reason = (int(v) for v in info)
        if st not in (_lib.OK, _lib.NONCONVERGED, _lib.BREAKDOWN, _lib.NONFINITE):
            _lib.check(st, "phastb_h8_pfczm_damage_solve")
        if st != _lib.OK:
            if reason == 1:
                msg = "damage PF-CZM energy is not finite"
            elif reason == 2:
                msg = "damage PF-CZM gradient is not finite"
            elif reason == 3 and st in (_lib.BREAKDOWN, _lib.NONFINITE):
                msg = f"damage PF-CZM Newton subproblem PCG breakdown (status {st})"
            elif reason == 3:
                msg = (f"damage PF-CZM Newton subproblem failed at Newton iteration {its + 1}: H8 scalar box-KKT "
                       f"failed ({pcg} PCG iterations, {sets} active-set iterations in total)")
            elif reason == 4:
                msg = (f"damage PF-CZM line search failed at Newton iteration {its + 1} "
                       "(no decrease after 30 halvings)")
            else:
                msg = (f"damage PF-CZM Newton did not converge in {cfg.pfczm_max_newton} iterations "
                       f"(projected gradient {rinfo[0]:.3e} > damage_kkt_tol {cfg.damage_kkt_tol:.3e})")
            raise _AttemptFailure(msg)
        self.last_newton_iters = its
        self._newton_count += its
        return out, pcg, sets, True

    def _predictor(self, state, previous, target):
        """x * (target / previous) with E[c] = target; zero start from an unloaded state (staggered.py:1207-1213)."""
        x = torch.empty_like(state.x)
        _lib.call("phastb_scale_set", self.op.n_mech, ptr(state.x), target / previous if previous != 0.0 else 0.0,
                  self._n_u + self._c, float(target), ptr(x), stream())
        return x

    # -- one attempt -------------------------------------------------------------------------
    def advance(self, state, target, *, increment=None, cutbacks=0):
        """Solve one (sub-)increment from ``state`` to ``E_c = target``, a single attempt (staggered.py:1215-1257).

        Raises :class:`StaggerConvergenceError` (no cutback) on failure.
        """
        self._check_state(state)
        target = float(target)
        if not math.isfinite(target):
            raise ValueError(f"target must be finite, got {target!r}")
        previous = float(state.macro_strain[self._c])
        if target == previous:
            raise ValueError(f"target {target!r} equals the current controlled strain")
        increment = state.increment + 1 if increment is None else int(increment)
        self.n_attempts += 1
        t0 = perf_counter()
        # lambda_max of the Jacobi-scaled operator barely moves with the damage
        # field; the multigrid re-estimates it every `lmax_every` increments
        if (increment - 1) % self.lmax_every == 0 and cutbacks == 0:
            self._lmax[0] = 0.0
        try:
            new_state, record = self._attempt(state, target, previous, increment, int(cutbacks), t0)
        except _AttemptFailure as exc:
            self.n_failed_attempts += 1
            raise StaggerConvergenceError(
                f"increment {increment} (cutback level {cutbacks}) to E[{self._c}] = {target:.6e} failed: {exc}",
                state=state, target=target, increment=increment, cutbacks=int(cutbacks), reason=str(exc)) from exc
        self.last_state = new_state
        return new_state, record

    def _attempt(self, state, target, previous, increment, cutbacks, t0):
        op, cfg = self.op, self.cfg
        self._newton_count = 0
        # mech_fixed_values(target) as one kernel: zero except E[controlled] = target
        values = torch.empty(op.n_mech, dtype=torch.float64, device=op.device)
        _lib.call("phastb_scale_set", op.n_mech, ptr(self._zeros), 0.0, self._n_u + self._c, float(target), ptr(values),
                  stream())
        step_size = abs(target - previous)
        x_old = self._predictor(state, previous, target)
        d_old = state.d.clone()
        lower = state.d
        pm = pp = sets = 0
        kkt = True
        H = state.H
        change = math.inf
        converged = False
        info = None
        closure = op.has_closure
        closure_solves = 0
        # Anderson mixing: a fresh history for every attempt; a mixed input is judged by its own
        # iteration against the plain iterate it replaced (staggered.py:1282-1400)
        anderson = ProjectedAnderson(cfg.anderson_depth, n=op.n_red, device=op.device) \
            if cfg.anderson_depth > 0 else None
        best_energy = math.inf
        n_accepted = n_rejected = 0
        fallback = None
        for k in range(1, cfg.max_stagger + 1):
            try:
                x_new, info = self._mechanics(d_old, values, x_old)
                pm += info.iterations
                if closure:
                    closure_solves += self.last_interface_solves
                H = op.driving_history(x_new, state.H if cfg.history == "max" else None)[1]
                d_new, its, s, kkt = self._damage(H, lower, d_old)
                pp += its
                sets += s
                change = self._change(x_new, x_old, d_new, d_old, step_size)
            except _AttemptFailure:
                if fallback is None:
                    raise
                # the iteration from a mixed input failed: return to the plain iterate
                n_rejected += 1
                x_old, d_old = fallback[1], fallback[0]
                fallback = None
                anderson.reset()
                continue
            rejected = False
            residual = None
            if anderson is not None:
                residual = float(torch.linalg.vector_norm(d_new - d_old))
                rec = op.increment_record(x_new, d_new, None, cfg.damaged_threshold)
                total = rec["energy"] + rec["local"] + rec["gradient"]
                if fallback is not None:
                    # the end-of-iteration total energy must not rise above the lowest of the
                    # attempt, and the fixed-point residual not above the replaced iteration's
                    rejected = (total > best_energy + _ANDERSON_ENERGY_RTOL * abs(best_energy)) or \
                        (residual > fallback[2])
                    if rejected:
                        n_rejected += 1
                    else:
                        n_accepted += 1
                if not rejected:
                    best_energy = min(best_energy, total)
            if rejected:
                x_old, d_old = fallback[1], fallback[0]
                fallback = None
                anderson.reset()
                continue
            fallback = None
            if change <= cfg.stagger_tol and k >= cfg.min_stagger:
                x_old, d_old = x_new, d_new
                converged = True
                break
            if anderson is not None:
                mixed = anderson.push_mix(d_old, d_new, lower, mix=k >= cfg.anderson_start)
                if mixed is not None:
                    fallback = (d_new, x_new, residual)
                    x_old, d_old = x_new, mixed
                    continue
            x_old, d_old = x_new, d_new
        if not converged:
            raise _AttemptFailure(f"staggered iteration did not converge in {cfg.max_stagger} iterations "
                                  f"(change {change:.3e} > stagger_tol {cfg.stagger_tol:.3e})")
        d = d_old
        if cfg.final_mechanics_resolve:
            x, info = self._mechanics(d, values, x_old)
            pm += info.iterations
            if closure:
                closure_solves += self.last_interface_solves
        else:
            x = x_old
        # every scalar of the record in one kernel pair and one host read
        rec = op.increment_record(x, d, H, cfg.damaged_threshold)
        E = rec["E"]
        sigma = rec["rE"] / op.volume
        elastic = rec["energy"]
        fracture = rec["local"] + rec["gradient"]
        scalars = np.concatenate([E, sigma, [elastic, fracture, rec["max_d"], rec["max_H"]]])
        if not np.isfinite(scalars).all():
            raise _AttemptFailure("accepted state has non-finite stress, strain or energy")
        closure_record = {}
        if closure:
            # the closure solves of the increment and the kinematic guard of the accepted state
            guard = op.kinematic_guard(x, d)
            closure_record = {"closure_solves": int(closure_solves), "min_normal_strain": guard["min_normal_strain"],
                              "min_principal_strain": guard["min_principal_strain"],
                              "min_det_F": guard["min_det_F"]}
        mean_work = 2.0 * elastic / op.volume
        macro_work = float(np.dot(sigma, E))
        scale = max(abs(mean_work), abs(macro_work))
        hill_rel = abs(mean_work - macro_work) / scale if scale > 0 else 0.0
        c = self._c
        external = state.external_work + op.volume * 0.5 * (sigma[c] + float(state.macro_stress[c])) * \
            (target - previous)
        residual = external - (elastic + fracture)
        completes = 1 <= increment <= self.load.n_increments and target == self.load.targets[increment - 1]
        new_state = SolverState(state.step + 1, x, d, H, torch.as_tensor(E.copy()), torch.as_tensor(sigma.copy()),
                                float(external), state.d, increment if completes else state.increment)
        macro_strain = tuple(float(v) for v in E)
        macro_stress = tuple(float(v) for v in sigma)
        record = IncrementRecord(
            step=new_state.step, increment=increment, load_factor=target / self._max_abs_target,
            macro_strain=macro_strain, macro_stress=macro_stress,
            applied_disp=macro_strain[self._load_axis] * self._load_length,
            reaction_force=macro_stress[self._load_axis] * self._face, elastic=float(elastic),
            fracture=float(fracture), fracture_by_phase=dict(rec["by_phase"]), external=float(external),
            balance_residual=float(residual), balance_residual_rel=float(residual / max(abs(external), _TINY)),
            max_damage=float(rec["max_d"]), mean_damage=float(rec["sum_element_d"] / op.n_elements),
            damaged_volume_fraction=float(rec["damaged"] / op.n_elements), max_H=float(rec["max_H"]),
            stagger_iters=k, pcg_iters_mech=pm, pcg_iters_pf=pp, active_set_iters=sets, cutbacks=int(cutbacks),
            converged=True, kkt_ok=bool(kkt), stagger_change=float(change),
            mech_relative_residual=float(info.relative_residual), hill_mandel_rel=float(hill_rel),
            wall_s=perf_counter() - t0, mean_strain=macro_strain,
            newton_iters_pf=self._newton_count if op.is_pfczm else None,
            anderson_accepted=n_accepted if anderson is not None else None,
            anderson_rejected=n_rejected if anderson is not None else None, **closure_record)
        return new_state, record

    # -- increments with cutback, and the load path -------------------------------------------
    def advance_increment(self, state, target, *, increment=None, on_increment=None):
        """One load-case increment with recursive half-step cutback (staggered.py:1523-1582).

        A failed attempt with ``on_stagger_failure='cutback'`` splits the remaining
        interval into two halves, each solved the same way, down to ``max_cutbacks``
        levels; deeper failures (or any failure with ``'raise'``) raise
        :class:`StaggerConvergenceError` with the last accepted state and the sub-steps
        accepted so far.  ``on_increment(state, record)`` follows every accepted sub-step.
        Returns ``(state, records)``.
        """
        increment = state.increment + 1 if increment is None else int(increment)
        target = float(target)
        accepted, latest, attempts = [], [state], [0]

        def solve(current, end, depth):
            attempts[0] += 1
            try:
                new_state, record = self.advance(current, end, increment=increment, cutbacks=depth)
            except StaggerConvergenceError as exc:
                if self.cfg.on_stagger_failure == "raise" or depth >= self.cfg.max_cutbacks:
                    raise StaggerConvergenceError(
                        f"increment {increment} to E[{self._c}] = {target:.6e} failed at cutback level {depth} "
                        f"(max_cutbacks={self.cfg.max_cutbacks}, on_stagger_failure="
                        f"{self.cfg.on_stagger_failure!r}): {exc.reason}",
                        state=latest[0], target=end, increment=increment, cutbacks=depth, reason=exc.reason,
                        attempts=attempts[0], records=tuple(accepted)) from exc
                middle = 0.5 * (float(current.macro_strain[self._c]) + end)
                current = solve(current, middle, depth + 1)
                return solve(current, end, depth + 1)
            accepted.append(record)
            latest[0] = new_state
            if on_increment is not None:
                on_increment(new_state, record)
            return new_state

        final = solve(state, target, 0)
        if final.increment != increment:
            final = dataclasses.replace(final, increment=increment)
            self.last_state = final
        return final, accepted

    def run(self, *, start_state=None, max_increments=None, on_increment=None):
        """Follow the load path from ``start_state`` (default the initial state), solving increments
        ``start_state.increment + 1, ...`` (at most ``max_increments``); returns every accepted record
        in order, the final state is ``last_state`` (staggered.py:1584-1636)."""
        state = self.initial_state() if start_state is None else start_state
        self._check_state(state)
        self.last_state = state
        first = int(state.increment)
        last = self.load.n_increments
        if max_increments is not None:
            if isinstance(max_increments, bool) or int(max_increments) != max_increments or max_increments < 0:
                raise ValueError(f"max_increments must be an integer >= 0, got {max_increments!r}")
            last = min(last, first + int(max_increments))
        records = []

        def accepted(new_state, record):
            records.append(record)
            if on_increment is not None:
                on_increment(new_state, record)

        for index in range(first, last):
            try:
                state, _ = self.advance_increment(state, self.load.targets[index], increment=index + 1,
                                                  on_increment=accepted)
            except StaggerConvergenceError as exc:
                exc.records = tuple(records)
                self.last_state = exc.state
                raise
        self.last_state = state
        return records

"""Anderson mixing (type II) of the 2D staggered damage fixed point in numpy.

TEST ORACLE ONLY.  Restates PhAST's ``_AndersonAccelerator`` (src/phast/solvers/
staggered_solver.py:165-255): the history of the last depth + 1 pairs (d_in, G(d_in)),
the regularised normal equations of the residual differences, the extrapolated field,
the 1.5x residual safeguard and the clamp to [floor, 1].
"""
from __future__ import annotations

from collections import deque

import numpy as np


class AndersonAccelerator:
    def __init__(self, m=5, reg=1e-10):
        self.m, self.reg = m, reg
        self.g_hist = deque(maxlen=m + 1)
        self.f_hist = deque(maxlen=m + 1)

    def reset(self):
        self.g_hist.clear()
        self.f_hist.clear()

    def step(self, d_in, d_out, floor=None):
        """The mixed field (staggered_solver.py:194-255)."""
        f = d_out - d_in
        self.g_hist.append(d_out.copy())
        self.f_hist.append(f.copy())
        mk = len(self.f_hist) - 1
        if mk == 0:
            return d_out
        dF = np.stack([self.f_hist[i + 1] - self.f_hist[i] for i in range(mk)], axis=1)
        FtF = dF.T @ dF + self.reg * np.eye(mk)
        Ftf = dF.T @ self.f_hist[-1]
        try:
            gamma = np.linalg.solve(FtF, Ftf)
        except np.linalg.LinAlgError:
            return d_out
        dG = np.stack([self.g_hist[i + 1] - self.g_hist[i] for i in range(mk)], axis=1)
        d_aa = d_out - dG @ gamma
        if np.linalg.norm(d_aa - d_in) > 1.5 * np.linalg.norm(f):
            return d_out
        d_aa = np.maximum(d_aa, floor) if floor is not None else np.maximum(d_aa, 0.0)
        return np.minimum(d_aa, 1.0)


class ProjectedAnderson:
    """ProjectedAnderson (solid3d/staggered.py:290-376): unit-norm residual differences, relative
    regularisation 1e-10, projection onto [lower, upper], no safeguard (the caller judges)."""

    def __init__(self, depth, reg=1e-10):
        self.depth, self.reg = depth, reg
        self.ins = deque(maxlen=depth + 1)
        self.outs = deque(maxlen=depth + 1)

    def reset(self):
        self.ins.clear()
        self.outs.clear()

    def push(self, d_in, d_out):
        self.ins.append(d_in.copy())
        self.outs.append(d_out.copy())

    def mix(self, lower, upper=1.0):
        if len(self.ins) < 2:
            return None
        res = [o - i for i, o in zip(self.ins, self.outs)]
        outs = list(self.outs)
        dF = np.stack([res[i + 1] - res[i] for i in range(len(res) - 1)], axis=1)
        dG = np.stack([outs[i + 1] - outs[i] for i in range(len(outs) - 1)], axis=1)
        scale = np.linalg.norm(dF, axis=0)
        keep = scale > 0.0
        if not keep.any():
            return None
        dF, dG, scale = dF[:, keep], dG[:, keep], scale[keep]
        A = dF / scale
        normal = A.T @ A + self.reg * np.eye(A.shape[1])
        try:
            beta = np.linalg.solve(normal, A.T @ res[-1])
        except np.linalg.LinAlgError:
            return None
        mixed = outs[-1] - dG @ (beta / scale)
        if not np.isfinite(mixed).all():
            return None
        return np.minimum(np.maximum(mixed, lower), upper)


def increment_anderson(op, cfg, x, d, H_prev, previous, target, depth, start=2):
    """One staggered _attempt of the AT2 cell with projected Anderson mixing
    (staggered.py:1282-1400): returns (x, d, stagger_iters, pcg_mech, pcg_pf, accepted, rejected)."""
    import math as _m
    from . import h8
    nu = 3 * op.n_red
    x_old = x * (target / previous) if previous != 0.0 else np.zeros_like(x)
    x_old[nu + op.controlled] = target
    d_old = d.copy()
    lower = d
    values = op.fixed_values(target)
    mask = op.fixed_mask()
    step = abs(target - previous)
    u_floor = min(op.h) * _m.sqrt(nu)
    pm = pp = 0
    aa = ProjectedAnderson(depth)
    best = _m.inf
    acc = rej = 0
    fallback = None
    for k in range(1, cfg.max_stagger + 1):
        g = op.degradation(d_old)
        x_new, its, conv, _, _ = h8.solve_constrained(lambda v: op.mech_action(v, g), op.mech_diagonal(g), mask,
                                                      values, x0=x_old, rtol=cfg.pcg_rtol_mech,
                                                      maxiter=cfg.pcg_maxit_mech, check_every=cfg.check_every)
        pm += its
        H = np.maximum(H_prev, op.driving_force(x_new))
        d_new, its = h8._damage_at2(op, cfg, H, lower, d_old)
        pp += its
        du = float(np.linalg.norm(x_new[:nu] - x_old[:nu]))
        un = float(np.linalg.norm(x_new[:nu]))
        dE = float(np.abs(x_new[nu:] - x_old[nu:]).max())
        sE = max(float(np.abs(x_new[nu:]).max()), step)
        uref = max(un, sE * u_floor)
        change = max(du / uref if uref > 0 else 0.0, dE / sE if sE > 0 else 0.0, float(np.abs(d_new - d_old).max()))
        residual = float(np.linalg.norm(d_new - d_old))
        total = op.elastic_energy(x_new, op.degradation(d_new)) + op.fracture_energy(d_new)
        rejected = False
        if fallback is not None:
            rejected = total > best + 1e-12 * abs(best) or residual > fallback[2]
            rej += int(rejected)
            acc += int(not rejected)
        if not rejected:
            best = min(best, total)
        if rejected:
            d_old, x_old = fallback[0], fallback[1]
            fallback = None
            aa.reset()
            continue
        fallback = None
        if change <= cfg.stagger_tol and k >= cfg.min_stagger:
            return x_new, d_new, k, pm, pp, acc, rej
        aa.push(d_old, d_new)
        mixed = aa.mix(lower) if k >= start else None
        if mixed is not None and not np.array_equal(mixed, d_new):
            fallback = (d_new, x_new, residual)
            x_old, d_old = x_new, mixed
            continue
        x_old, d_old = x_new, d_new
    raise RuntimeError("stagger did not converge")

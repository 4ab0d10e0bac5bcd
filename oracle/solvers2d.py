"""2D damage and mechanics solvers in numpy.  TEST ORACLE ONLY.

Restates the control flow of PhAST's
``PhaseFieldDamageSolver._solve_projected_cg`` (solvers/damage_solver.py:3528-3775),
``ExplicitDynamics`` (solvers/mechanics_solver.py:86-239),
``QuasiStaticSolver.solve`` / ``_cg_solve`` (mechanics_solver.py:1597-1783, 1984-2043)
and ``StaggeredSolver.step_full`` (solvers/staggered_solver.py:1103-1344).
"""
from __future__ import annotations

import math

import numpy as np

from . import q4


def active_mask(d, lb, r, ub=1.0, atol=1e-14, fixed=None):
    """projected_damage_active_mask (damage_solver.py:109-124)."""
    a = ((d <= lb + atol) & (r < 0)) | ((d >= ub - atol) & (r > 0))
    if fixed is not None:
        a = a | fixed
    return a


def projected_cg(Ax, b, M_inv, d0, lb, tol, max_iter, fixed=None, vals=None, check_every=10):
    """_solve_projected_cg (damage_solver.py:3528-3775), Jacobi branch.

    Returns ``(d, last_iter)``.
    """
    d = d0.copy()
    lb = lb.copy()
    if fixed is not None:
        d = np.where(fixed, vals, d)
        lb = np.where(fixed, vals, lb)
    ub = 1.0
    r = b - Ax(d)
    if fixed is not None:
        r[fixed] = 0.0
        M_inv = M_inv.copy()
        M_inv[fixed] = 0.0
    r0sq = float(r @ r)
    ref = max(math.sqrt(float(b @ b)), math.sqrt(r0sq), 1e-30)
    tol_sq = (tol * ref) ** 2
    active = active_mask(d, lb, r, fixed=fixed)
    rf = np.where(active, 0.0, r)
    z = rf * M_inv
    z[active] = 0.0
    p = z.copy()
    rz = float(rf @ z)
    last_iter = max_iter
    for i in range(max_iter):
        it = i + 1
        Ap = Ax(p)
        pAp = float(p @ Ap)
        if pAp <= 0:
            last_iter = it
            break
        a_cg = rz / (pAp + 1e-30)
        a_max = a_cg
        pos = p > 0
        if pos.any():
            a_max = min(a_max, float(((ub - d[pos]) / p[pos]).min()))
        neg = p < 0
        if neg.any():
            a_max = min(a_max, float(((lb[neg] - d[neg]) / p[neg]).min()))
        if a_max < a_cg and a_max >= 0:
            d = d + a_max * p
            d = np.minimum(np.maximum(d, lb), ub)
            r = b - Ax(d)
            if fixed is not None:
                r[fixed] = 0.0
            active = active_mask(d, lb, r, fixed=fixed)
            rf = np.where(active, 0.0, r)
            rfsq = float(rf @ rf)
            if rfsq < tol_sq:
                last_iter = it
                break
            if rfsq > 1e12 * max(r0sq, 1e-30):
                last_iter = it
                break
            z = rf * M_inv
            z[active] = 0.0
            p = z.copy()
            rz = float(rf @ z)
            continue
        d = d + a_cg * p
        r = r - a_cg * Ap
        if it % check_every == 0:
            r = b - Ax(d)
            if fixed is not None:
                r[fixed] = 0.0
            old = active
            active = active_mask(d, lb, r, fixed=fixed)
            changed = bool((active != old).any())
            rf = np.where(active, 0.0, r)
            rfsq = float(rf @ rf)
            if rfsq < tol_sq:
                last_iter = it
                break
            if rfsq > 1e12 * max(r0sq, 1e-30):
                last_iter = it
                break
            if changed:
                z = rf * M_inv
                z[active] = 0.0
                p = z.copy()
                rz = float(rf @ z)
                continue
        else:
            rf = np.where(active, 0.0, r)
        zn = rf * M_inv
        zn[active] = 0.0
        rzn = float(rf @ zn)
        beta = rzn / (rz + 1e-30)
        p = beta * p + zn
        p[active] = 0.0
        rz = rzn
    d = np.minimum(np.maximum(d, lb), ub)
    if fixed is not None:
        d = np.where(fixed, vals, d)
    return d, last_iter


def damage_solve_q4(geo, mat: q4.Mat2D, H_q, d_prev, tol, max_iter, initial=None,
                    fixed=None, vals=None, gc_e=None):
    """PhaseFieldDamageSolver.solve -> _solve_projected_cg for native Q4 AT2."""
    gc_l0 = mat.Gc * mat.l0
    gc_over = mat.Gc / mat.l0
    gc_l0_e = None if gc_e is None else gc_e * mat.l0
    gc_over_e = None if gc_e is None else gc_e / mat.l0
    rd, b, M_inv = q4.damage_prepare(geo, H_q, gc_over, gc_l0, gc_over_e, gc_l0_e)
    d0 = d_prev if initial is None else initial

    def Ax(x):
        return q4.damage_apply(geo, x, rd, gc_l0, gc_l0_e)

    return projected_cg(Ax, b, M_inv, d0, d_prev, tol, max_iter, fixed, vals)


# ----------------------------------------------------------------------------
# mechanics
# ----------------------------------------------------------------------------

def explicit_step(geo, mat, dt, u, v, a, d, f_ext, bc_mask, bc_vals):
    """ExplicitDynamics.predictor/corrector (mechanics_solver.py:153-202), no damping."""
    un = u + dt * v + 0.5 * dt * dt * a
    un[bc_mask] = bc_vals[bc_mask]
    f = q4.internal_force(geo, mat, un, d)
    Minv = 1.0 / (mat.rho * geo.M_scalar + 1e-30)
    an = Minv[:, None] * (f_ext - f)
    vn = v + 0.5 * dt * (a + an)
    an[bc_mask] = 0.0
    vn[bc_mask] = 0.0
    return un, vn, an


def qs_solve(geo, mat, d, f_ext, bc_mask, bc_vals, u_init, tol, cg_tol, cg_max_iter,
             max_iter=50):
    """QuasiStaticSolver.solve with backend='cg', isotropic split, no line search.

    Newton loop mechanics_solver.py:1753-1783; _cg_solve :1984-2043.
    Returns ``(u, converged, n_iter)``.
    """
    u = u_init.copy()
    u[bc_mask] = bc_vals[bc_mask]
    free = (~bc_mask).astype(np.float64)
    for it in range(max_iter):
        res = (f_ext - q4.internal_force(geo, mat, u, d)) * free
        if np.linalg.norm(res) <= tol:
            return u, True, it
        du = np.zeros_like(res)
        r = res.copy()
        p = r.copy()
        rr = float((r * r).sum())
        rr0 = rr
        for i in range(cg_max_iter):
            Ap = q4.internal_force(geo, mat, p, d) * free
            pAp = float((p * Ap).sum())
            if pAp <= 1e-30:
                break
            alpha = rr / (pAp + 1e-30)
            du = du + alpha * p
            r = r - alpha * Ap
            rrn = float((r * r).sum())
            p = (rrn / (rr + 1e-30)) * p + r
            rr = rrn
            if (i + 1) % 50 == 0:
                if rr < cg_tol ** 2 or rr > 1e12 * rr0:
                    break
        u = u + du
        u[bc_mask] = bc_vals[bc_mask]
    return u, False, max_iter


def relative_change(new, old):
    """'relative' stagger criterion with l2 norms (staggered_solver.py:1285-1289)."""
    return float(np.linalg.norm(new - old) / (np.linalg.norm(new) + 1e-30))

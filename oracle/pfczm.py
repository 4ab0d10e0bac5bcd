"""PF-CZM damage law of the periodic voxel cell in numpy.

TEST ORACLE ONLY.  Restates PhAST's ``src/phast/physics/pfczm.py`` (Wu's rational
degradation, ``a1``, softening parameters), the PF-CZM parts of
``solid3d/operator.py`` (energy, gradient, Newton tangent, Newton system:
operator.py:326-606) and the projected Newton damage solve of
``solid3d/staggered.py:843-1096``, on top of the AT2 voxel oracle in ``h8.py``.
"""
from __future__ import annotations

import math

import numpy as np

from . import h8

C_ALPHA = math.pi              # pfczm.py:6
TANGENT_FLOOR = 0.25           # operator.py:125
ARMIJO = 1.0e-4                # staggered.py:118
ENERGY_RTOL = 1.0e-12          # staggered.py:121
MAX_HALVINGS = 30              # staggered.py:124
MAX_DOUBLINGS = 6              # staggered.py:127
INNER_KKT_FRACTION = 0.1       # staggered.py:130
MIN_LINEAR_TOLERANCE = 4.0 * float(np.finfo(np.float64).eps)  # staggered.py:97


def softening_parameters(softening):
    """(a2, a3) of Wu's softening laws (pfczm.py:57-65)."""
    if softening == "linear":
        return -0.5, 0.0
    if softening == "exponential":
        return 2.0 ** (5.0 / 3.0) - 3.0, 0.0
    raise ValueError(softening)


def onset_bound(a2, p=2):
    """Smallest a1 with g''(0) >= 0 (pfczm.py:68-76)."""
    return float(p) + float(a2)


def a1_of(E, Gc, ell, f_t, eta=0.0):
    """a1 = 4 E Gc / (pi ell f_t^2 (1 - eta)) (pfczm.py:16-31)."""
    return 4.0 * E * Gc / (math.pi * ell * f_t ** 2 * max(1.0 - float(eta), 1e-30))


def degradation_derivatives(d, a1, a2, a3, p=2, eta=0.0):
    """g, g', g'' of A/(A+Q) blended to [eta, 1] (pfczm.py:79-125); a1 broadcasts over the
    trailing axis of d."""
    a1 = np.asarray(a1, dtype=np.float64)
    while a1.ndim < np.ndim(d):
        a1 = a1[..., None]
    p = int(p) if float(p).is_integer() else float(p)
    omd = np.maximum(1.0 - d, 0.0)
    A = omd ** p
    Ap = -float(p) * omd ** (p - 1)
    App = np.full_like(d, 2.0) if p == 2 else float(p * (p - 1)) * omd ** (p - 2)
    Q = a1 * d * (1.0 + a2 * d + a2 * a3 * d * d)
    Qp = a1 * (1.0 + 2.0 * a2 * d + 3.0 * a2 * a3 * d * d)
    Qpp = a1 * (2.0 * a2 + 6.0 * a2 * a3 * d)
    S = np.maximum(A + Q, 1e-30)
    N = Ap * Q - A * Qp
    Np = App * Q - A * Qpp
    s = 1.0 - eta
    return (s * (A / S) + eta, s * (N / (S * S)), s * (Np / (S * S) - 2.0 * N * (Ap + Qp) / (S * S * S)))


class PfczmOperator:
    """The PF-CZM operators of one voxel cell (operator.py:326-606).

    ``base`` is an ``h8.VoxelOperator``; ``E_ref`` and ``f_t`` are per-slot tables
    (the isotropic phase modulus and tensile strength).
    """

    def __init__(self, base, E_ref, f_t, softening="linear", p=2):
        self.base = base
        self.a2, self.a3 = softening_parameters(softening)
        self.p = p
        self.bound = onset_bound(self.a2, p)
        E_ref, f_t = np.asarray(E_ref, np.float64), np.asarray(f_t, np.float64)
        self.a1_slot = a1_of(E_ref, base.Gc, base.ell, f_t, base.kappa)
        self.a1 = self.a1_slot[base.slot]
        self.m = base.ref.M.sum(axis=1)
        self.K = (2.0 / C_ALPHA) * base.ell * base.ref.L

    # -- per element --------------------------------------------------------------
    def _dq(self, d):
        return d[self.base.nodes] @ self.base.ref.N.T

    def degradation(self, d):
        """degradation with the PF-CZM law (operator.py:939-946)."""
        b = self.base
        return degradation_derivatives(self._dq(d), self.a1, self.a2, self.a3, self.p, b.kappa)[0]

    def energy(self, d, H):
        """pfczm_damage_energy (operator.py:465-489)."""
        b = self.base
        de = d[b.nodes]
        G = b.Gc[b.slot]
        local = 2.0 * (de @ self.m) - ((de @ b.ref.M) * de).sum(-1)
        grad = ((de @ b.ref.L) * de).sum(-1)
        total = float((G * (local / (C_ALPHA * b.ell) + (b.ell / C_ALPHA) * grad)).sum())
        if H is not None:
            g = degradation_derivatives(de @ b.ref.N.T, self.a1, self.a2, self.a3, self.p, b.kappa)[0]
            total += float(((H * b.ref.w) * g).sum())
        return total

    def gradient(self, d, H):
        """pfczm_damage_gradient, unscaled (operator.py:491-513)."""
        b = self.base
        de = d[b.nodes]
        G = b.Gc[b.slot][:, None]
        y = G * ((2.0 / (C_ALPHA * b.ell)) * (self.m - de @ b.ref.M) + (2.0 * b.ell / C_ALPHA) * (de @ b.ref.L))
        if H is not None:
            gp = degradation_derivatives(de @ b.ref.N.T, self.a1, self.a2, self.a3, self.p, b.kappa)[1]
            y = y + ((H * b.ref.w) * gp) @ b.ref.N
        out = np.zeros(b.n_red)
        np.add.at(out, b.nodes.reshape(-1), y.reshape(-1))
        return out

    def tangent_weights(self, d, H):
        """pfczm_tangent_weights (operator.py:515-539)."""
        b = self.base
        concave = (2.0 / (C_ALPHA * b.ell) * b.Gc[b.slot])[:, None]
        floor = TANGENT_FLOOR * concave
        if H is None:
            return np.repeat(floor, 8, axis=1)
        gpp = degradation_derivatives(self._dq(d), self.a1, self.a2, self.a3, self.p, b.kappa)[2]
        return np.maximum(H * gpp - concave, floor)

    def tangent_action(self, f, W):
        """pfczm_tangent_action, unscaled (operator.py:541-553)."""
        b = self.base
        fe = f[b.nodes]
        y = b.Gc[b.slot][:, None] * (fe @ self.K) + ((W * b.ref.w) * (fe @ b.ref.N.T)) @ b.ref.N
        out = np.zeros(b.n_red)
        np.add.at(out, b.nodes.reshape(-1), y.reshape(-1))
        return out

    def tangent_diagonal(self, W):
        """pfczm_tangent_diagonal, unscaled (operator.py:555-566)."""
        b = self.base
        y = b.Gc[b.slot][:, None] * np.diag(self.K)[None, :] + (W * b.ref.w) @ (b.ref.N ** 2)
        out = np.zeros(b.n_red)
        np.add.at(out, b.nodes.reshape(-1), y.reshape(-1))
        return out

    def newton_system(self, d, H):
        """pfczm_newton_system, scaled (operator.py:568-606): (action, rhs, diag, gradient)."""
        s = self.base.damage_scale
        W = self.tangent_weights(d, H)
        grad = s * self.gradient(d, H)
        action = lambda v: s * self.tangent_action(v, W)  # noqa: E731
        return action, action(d) - grad, s * self.tangent_diagonal(W), grad

    def fracture_energy(self, d):
        """_pfczm_fracture_energy total (operator.py:608-631)."""
        return self.energy(d, None)


def _projected(grad, d, lower):
    pg = np.where(d <= lower, np.minimum(grad, 0.0), grad)
    return np.where(d >= 1.0, np.maximum(pg, 0.0), pg)


def damage_pfczm(op: PfczmOperator, cfg, H, lower, initial, max_newton=100):
    """StaggeredSolver._damage_pfczm (staggered.py:843-1096), absolute-field QP.

    Returns (d, pcg iterations, active-set iterations, Newton iterations, energies)."""
    tol = cfg.damage_kkt_tol
    inner = INNER_KKT_FRACTION * tol
    s = op.base.damage_scale
    d = initial.copy()
    energy = op.energy(d, H)
    if not math.isfinite(energy):
        raise RuntimeError("PF-CZM energy is not finite")
    energies = [energy]
    pcg = sets = 0
    for it in range(max_newton + 1):
        action, rhs, diag, grad = op.newton_system(d, H)
        res = float(np.abs(_projected(grad, d, lower)).max())
        if not math.isfinite(res):
            raise RuntimeError("PF-CZM gradient is not finite")
        if res <= tol:
            return d, pcg, sets, it, energies
        if it == max_newton:
            break
        hold_lower = (d <= lower) & (grad > tol)
        hold_upper = (d >= 1.0) & (grad < -tol)
        upper_k = np.where(hold_lower, lower, 1.0)
        lower_k = np.where(hold_upper, 1.0, lower)
        r0 = float(np.linalg.norm(grad))
        lt = max(min(cfg.damage_linear_tol, 0.1 * inner / max(r0, 1.0)), MIN_LINEAR_TOLERANCE)
        target, its, ai, _ = h8.box_kkt(action, rhs, diag, lower_k, upper_k, d, lt, inner, cfg.damage_maxit,
                                        cfg.damage_max_active_set)
        pcg += its
        sets += ai
        step = target - d
        slope = float((grad * step).sum()) / s
        t = 1.0
        for _ in range(MAX_HALVINGS + 1):
            trial = target if t == 1.0 else np.minimum(np.maximum(d + t * step, lower), 1.0)
            te = op.energy(trial, H)
            if math.isfinite(te) and te <= energy + ARMIJO * t * slope + ENERGY_RTOL * abs(energy):
                break
            t *= 0.5
        else:
            raise RuntimeError("PF-CZM line search failed")
        if t == 1.0:
            tr = float(np.abs(_projected(s * op.gradient(trial, H), trial, lower)).max())
            if not tr <= tol:
                for _ in range(MAX_DOUBLINGS):
                    t *= 2.0
                    further = np.minimum(np.maximum(d + t * step, lower), 1.0)
                    if np.array_equal(further, trial):
                        break
                    fe = op.energy(further, H)
                    if not (math.isfinite(fe) and fe < te):
                        break
                    trial, te = further, fe
        d, energy = trial, te
        energies.append(energy)
    raise RuntimeError("PF-CZM Newton did not converge")


def increment(op: PfczmOperator, cfg, x, d, H_prev, previous, target, max_newton=100):
    """One staggered _attempt with the PF-CZM law (staggered.py:1259-1517): returns
    (x, d, H, stagger_iters, pcg_mech, pcg_pf, active_sets, newton, macro_stress)."""
    counts = [0, 0, 0]

    def damage(H, lower, initial):
        dn, its, ai, nw, _ = damage_pfczm(op, cfg, H, lower, initial, max_newton)
        counts[0] += ai
        counts[1] += nw
        return dn, its

    out = h8.increment(op.base, cfg, x, d, H_prev, previous, target, degradation=op.degradation, damage=damage)
    x, d, H, k, pm, pp, sig = out
    return x, d, H, k, pm, pp, counts[0], counts[1], sig

"""Crack closure of the voxel cell (``crack_closure='axes'``, isotropic group) in numpy.

TEST ORACLE ONLY.  Restates PhAST's ``src/phast/solid3d/splits.py`` closure rows and
moduli (closure_isotropic_rows / closure_isotropic_moduli, splits.py:486-503), the
closure parts of ``solid3d/operator.py`` (pattern, pattern change, the stress pass with
the (1 - g) sigma_c add-back, the diagonal, the kinematic guard: operator.py:770-877,
1039-1302, 1713-1770) and the closure mechanics of ``solid3d/staggered.py``
(_closure_mechanics with the energy line search, staggered.py:550-751) on top of the
AT2 voxel oracle in ``h8.py``.
"""
from __future__ import annotations

import math

import numpy as np

from . import h8

MAX_SOLVES = 50                 # INTERFACE_MAX_SOLVES, staggered.py:99
PATTERN_TOLERANCE = 1.0e-8      # CLOSURE_PATTERN_TOLERANCE, staggered.py:105
LS_ARMIJO = 1.0e-4              # LINE_SEARCH_ARMIJO, staggered.py:109
LS_ENERGY_RTOL = 1.0e-12        # LINE_SEARCH_ENERGY_RTOL, staggered.py:112
LS_MAX_HALVINGS = 30            # LINE_SEARCH_MAX_HALVINGS, staggered.py:115

# rows v_k: the trace and e_x, e_y, e_z (splits.py:489-495)
ROWS = np.zeros((4, 6))
ROWS[0, :3] = 1.0
ROWS[1, 0] = ROWS[2, 1] = ROWS[3, 2] = 1.0


class ClosureOperator:
    """The isotropic closure group of one cell: moduli (lam, 2 mu, 2 mu, 2 mu) per element
    where the element has a damage driver, zero elsewhere."""

    def __init__(self, base: h8.VoxelOperator):
        self.base = base
        on = base.driver[base.slot] != h8.DRIVER_NONE
        lam = np.where(on, base.lam[base.slot], 0.0)
        mu = np.where(on, base.mu[base.slot], 0.0)
        self.mask = on
        self.k = np.stack([lam, 2.0 * mu, 2.0 * mu, 2.0 * mu], -1)   # (E, 4)

    def values(self, x):
        """v_k . eps (E, 8, 4) (_iso_closure_values, operator.py:789-794)."""
        return self.base.qp_strain(x) @ ROWS.T

    def pattern(self, x):
        """closure_pattern (operator.py:821-834)."""
        return (self.values(x) < 0.0) & self.mask[:, None, None]

    def stress_pass(self, x, g, pattern=None):
        """_stress_pass_closure (operator.py:1039-1108), isotropic group: (r_u, r_E, energy)."""
        b = self.base
        eps = b.qp_strain(x)
        sig = np.einsum("eij,eqj->eqi", b.C[b.slot], eps)
        if g is not None:
            vals = eps @ ROWS.T
            active = vals < 0.0 if pattern is None else pattern
            coef = np.where(active, vals, 0.0) * self.k[:, None, :]
            sig = g[..., None] * sig + (1.0 - g)[..., None] * (coef @ ROWS)
        wsig = sig * b.ref.w[None, :, None]
        rE = wsig.sum((0, 1))
        energy = 0.5 * float((wsig * eps).sum())
        local = wsig.reshape(-1, 48) @ b.Bflat.T
        ru = np.zeros(3 * b.n_red)
        np.add.at(ru, b.dofs.reshape(-1), local.reshape(-1))
        return ru, rE, energy

    def mech_action(self, x, g, pattern=None):
        ru, rE, _ = self.stress_pass(x, g, pattern)
        return np.concatenate([ru, rE])

    def elastic_energy(self, x, g):
        return self.stress_pass(x, g)[2]

    def macro_stress(self, x, g):
        return self.stress_pass(x, g)[1] / self.base.volume

    def mech_diagonal(self, g, pattern=None):
        """mech_diagonal with the closure terms (operator.py:1196-1302); all bits without a pattern."""
        b = self.base
        diag = b.mech_diagonal(g)
        coef = (1.0 - g)[..., None] * self.k[:, None, :] * b.ref.w[None, :, None]
        if pattern is not None:
            coef = coef * pattern
        BtR = np.einsum("qia,ki->qka", b.ref.B, ROWS)                  # (8, 4, 24)
        local = np.einsum("eqk,qka->ea", coef, BtR ** 2)
        du = np.zeros(3 * b.n_red)
        np.add.at(du, b.dofs.reshape(-1), local.reshape(-1))
        dE = np.einsum("ek,ki->i", coef.sum(1), ROWS ** 2)
        return diag + np.concatenate([du, dE])

    def pattern_change(self, x, old, g, tolerance=PATTERN_TOLERANCE):
        """closure_pattern_change (operator.py:836-873): (new pattern, changed)."""
        vals = self.values(x)
        new = (vals < 0.0) & self.mask[:, None, None]
        strength = self.k[:, None, :] * np.abs(vals)
        flipped = new != old
        changed = False
        if flipped.any():
            jump = (1.0 - g)[..., None] * strength
            changed = float(jump[flipped].max()) > tolerance * float(strength.max())
        return new, changed

    def kinematic_guard(self, x):
        """kinematic_guard min values (operator.py:1713-1770)."""
        b = self.base
        strain = b.qp_strain(x).mean(1)
        T = h8.voigt_to_tensor(strain)
        principal = np.linalg.eigvalsh(T)[:, 0]
        u = x[: 3 * b.n_red].reshape(-1, 3)
        E = h8.voigt_to_tensor(x[3 * b.n_red:])
        grad = np.einsum("eai,qaj->eqij", u[b.nodes], b.ref.grad)
        det = np.linalg.det(np.eye(3) + E + grad)
        return float(strain[:, :3].min()), float(principal.min()), float(det.min())


def energy_line_search(cl: ClosureOperator, x, y, g, free):
    """_energy_line_search (staggered.py:589-626): (point, alpha)."""
    p = y - x
    e0 = cl.elastic_energy(x, g)
    force = cl.mech_action(x, g)
    slope = min(float(force[free] @ p[free]), 0.0)
    allowance = LS_ENERGY_RTOL * abs(e0)
    alpha = 1.0
    for _ in range(LS_MAX_HALVINGS + 1):
        trial = y if alpha == 1.0 else x + alpha * p
        e = cl.elastic_energy(trial, g)
        if not math.isfinite(e):
            raise RuntimeError("mechanics energy is not finite in the line search")
        if e <= e0 + LS_ARMIJO * alpha * slope + allowance:
            return trial, alpha
        alpha *= 0.5
    raise RuntimeError("closure line search found no decrease")


def closure_mechanics(cl: ClosureOperator, cfg, g, values, x0):
    """_closure_mechanics (staggered.py:698-751): (x, PCG iterations, solves)."""
    b = cl.base
    mask = b.fixed_mask()
    free = ~mask
    pattern = cl.pattern(x0)
    its = 0
    for solve in range(1, MAX_SOLVES + 1):
        y, k, conv, _, _ = h8.solve_constrained(lambda v: cl.mech_action(v, g, pattern), cl.mech_diagonal(g, pattern),
                                                mask, values, x0=x0, rtol=cfg.pcg_rtol_mech,
                                                maxiter=cfg.pcg_maxit_mech, check_every=cfg.check_every)
        if not conv:
            raise RuntimeError("mechanics PCG did not converge")
        its += k
        x, alpha = energy_line_search(cl, x0, y, g, free)
        pattern, changed = cl.pattern_change(x, pattern, g)
        if not changed and alpha == 1.0:
            return x, its, solve
        x0 = x
    raise RuntimeError("closure pattern did not settle")


def increment(cl: ClosureOperator, cfg, x, d, H_prev, previous, target):
    """One staggered _attempt with the crack closure (staggered.py:1259-1517): returns
    (x, d, H, stagger_iters, pcg_mech, pcg_pf, closure_solves, macro_stress, guard)."""
    solves = [0]

    def mechanics(g, values, x0):
        xs, its, n = closure_mechanics(cl, cfg, g, values, x0)
        solves[0] += n
        return xs, its

    x, d, H, k, pm, pp, _ = h8.increment(cl.base, cfg, x, d, H_prev, previous, target, mechanics=mechanics)
    g = cl.base.degradation(d)
    return x, d, H, k, pm, pp, solves[0], cl.macro_stress(x, g), cl.kinematic_guard(x)

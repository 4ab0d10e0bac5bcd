"""Periodic voxel H8 operators, PCG, box-KKT and the staggered increment in numpy.

TEST ORACLE ONLY.  Restates PhAST's ``src/phast/solid3d/periodic.py``,
``solid3d/operator.py`` (AT2 parts), ``solid3d/splits.py``, ``solid3d/linalg.py``,
``solvers/box_kkt_h8.py`` and ``solid3d/staggered.py`` (plain alternate
minimisation with ``history='max'`` and ``irreversibility='box_kkt'``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

_A = 1.0 / math.sqrt(3.0)
# Local corner signs (core/hex8.py:16-36).
SIGNS = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                  [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.float64)
# Gauss points, xi fastest (core/hex8.py:157-178).
QPTS = np.array([[sx * _A, sy * _A, sz * _A] for sz in (-1, 1) for sy in (-1, 1) for sx in (-1, 1)])


@dataclass
class RefVoxel:
    """reference_voxel (solid3d/periodic.py:193-221)."""
    h: tuple
    N: np.ndarray      # (8 q, 8 a)
    grad: np.ndarray   # (8 q, 8 a, 3)
    w: np.ndarray      # (8,)
    B: np.ndarray      # (8, 6, 24)
    M: np.ndarray
    L: np.ndarray
    volume: float


def reference_voxel(h):
    hx, hy, hz = (float(v) for v in h)
    xi, eta, ze = QPTS[:, 0:1], QPTS[:, 1:2], QPTS[:, 2:3]
    sx, sy, sz = SIGNS[None, :, 0], SIGNS[None, :, 1], SIGNS[None, :, 2]
    N = 0.125 * (1 + sx * xi) * (1 + sy * eta) * (1 + sz * ze)
    gx = 0.125 * sx * (1 + sy * eta) * (1 + sz * ze) * (2.0 / hx)
    gy = 0.125 * (1 + sx * xi) * sy * (1 + sz * ze) * (2.0 / hy)
    gz = 0.125 * (1 + sx * xi) * (1 + sy * eta) * sz * (2.0 / hz)
    grad = np.stack([gx, gy, gz], -1)
    w = np.full(8, hx * hy * hz / 8.0)
    B = np.zeros((8, 6, 24))
    for a in range(8):
        B[:, 0, 3 * a] = gx[:, a]
        B[:, 1, 3 * a + 1] = gy[:, a]
        B[:, 2, 3 * a + 2] = gz[:, a]
        B[:, 3, 3 * a + 1] = gz[:, a]
        B[:, 3, 3 * a + 2] = gy[:, a]
        B[:, 4, 3 * a] = gz[:, a]
        B[:, 4, 3 * a + 2] = gx[:, a]
        B[:, 5, 3 * a] = gy[:, a]
        B[:, 5, 3 * a + 1] = gx[:, a]
    M = np.einsum("q,qa,qb->ab", w, N, N)
    L = np.einsum("q,qaj,qbj->ab", w, grad, grad)
    return RefVoxel((hx, hy, hz), N, grad, w, B, 0.5 * (M + M.T), 0.5 * (L + L.T), hx * hy * hz)


def periodic_map(shape, periodic=(True, True, True)):
    """PeriodicVoxelMap.build (solid3d/periodic.py:61-113): element_nodes (E, 8), n_red."""
    nx, ny, nz = shape
    px, py, pz = periodic
    rx, ry, rz = (nx if px else nx + 1), (ny if py else ny + 1), (nz if pz else nz + 1)
    ke, je, ie = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    off = ((SIGNS + 1) / 2).astype(np.int64)
    i = ie.reshape(-1, 1) + off[:, 0]
    j = je.reshape(-1, 1) + off[:, 1]
    k = ke.reshape(-1, 1) + off[:, 2]
    if px:
        i = i % nx
    if py:
        j = j % ny
    if pz:
        k = k % nz
    return i + rx * (j + ry * k), rx * ry * rz, (rx, ry, rz)


def isotropic_C(E, nu):
    """Isotropic 6x6 engineering-Voigt stiffness (core/hex8.py:isotropic_stiffness_3d)."""
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    C = np.zeros((6, 6))
    C[:3, :3] = lam
    C[[0, 1, 2], [0, 1, 2]] = lam + 2 * mu
    C[[3, 4, 5], [3, 4, 5]] = mu
    return C, lam, mu


def eigvalsh3_closed(T):
    """symmetric_eigvalsh_3x3 (solid3d/splits.py:93-125), ascending."""
    a11, a22, a33 = T[..., 0, 0], T[..., 1, 1], T[..., 2, 2]
    a12, a13, a23 = T[..., 0, 1], T[..., 0, 2], T[..., 1, 2]
    q = (a11 + a22 + a33) / 3.0
    b11, b22, b33 = a11 - q, a22 - q, a33 - q
    p1 = a12 ** 2 + a13 ** 2 + a23 ** 2
    p = np.sqrt((b11 ** 2 + b22 ** 2 + b33 ** 2 + 2 * p1) / 6.0)
    det = b11 * (b22 * b33 - a23 ** 2) - a12 * (a12 * b33 - a23 * a13) + a13 * (a12 * a23 - b22 * a13)
    iso = p <= np.finfo(np.float64).tiny
    ps = np.where(iso, 1.0, p)
    r = np.clip(det / (2 * ps ** 3), -1, 1)
    phi = np.arccos(r) / 3
    big = q + 2 * p * np.cos(phi)
    small = q + 2 * p * np.cos(phi + 2 * math.pi / 3)
    mid = 3 * q - big - small
    out = np.stack([small, mid, big], -1)
    return np.where(iso[..., None], q[..., None], out)


def voigt_to_tensor(eps):
    """engineering_strain_to_tensor: halve the shears."""
    T = np.empty(eps.shape[:-1] + (3, 3))
    T[..., 0, 0], T[..., 1, 1], T[..., 2, 2] = eps[..., 0], eps[..., 1], eps[..., 2]
    T[..., 1, 2] = T[..., 2, 1] = 0.5 * eps[..., 3]
    T[..., 0, 2] = T[..., 2, 0] = 0.5 * eps[..., 4]
    T[..., 0, 1] = T[..., 1, 0] = 0.5 * eps[..., 5]
    return T


DRIVER_NONE, DRIVER_FULL, DRIVER_SPECTRAL = 0, 1, 2


@dataclass
class VoxelOperator:
    """PeriodicVoxelPhaseFieldOperator AT2 parts (solid3d/operator.py:133-1544).

    ``slot`` (E,) indexes per-phase tables ``C`` (S,6,6), ``lam``, ``mu``,
    ``Gc`` (S,) and ``driver`` (S,).
    """
    shape: tuple
    h: tuple
    slot: np.ndarray
    C: np.ndarray
    lam: np.ndarray
    mu: np.ndarray
    Gc: np.ndarray
    driver: np.ndarray
    ell: float
    kappa: float
    pinned_node: int
    controlled: int
    fixed_zero: tuple
    periodic: tuple = (True, True, True)
    eig: str = "eigvalsh"
    nodes: np.ndarray = field(init=False)
    n_red: int = field(init=False)

    def __post_init__(self):
        self.nodes, self.n_red, self.reduced_shape = periodic_map(self.shape, self.periodic)
        self.ref = reference_voxel(self.h)
        self.n_mech = 3 * self.n_red + 6
        self.n_elements = self.nodes.shape[0]
        nx, ny, nz = self.shape
        self.volume = nx * ny * nz * self.ref.volume
        Ge = self.Gc[self.slot]
        self.damage_scale = self.ell / (float(Ge.min()) * self.ref.volume)
        self.dofs = (3 * self.nodes[:, :, None] + np.arange(3)).reshape(-1, 24)
        self.Bflat = self.ref.B.transpose(2, 0, 1).reshape(24, 48)
        self.Kd = self.ref.M / self.ell + self.ell * self.ref.L

    # -- mechanics ----------------------------------------------------------
    def degradation(self, d):
        """degradation (operator.py:939-946; splits.py:56-59)."""
        dq = d[self.nodes] @ self.ref.N.T
        return (1 - self.kappa) * (1 - dq) ** 2 + self.kappa

    def qp_strain(self, x):
        u = x[: 3 * self.n_red]
        E = x[3 * self.n_red:]
        return (u[self.dofs] @ self.Bflat).reshape(-1, 8, 6) + E

    def stress_pass(self, x, g):
        """_stress_pass (operator.py:1108-1169) without interface/closure terms."""
        eps = self.qp_strain(x)
        Ce = self.C[self.slot]
        sig = np.einsum("eij,eqj->eqi", Ce, eps)
        if g is not None:
            sig = g[..., None] * sig
        wsig = sig * self.ref.w[None, :, None]
        rE = wsig.sum((0, 1))
        energy = 0.5 * float((wsig * eps).sum())
        local = wsig.reshape(-1, 48) @ self.Bflat.T
        ru = np.zeros(3 * self.n_red)
        np.add.at(ru, self.dofs.reshape(-1), local.reshape(-1))
        return ru, rE, energy

    def mech_action(self, x, g=None):
        ru, rE, _ = self.stress_pass(x, g)
        return np.concatenate([ru, rE])

    def mech_diagonal(self, g=None):
        """mech_diagonal (operator.py:1196-1254)."""
        B = self.ref.B
        Ce = self.C[self.slot]
        gw = np.broadcast_to(self.ref.w, (self.n_elements, 8)) if g is None else g * self.ref.w
        per_qp = np.einsum("qia,eij,qja->eqa", B, Ce, B)
        local = (gw[..., None] * per_qp).sum(1)
        du = np.zeros(3 * self.n_red)
        np.add.at(du, self.dofs.reshape(-1), local.reshape(-1))
        dE = (gw.sum(1)[:, None] * np.diagonal(Ce, axis1=1, axis2=2)).sum(0)
        return np.concatenate([du, dE])

    def macro_stress(self, x, g=None):
        return self.stress_pass(x, g)[1] / self.volume

    def elastic_energy(self, x, g=None):
        return self.stress_pass(x, g)[2]

    def fixed_mask(self):
        """mech_fixed_mask (operator.py:~905-915)."""
        m = np.zeros(self.n_mech, dtype=bool)
        m[3 * self.pinned_node: 3 * self.pinned_node + 3] = True
        m[3 * self.n_red + self.controlled] = True
        for c in self.fixed_zero:
            m[3 * self.n_red + c] = True
        return m

    def fixed_values(self, e_c):
        v = np.zeros(self.n_mech)
        v[3 * self.n_red + self.controlled] = e_c
        return v

    def driving_force(self, x):
        """driving_force (operator.py:1415-1444): spectral or full driver per slot."""
        eps = self.qp_strain(x)
        drv = self.driver[self.slot]
        Y = np.zeros((self.n_elements, 8))
        full = drv == DRIVER_FULL
        if full.any():
            Ce = self.C[self.slot[full]]
            Y[full] = 0.5 * np.einsum("eqi,eij,eqj->eq", eps[full], Ce, eps[full])
        spec = drv == DRIVER_SPECTRAL
        if spec.any():
            e = eps[spec]
            T = voigt_to_tensor(e)
            pr = np.linalg.eigvalsh(T) if self.eig == "eigvalsh" else eigvalsh3_closed(T)
            trp = np.maximum(e[..., :3].sum(-1), 0)
            lam = self.lam[self.slot[spec]][:, None]
            mu = self.mu[self.slot[spec]][:, None]
            Y[spec] = 0.5 * lam * trp ** 2 + mu * (np.maximum(pr, 0) ** 2).sum(-1)
        return Y

    # -- damage ---------------------------------------------------------------
    def damage_action(self, d, H=None):
        """damage_action (operator.py:1450-1466), unscaled."""
        de = d[self.nodes]
        y = self.Gc[self.slot][:, None] * (de @ self.Kd)
        if H is not None:
            dq = de @ self.ref.N.T
            y = y + 2 * (1 - self.kappa) * ((H * self.ref.w) * dq) @ self.ref.N
        out = np.zeros(self.n_red)
        np.add.at(out, self.nodes.reshape(-1), y.reshape(-1))
        return out

    def damage_rhs(self, H):
        y = 2 * (1 - self.kappa) * (H * self.ref.w) @ self.ref.N
        out = np.zeros(self.n_red)
        np.add.at(out, self.nodes.reshape(-1), y.reshape(-1))
        return out

    def damage_diagonal(self, H=None):
        y = self.Gc[self.slot][:, None] * np.diag(self.Kd)[None, :]
        if H is not None:
            y = y + 2 * (1 - self.kappa) * (H * self.ref.w) @ (self.ref.N ** 2)
        out = np.zeros(self.n_red)
        np.add.at(out, self.nodes.reshape(-1), y.reshape(-1))
        return out

    def fracture_energy(self, d):
        de = d[self.nodes]
        G = self.Gc[self.slot]
        loc = G / (2 * self.ell) * ((de @ self.ref.M) * de).sum(-1)
        grd = 0.5 * G * self.ell * ((de @ self.ref.L) * de).sum(-1)
        return float(loc.sum() + grd.sum())


# ----------------------------------------------------------------------------
# linear algebra (solid3d/linalg.py, solvers/box_kkt_h8.py)
# ----------------------------------------------------------------------------

class Breakdown(RuntimeError):
    pass


def pcg(action, rhs, diag, x0=None, rtol=1e-8, atol=0.0, maxiter=5000, check_every=10):
    """linalg.pcg (solid3d/linalg.py:99-220).  Returns (x, iterations, converged, rnorm, bnorm)."""
    bn = float(np.linalg.norm(rhs))
    if bn == 0.0:
        return np.zeros_like(rhs), 0, True, 0.0, 0.0
    thr = max(rtol * bn, atol)
    if x0 is None:
        x = np.zeros_like(rhs)
        r = rhs.copy()
        rn = bn
    else:
        x = x0.copy()
        r = rhs - action(x)
        rn = float(np.linalg.norm(r))
    if rn <= thr:
        return x, 0, True, rn, bn
    inv = 1.0 / diag
    z = r * inv
    p = z.copy()
    rz = float(r @ z)
    active = True
    done = 0
    rr = float(r @ r)
    for it in range(1, maxiter + 1):
        Ap = action(p)
        pAp = float(p @ Ap)
        if active and not pAp > 0:
            raise Breakdown("non-positive curvature")
        alpha = rz / pAp if active else 0.0
        x = x + alpha * p
        r = r - alpha * Ap
        done += int(active)
        z = r * inv
        rzn = float(r @ z)
        rr = float(r @ r)
        active = active and rr > thr * thr
        beta = rzn / rz if (active and rz > 0) else 0.0
        p = z + beta * p
        rz = rzn
        if it % check_every == 0 or it == maxiter:
            if not active:
                return x, done, True, math.sqrt(rr), bn
    return x, maxiter, False, math.sqrt(rr), bn


def solve_constrained(action, diag, fixed, values, rhs=None, x0=None, rtol=1e-8, maxiter=5000, check_every=10):
    """solve_constrained (solid3d/linalg.py:223-287)."""
    free = ~fixed
    xc = np.where(fixed, values, 0.0)
    img = action(xc)
    b = -img if rhs is None else rhs - img
    bf = np.where(free, b, 0.0)
    dg = np.where(free, diag, 1.0)
    x0f = None if x0 is None else np.where(free, x0, 0.0)
    y, it, conv, rn, bn = pcg(lambda v: np.where(free, action(v), 0.0), bf, dg, x0f, rtol, 0.0, maxiter, check_every)
    return np.where(free, y, xc), it, conv, rn, bn


def dirichlet_pcg(action, rhs, diag, fixed, values, initial, tol, maxit):
    """solve_h8_scalar_dirichlet_pcg + _pcg (box_kkt_h8.py:256-432)."""
    known = np.where(fixed, values, 0.0)
    free = ~fixed
    if not free.any():
        return known, 0, True
    rr = (rhs - action(known))[free]
    dg = diag[free]

    def red(v):
        full = np.zeros_like(rhs)
        full[free] = v
        return action(full)[free]

    x = np.zeros_like(rr) if initial is None else initial[free].copy()
    res = rr - red(x)
    n0 = float(np.linalg.norm(res))
    ref = max(n0, 1.0)
    conv, its = False, maxit
    if n0 <= tol * ref:
        conv, its = True, 0
    else:
        pre = res / dg
        dirn = pre.copy()
        rz = float(res @ pre)
        for it in range(1, maxit + 1):
            img = red(dirn)
            den = float(dirn @ img)
            if not den > 0:
                raise Breakdown("PCG operator is not positive definite on the free space")
            a = rz / den
            x = x + a * dirn
            res = res - a * img
            if float(np.linalg.norm(res)) <= tol * ref:
                conv, its = True, it
                break
            pre = res / dg
            nd = float(res @ pre)
            dirn = pre + (nd / rz) * dirn
            rz = nd
    sol = known.copy()
    sol[free] = x
    return sol, its, conv


def box_kkt(action, rhs, diag, lower, upper, initial, lin_tol, kkt_tol, max_lin, max_active):
    """solve_h8_scalar_box_kkt (box_kkt_h8.py:603-778).  Returns (d, pcg_iters, active_iters, kkt_ok)."""
    lower = np.broadcast_to(lower, rhs.shape).astype(np.float64)
    upper = np.broadcast_to(upper, rhs.shape).astype(np.float64)
    peq = lower == upper
    la = np.zeros_like(peq)
    ua = np.zeros_like(peq)
    cinit = initial
    total = 0
    cand = None
    for ai in range(1, max_active + 1):
        fixed = la | ua | peq
        vals = lower.copy()
        vals[ua] = upper[ua]
        cand, its, conv = dirichlet_pcg(action, rhs, diag, fixed, vals, cinit, lin_tol, max_lin)
        total += its
        grad = action(cand) - rhs
        free = ~fixed
        add_l = free & (cand < lower)
        add_u = free & (cand > upper)
        rel_l = la & (grad < -kkt_tol)
        rel_u = ua & (grad > kkt_tol)
        if not conv:
            raise RuntimeError("box-KKT PCG did not converge")
        if not (add_l | add_u | rel_l | rel_u).any():
            return cand, total, ai, kkt_ok(grad, cand, lower, upper, la, ua, peq, kkt_tol)
        if ai == max_active:
            break
        la = (la | add_l) & ~rel_l
        ua = (ua | add_u) & ~rel_u
        cinit = cand
    raise RuntimeError("box-KKT active set did not stabilise")


def kkt_ok(grad, sol, lo, up, la, ua, peq, tol):
    """_kkt_diagnostics satisfies_kkt (box_kkt_h8.py:459-558)."""
    fixed = la | ua | peq
    free = ~fixed
    lr = grad[la]
    ur = -grad[ua]
    pg = np.zeros_like(grad)
    pg[free] = grad[free]
    pg[la] = np.minimum(lr, 0)
    pg[ua] = np.maximum(grad[ua], 0)
    lm = np.zeros_like(grad)
    um = np.zeros_like(grad)
    lm[la] = np.maximum(lr, 0)
    um[ua] = np.maximum(ur, 0)
    comp = np.concatenate([lm * (sol - lo), um * (up - sol)])
    mx = lambda a: float(np.abs(a).max()) if a.size else 0.0
    return bool(not (sol < lo).any() and not (sol > up).any() and not (lr < -tol).any()
                and not (ur < -tol).any() and mx(grad[free]) <= tol and mx(pg) <= tol and mx(comp) <= tol)


# ----------------------------------------------------------------------------
# staggered increment (solid3d/staggered.py:1259-1517), plain AM, box_kkt
# ----------------------------------------------------------------------------

@dataclass
class Cfg3D:
    stagger_tol: float = 1e-4
    max_stagger: int = 2000
    min_stagger: int = 2
    pcg_rtol_mech: float = 1e-8
    pcg_maxit_mech: int = 20000
    check_every: int = 10
    damage_linear_tol: float = 1e-10
    damage_kkt_tol: float = 1e-8
    damage_maxit: int = 4000
    damage_max_active_set: int = 64


def _damage_at2(op, cfg, H, lower, initial):
    """The box-KKT AT2 damage solve of one staggered iteration (staggered.py:753-800)."""
    s = op.damage_scale
    rhs = s * op.damage_rhs(H)
    dg = s * op.damage_diagonal(H)
    act = lambda v: s * op.damage_action(v, H)  # noqa: E731
    r0 = float(np.linalg.norm(rhs - act(initial)))
    tol = min(cfg.damage_linear_tol, 0.1 * cfg.damage_kkt_tol / max(r0, 1.0))
    tol = max(tol, 4.0 * float(np.finfo(np.float64).eps))
    d_new, its, _, _ = box_kkt(act, rhs, dg, lower, 1.0, initial, tol, cfg.damage_kkt_tol, cfg.damage_maxit,
                               cfg.damage_max_active_set)
    return d_new, its


def increment(op: VoxelOperator, cfg: Cfg3D, x, d, H_prev, previous, target, degradation=None, damage=None,
              mechanics=None):
    """One _attempt: returns (x, d, H, stagger_iters, pcg_mech, pcg_pf, macro_stress).

    ``degradation(d)`` and ``damage(H, lower, initial) -> (d, pcg iterations)`` replace the
    AT2 law when given (the PF-CZM law of ``pfczm.py``); ``mechanics(g, values, x0) ->
    (x, pcg iterations)`` replaces the linear mechanics solve (the closure of ``closure.py``)."""
    degradation = op.degradation if degradation is None else degradation
    mask = op.fixed_mask()

    def _linear(g, values, x0):
        xs, its, conv, _, _ = solve_constrained(lambda v: op.mech_action(v, g), op.mech_diagonal(g), mask, values,
                                                x0=x0, rtol=cfg.pcg_rtol_mech, maxiter=cfg.pcg_maxit_mech,
                                                check_every=cfg.check_every)
        if not conv:
            raise RuntimeError("mechanics PCG did not converge")
        return xs, its

    mechanics = _linear if mechanics is None else mechanics
    nu = 3 * op.n_red
    if previous != 0.0:
        x_old = x * (target / previous)
    else:
        x_old = np.zeros_like(x)
    x_old[nu + op.controlled] = target
    d_old = d.copy()
    lower = d
    values = op.fixed_values(target)
    mask = op.fixed_mask()
    step = abs(target - previous)
    u_floor = min(op.h) * math.sqrt(nu)
    pm = pp = 0
    H = H_prev
    for k in range(1, cfg.max_stagger + 1):
        g = degradation(d_old)
        x_new, its = mechanics(g, values, x_old)
        pm += its
        Y = op.driving_force(x_new)
        H = np.maximum(H_prev, Y)
        if damage is None:
            d_new, its = _damage_at2(op, cfg, H, lower, d_old)
        else:
            d_new, its = damage(H, lower, d_old)
        pp += its
        du = float(np.linalg.norm(x_new[:nu] - x_old[:nu]))
        un = float(np.linalg.norm(x_new[:nu]))
        dE = float(np.abs(x_new[nu:] - x_old[nu:]).max())
        Einf = float(np.abs(x_new[nu:]).max())
        dd = float(np.abs(d_new - d_old).max())
        sE = max(Einf, step)
        uref = max(un, sE * u_floor)
        change = max(du / uref if uref > 0 else 0.0, dE / sE if sE > 0 else 0.0, dd)
        x_old, d_old = x_new, d_new
        if change <= cfg.stagger_tol and k >= cfg.min_stagger:
            break
    else:
        raise RuntimeError("stagger did not converge")
    g = degradation(d_old)
    x_fin, its = mechanics(g, values, x_old)
    pm += its
    return x_fin, d_old, H, k, pm, pp, op.macro_stress(x_fin, g)

"""Q4 (bilinear quadrilateral, 2x2 Gauss) operators in numpy.  TEST ORACLE ONLY.

Restates ``src/phast/core/fem_operators.py`` (Q4 branches) and
``src/phast/core/quad_elements.py`` / ``src/phast/core/mesh.py`` of PhAST.
Arrays follow the reference layouts: ``u (N, 2)``, ``d (N,)``, Gauss-point
fields ``(E, 4)``, element connectivity ``(E, 4)`` counter-clockwise.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

_A = 1.0 / math.sqrt(3.0)
# Gauss points, xi fastest (quad_elements.py:quad_gauss_points, order 2).
QPTS = np.array([[-_A, -_A], [_A, -_A], [-_A, _A], [_A, _A]])
# Corner signs in CCW order (quad_elements.py:q4_shape_functions).
CORNERS = np.array([[-1.0, -1.0], [1.0, -1.0], [1.0, 1.0], [-1.0, 1.0]])


def shape_N():
    """N_q (4 q, 4 a) -- quad_elements.py:q4_shape_functions."""
    xi, eta = QPTS[:, 0:1], QPTS[:, 1:2]
    return 0.25 * (1 + CORNERS[None, :, 0] * xi) * (1 + CORNERS[None, :, 1] * eta)


def shape_dN():
    """dN/d(xi, eta) (4 q, 4 a, 2)."""
    xi, eta = QPTS[:, 0:1], QPTS[:, 1:2]
    sx, sy = CORNERS[None, :, 0], CORNERS[None, :, 1]
    dxi = 0.25 * sx * (1 + sy * eta)
    deta = 0.25 * (1 + sx * xi) * sy
    return np.stack([dxi, deta], axis=-1)


@dataclass
class Q4Geometry:
    """Per-element Gauss geometry (mesh.py:_precompute_q4, quad_elements.py:315-349)."""
    nodes: np.ndarray
    elements: np.ndarray
    N: np.ndarray          # (4, 4)
    grad: np.ndarray       # (E, 4 q, 4 a, 2)
    wdet: np.ndarray       # (E, 4)
    M_scalar: np.ndarray   # (N,) lumped mass  (mesh.py:_precompute_q4)
    h_min: float

    @property
    def n_nodes(self):
        return self.nodes.shape[0]

    @property
    def n_elems(self):
        return self.elements.shape[0]


def geometry(nodes, elements) -> Q4Geometry:
    nodes = np.asarray(nodes, dtype=np.float64)
    elements = np.asarray(elements, dtype=np.int64)
    coords = nodes[elements]                       # (E, 4, 2)
    N = shape_N()
    dN = shape_dN()
    J = np.einsum("qai,eaj->eqij", dN, coords)      # (E, 4, 2, 2)
    det = np.linalg.det(J)
    invJ = np.linalg.inv(J)
    grad = np.einsum("qai,eqji->eqaj", dN, invJ)
    wdet = det * 1.0
    Ms = np.zeros(nodes.shape[0])
    np.add.at(Ms, elements.reshape(-1), np.einsum("qa,eq->ea", N, wdet).reshape(-1))
    edges = np.stack([np.linalg.norm(coords[:, (k + 1) % 4] - coords[:, k], axis=1) for k in range(4)], 1)
    return Q4Geometry(nodes, elements, N, grad, wdet, Ms, float(edges.min()))


def structured_mesh(width, height, nx, ny):
    """structured_q4_mesh (quad_elements.py:458-487): nodes row-major in y, CCW quads."""
    xs = np.linspace(0.0, width, nx + 1)
    ys = np.linspace(0.0, height, ny + 1)
    yy, xx = np.meshgrid(ys, xs, indexing="ij")
    nodes = np.stack([xx.reshape(-1), yy.reshape(-1)], 1)
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    n0 = (j * (nx + 1) + i).reshape(-1)
    quads = np.stack([n0, n0 + 1, n0 + nx + 2, n0 + nx + 1], 1)
    return nodes, quads


# ----------------------------------------------------------------------------
# material
# ----------------------------------------------------------------------------

@dataclass
class Mat2D:
    """The Material fields the hot path reads (physics/material.py:379-529)."""
    E: float
    nu: float
    Gc: float
    l0: float
    eta: float = 1e-8           # eta_residual
    rho: float = 1.0
    plane_stress: bool = False
    split: str = "isotropic"    # energy_split (psi+ and history)
    stress_split: str | None = None  # effective_stress_split(); None -> split
    spectral_eps: float = 1e-12

    @property
    def lam(self):
        if self.plane_stress:
            return self.E * self.nu / (1.0 - self.nu ** 2)
        return self.E * self.nu / ((1 + self.nu) * (1 - 2 * self.nu))

    @property
    def mu(self):
        return self.E / (2 * (1 + self.nu))

    @property
    def kappa(self):
        return self.E / (3.0 * (1.0 - 2.0 * self.nu))

    @property
    def c_p(self):
        return math.sqrt((self.lam + 2 * self.mu) / self.rho)

    def degradation(self, d):
        """'standard' g(d) = (1-d)^2 (1-eta) + eta  (material.py:528)."""
        return (1.0 - d) ** 2 * (1.0 - self.eta) + self.eta


# ----------------------------------------------------------------------------
# strain / stress / energy  (fem_operators.py)
# ----------------------------------------------------------------------------

def strain(geo: Q4Geometry, u):
    """_compute_strain_q4 (fem_operators.py:244-254)."""
    gp = geo.grad
    ue = u[geo.elements]
    exx = np.einsum("eqa,ea->eq", gp[..., 0], ue[..., 0])
    eyy = np.einsum("eqa,ea->eq", gp[..., 1], ue[..., 1])
    gxy = np.einsum("eqa,ea->eq", gp[..., 1], ue[..., 0]) + np.einsum("eqa,ea->eq", gp[..., 0], ue[..., 1])
    return exx, eyy, gxy


def _ezz(mat, tr2):
    return -mat.nu / (1.0 - mat.nu) * tr2 if mat.plane_stress else 0.0 * tr2


class Dual:
    """A value and its directional derivative (forward-mode differentiation of the stress
    formulas below): the JVP QuasiStaticSolver takes of internal_force with autograd
    (mechanics_solver.py:1705-1733, 2000-2012), restated for the oracle."""

    __array_ufunc__ = None  # numpy arrays defer to the reflected operators below

    def __init__(self, v, d):
        self.v, self.d = np.asarray(v, dtype=float), np.asarray(d, dtype=float)

    @staticmethod
    def _split(o):
        return (o.v, o.d) if isinstance(o, Dual) else (o, 0.0)

    def __add__(self, o):
        ov, od = Dual._split(o)
        return Dual(self.v + ov, self.d + od)

    __radd__ = __add__

    def __sub__(self, o):
        ov, od = Dual._split(o)
        return Dual(self.v - ov, self.d - od)

    def __rsub__(self, o):
        ov, od = Dual._split(o)
        return Dual(ov - self.v, od - self.d)

    def __neg__(self):
        return Dual(-self.v, -self.d)

    def __mul__(self, o):
        ov, od = Dual._split(o)
        return Dual(self.v * ov, self.d * ov + self.v * od)

    __rmul__ = __mul__

    def __truediv__(self, o):
        ov, od = Dual._split(o)
        return Dual(self.v / ov, (self.d * ov - self.v * od) / (ov * ov))

    def __rtruediv__(self, o):
        ov, od = Dual._split(o)
        return Dual(ov / self.v, (od * self.v - ov * self.d) / (self.v * self.v))


def _value(x):
    return x.v if isinstance(x, Dual) else x


def _pos(x):
    """max(x, 0); its derivative is taken as 1 where x >= 0 (the JVP of clamp(min=0))."""
    if isinstance(x, Dual):
        return Dual(np.maximum(x.v, 0.0), np.where(x.v >= 0, x.d, 0.0))
    return np.maximum(x, 0.0)


def _sqrt(x):
    if isinstance(x, Dual):
        r = np.sqrt(x.v)
        return Dual(r, x.d / (2.0 * r))
    return np.sqrt(x)


def _where(c, a, b):
    if isinstance(a, Dual) or isinstance(b, Dual):
        av, ad = Dual._split(a)
        bv, bd = Dual._split(b)
        return Dual(np.where(c, av, bv), np.where(c, ad, bd))
    return np.where(c, a, b)


def stress_split(mat: Mat2D, split, exx, eyy, gxy, g):
    """compute_stress_* (fem_operators.py:283-560) for one split."""
    lam, mu, kap = mat.lam, mat.mu, mat.kappa
    if split == "linear":
        return (lam + 2 * mu) * exx + lam * eyy, lam * exx + (lam + 2 * mu) * eyy, mu * gxy
    if split == "isotropic":
        return (g * ((lam + 2 * mu) * exx + lam * eyy), g * (lam * exx + (lam + 2 * mu) * eyy), g * (mu * gxy))
    if split == "amor":
        tr2 = exx + eyy
        tr = tr2 + _ezz(mat, tr2)
        trp = _pos(tr)
        trm = tr - trp
        return (g * (kap * trp + 2 * mu * (exx - tr / 3.0)) + kap * trm,
                g * (kap * trp + 2 * mu * (eyy - tr / 3.0)) + kap * trm,
                g * mu * gxy)
    if split in ("spectral", "spectral_stress"):
        exy = gxy / 2.0
        trace = exx + eyy
        hd = (exx - eyy) / 2.0
        delta = _sqrt(hd * hd + exy * exy + mat.spectral_eps)
        e1 = trace / 2.0 + delta
        e2 = trace / 2.0 - delta
        inv2d = 1.0 / (2.0 * delta + 1e-30)
        pxx = (hd + delta) * inv2d
        pyy = (-hd + delta) * inv2d
        pxy = exy * inv2d
        if split == "spectral":
            e1p, e2p = _pos(e1), _pos(e2)
            trp = _pos(trace)
            trm = trace - trp
            xxp = e1p * pxx + e2p * (1 - pxx)
            yyp = e1p * pyy + e2p * (1 - pyy)
            xyp = (e1p - e2p) * pxy
            return (g * (lam * trp + 2 * mu * xxp) + (lam * trm + 2 * mu * (exx - xxp)),
                    g * (lam * trp + 2 * mu * yyp) + (lam * trm + 2 * mu * (eyy - yyp)),
                    g * (2 * mu * xyp) + 2 * mu * (exy - xyp))
        s1 = lam * trace + 2 * mu * e1
        s2 = lam * trace + 2 * mu * e2
        s1p, s2p = _pos(s1), _pos(s2)
        s1m, s2m = s1 - s1p, s2 - s2p
        return (g * (s1p * pxx + s2p * (1 - pxx)) + (s1m * pxx + s2m * (1 - pxx)),
                g * (s1p * pyy + s2p * (1 - pyy)) + (s1m * pyy + s2m * (1 - pyy)),
                g * ((s1p - s2p) * pxy) + (s1m - s2m) * pxy)
    if split == "star_convex":
        tr2 = exx + eyy
        tr = tr2 + _ezz(mat, tr2)
        t = _value(tr) >= 0
        sxx_t = g * ((lam + 2 * mu) * exx + lam * eyy)
        syy_t = g * (lam * exx + (lam + 2 * mu) * eyy)
        sxy_t = g * (mu * gxy)
        sxx_c = g * 2 * mu * (exx - tr / 3.0) + kap * tr
        syy_c = g * 2 * mu * (eyy - tr / 3.0) + kap * tr
        sxy_c = g * mu * gxy
        return _where(t, sxx_t, sxx_c), _where(t, syy_t, syy_c), _where(t, sxy_t, sxy_c)
    raise ValueError(split)


def psi_plus(mat: Mat2D, exx, eyy, gxy, split=None):
    """compute_psi_plus and _psi_plus_* (fem_operators.py:951-1161)."""
    split = mat.split if split is None else split
    lam, mu, kap = mat.lam, mat.mu, mat.kappa
    exy = gxy / 2.0
    if split == "isotropic":
        tr = exx + eyy
        return 0.5 * lam * tr ** 2 + mu * (exx ** 2 + eyy ** 2 + 2 * exy ** 2)
    if split == "amor":
        tr2 = exx + eyy
        ezz = _ezz(mat, tr2)
        tr = tr2 + ezz
        trp = np.maximum(tr, 0)
        dd = (exx - tr / 3) ** 2 + (eyy - tr / 3) ** 2 + (ezz - tr / 3) ** 2 + 2 * exy ** 2
        return 0.5 * kap * trp ** 2 + mu * dd
    if split in ("spectral", "spectral_stress"):
        trace = exx + eyy
        delta = np.sqrt(((exx - eyy) / 2) ** 2 + exy ** 2 + mat.spectral_eps)
        e1, e2 = trace / 2 + delta, trace / 2 - delta
        if split == "spectral":
            return 0.5 * lam * np.maximum(trace, 0) ** 2 + mu * (np.maximum(e1, 0) ** 2 + np.maximum(e2, 0) ** 2)
        s1p = np.maximum(lam * trace + 2 * mu * e1, 0)
        s2p = np.maximum(lam * trace + 2 * mu * e2, 0)
        return (s1p ** 2 + s2p ** 2 - 2.0 * mat.nu * s1p * s2p) / (2.0 * mat.E)
    if split == "star_convex":
        tr2 = exx + eyy
        ezz = _ezz(mat, tr2)
        tr = tr2 + ezz
        full = 0.5 * lam * tr2 ** 2 + mu * (exx ** 2 + eyy ** 2 + 2 * exy ** 2)
        dev = mu * ((exx - tr / 3) ** 2 + (eyy - tr / 3) ** 2 + (ezz - tr / 3) ** 2 + 2 * exy ** 2)
        return np.where(tr >= 0, full, dev)
    raise ValueError(split)


def d_at_qp(geo, d):
    return np.einsum("qa,ea->eq", geo.N, d[geo.elements])


def assemble_force(geo, sxx, syy, sxy):
    """_assemble_force_q4 (fem_operators.py:681-699)."""
    gp, w = geo.grad, geo.wdet
    fx = ((gp[..., 0] * sxx[..., None] + gp[..., 1] * sxy[..., None]) * w[..., None]).sum(1)
    fy = ((gp[..., 1] * syy[..., None] + gp[..., 0] * sxy[..., None]) * w[..., None]).sum(1)
    f = np.zeros((geo.n_nodes, 2))
    np.add.at(f[:, 0], geo.elements.reshape(-1), fx.reshape(-1))
    np.add.at(f[:, 1], geo.elements.reshape(-1), fy.reshape(-1))
    return f


def internal_force(geo, mat: Mat2D, u, d):
    """internal_force (fem_operators.py:598-612) with compute_stress (:614-653)."""
    exx, eyy, gxy = strain(geo, u)
    if d is None:
        s = stress_split(mat, "linear", exx, eyy, gxy, None)
    else:
        g = mat.degradation(d_at_qp(geo, d))
        s = stress_split(mat, mat.stress_split or mat.split, exx, eyy, gxy, g)
    return assemble_force(geo, *s)


def tangent_action(geo, mat: Mat2D, u, du, d):
    """d internal_force(u, d)/du [du]: the JVP QuasiStaticSolver uses as its CG operator for the
    spectral, Amor and star-convex splits (mechanics_solver.py:1705-1733, 2000-2012), by
    forward-mode differentiation of stress_split at the strain of u with g(d) fixed."""
    exx, eyy, gxy = strain(geo, u)
    dxx, dyy, dxy = strain(geo, du)
    g = mat.degradation(d_at_qp(geo, d))
    split = mat.stress_split or mat.split
    s = stress_split(mat, split, Dual(exx, dxx), Dual(eyy, dyy), Dual(gxy, dxy), g)
    return assemble_force(geo, *(x.d if isinstance(x, Dual) else 0.0 * exx for x in s))


def stiffness_diagonal(geo, mat: Mat2D, d=None):
    """stiffness_diagonal Q4 branch (fem_operators.py:1284-1320)."""
    lam, mu = mat.lam, mat.mu
    C00, C11, C22 = lam + 2 * mu, lam + 2 * mu, mu
    g = np.ones_like(geo.wdet) if d is None else mat.degradation(d_at_qp(geo, d))
    gp = geo.grad
    w = g * geo.wdet
    kxx = (w[..., None] * (C00 * gp[..., 0] ** 2 + C22 * gp[..., 1] ** 2)).sum(1)
    kyy = (w[..., None] * (C11 * gp[..., 1] ** 2 + C22 * gp[..., 0] ** 2)).sum(1)
    out = np.zeros((geo.n_nodes, 2))
    np.add.at(out[:, 0], geo.elements.reshape(-1), kxx.reshape(-1))
    np.add.at(out[:, 1], geo.elements.reshape(-1), kyy.reshape(-1))
    return out


def laplacian_matvec(geo, d):
    """_q4_laplacian_matvec (fem_operators.py:1253-1266)."""
    gp, w = geo.grad, geo.wdet
    de = d[geo.elements]
    gdx = np.einsum("eqa,ea->eq", gp[..., 0], de)
    gdy = np.einsum("eqa,ea->eq", gp[..., 1], de)
    r = ((gp[..., 0] * gdx[..., None] + gp[..., 1] * gdy[..., None]) * w[..., None]).sum(1)
    out = np.zeros(geo.n_nodes)
    np.add.at(out, geo.elements.reshape(-1), r.reshape(-1))
    return out


def mass_matvec(geo, d):
    """_q4_mass_matvec (fem_operators.py:1268-1277)."""
    dq = d_at_qp(geo, d)
    r = np.einsum("qa,eq,eq->ea", geo.N, dq, geo.wdet)
    out = np.zeros(geo.n_nodes)
    np.add.at(out, geo.elements.reshape(-1), r.reshape(-1))
    return out


# ----------------------------------------------------------------------------
# damage operator (solvers/damage_solver.py Q4 path)
# ----------------------------------------------------------------------------

def damage_apply(geo, d, reaction_density, gc_l0, gc_l0_e=None):
    """_Ax_q4 (damage_solver.py:1797-1838).

    ``reaction_density`` is ``2H_q + Gc/l0`` (E, 4); ``gc_l0`` the scalar
    ``Gc*l0`` and ``gc_l0_e`` an optional per-element ``Gc_e*l0`` (E,).
    """
    gp, w, N = geo.grad, geo.wdet, geo.N
    de = d[geo.elements]
    gdx = np.einsum("eqa,ea->eq", gp[..., 0], de)
    gdy = np.einsum("eqa,ea->eq", gp[..., 1], de)
    lap = (w[..., None] * (gp[..., 0] * gdx[..., None] + gp[..., 1] * gdy[..., None])).sum(1)
    lap = lap * (gc_l0 if gc_l0_e is None else gc_l0_e[:, None])
    dq = np.einsum("qa,ea->eq", N, de)
    mass = np.einsum("qa,eq->ea", N, reaction_density * dq * w)
    out = np.zeros(geo.n_nodes)
    np.add.at(out, geo.elements.reshape(-1), (lap + mass).reshape(-1))
    return out


def damage_prepare(geo, H_q, gc_over_l0, gc_l0, gc_over_l0_e=None, gc_l0_e=None):
    """_prepare_cg_q4 (damage_solver.py:2270-2301): (reaction_density, b, M_inv)."""
    N, w = geo.N, geo.wdet
    ratio = gc_over_l0 if gc_over_l0_e is None else gc_over_l0_e[:, None]
    rd = 2.0 * H_q + ratio
    b = np.zeros(geo.n_nodes)
    np.add.at(b, geo.elements.reshape(-1), np.einsum("qa,eq->ea", N, 2.0 * H_q * w).reshape(-1))
    diag_lap = (w[..., None] * (geo.grad[..., 0] ** 2 + geo.grad[..., 1] ** 2)).sum(1)
    lap_diag = (gc_l0 if gc_l0_e is None else gc_l0_e[:, None]) * diag_lap
    mass_diag = np.einsum("qa,eq->ea", N * N, rd * w)
    A = np.zeros(geo.n_nodes)
    np.add.at(A, geo.elements.reshape(-1), (lap_diag + mass_diag).reshape(-1))
    return rd, b, 1.0 / (A + 1e-30)


def energy_components(geo, mat: Mat2D, u, d, v=None):
    """compute_energy_components Q4 branch (fem_operators.py:1430-1496), AT2."""
    exx, eyy, gxy = strain(geo, u)
    pp = psi_plus(mat, exx, eyy, gxy)
    g = mat.degradation(d_at_qp(geo, d))
    pm = psi_plus(mat, exx, eyy, gxy, "isotropic") - pp
    el = float(((g * pp + pm) * geo.wdet).sum())
    surf = mat.Gc / (2 * mat.l0) * float(d @ mass_matvec(geo, d))
    grad = mat.Gc * mat.l0 / 2 * float(d @ laplacian_matvec(geo, d))
    kin = 0.0
    if v is not None:
        kin = 0.5 * mat.rho * float(((v ** 2).sum(1) * geo.M_scalar).sum())
    return {"elastic": el, "kinetic": kin, "fracture": surf + grad, "total": el + kin + surf + grad}


def reaction_force(geo, mat, u, d, nodes, component=1, f_ext=None):
    """compute_reaction_force (fem_operators.py:1502-1530)."""
    f = internal_force(geo, mat, u, d)
    r = f[nodes, component]
    if f_ext is not None:
        r = r - f_ext[nodes, component]
    return float(r.sum())

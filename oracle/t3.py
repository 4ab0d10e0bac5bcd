"""T3 (linear triangle, one-point) operators and damage system in numpy.  TEST ORACLE ONLY.

Restates the triangle branches of PhAST: ``FEMMesh._precompute`` (T3 geometry,
src/phast/core/mesh.py:236-303), ``FEMOperators.compute_strain`` /
``compute_stress`` / ``_assemble_force`` (src/phast/core/fem_operators.py:223-242,
614-680) and the element-H AT2 damage system of ``PhaseFieldDamageSolver``
(``_Ax`` damage_solver.py:1702-1755, ``_prepare_cg`` :2121-2265,
``_compute_preconditioner`` :2095-2119).  The stress splits and psi+ are the
pointwise functions of ``oracle.q4`` evaluated at the element centroid.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .q4 import Mat2D, psi_plus, stress_split


@dataclass
class T3Geometry:
    nodes: np.ndarray
    elements: np.ndarray  # (E, 3)
    areas: np.ndarray     # (E,)
    grad: np.ndarray      # (E, 3, 2)
    M_scalar: np.ndarray  # (N,) lumped mass (area / 3 per corner)

    @property
    def n_nodes(self):
        return self.nodes.shape[0]

    @property
    def n_elems(self):
        return self.elements.shape[0]


def geometry(nodes, elements) -> T3Geometry:
    """P1 gradients with the sign-preserving area regularisation of mesh.py:236-268."""
    nodes = np.asarray(nodes, dtype=np.float64)
    el = np.asarray(elements, dtype=np.int64)
    p0, p1, p2 = nodes[el[:, 0]], nodes[el[:, 1]], nodes[el[:, 2]]
    v01, v02 = p1 - p0, p2 - p0
    s2a = v01[:, 0] * v02[:, 1] - v01[:, 1] * v02[:, 0]
    areas = 0.5 * np.abs(s2a)
    sgn = np.sign(s2a)
    sgn[sgn == 0] = 1.0
    inv = 1.0 / np.where(np.abs(s2a) > 1e-10, s2a, sgn * 1e-10)
    g = np.zeros((el.shape[0], 3, 2))
    g[:, 0, 0] = (p1[:, 1] - p2[:, 1]) * inv
    g[:, 0, 1] = (p2[:, 0] - p1[:, 0]) * inv
    g[:, 1, 0] = (p2[:, 1] - p0[:, 1]) * inv
    g[:, 1, 1] = (p0[:, 0] - p2[:, 0]) * inv
    g[:, 2, 0] = (p0[:, 1] - p1[:, 1]) * inv
    g[:, 2, 1] = (p1[:, 0] - p0[:, 0]) * inv
    M = np.zeros(nodes.shape[0])
    np.add.at(M, el.reshape(-1), np.repeat(areas / 3.0, 3))
    return T3Geometry(nodes, el, areas, g, M)


def strain(geo, u):
    """compute_strain, fem_operators.py:223-242: one value per element."""
    ue = u[geo.elements]
    gp = geo.grad
    exx = (gp[:, :, 0] * ue[:, :, 0]).sum(1)
    eyy = (gp[:, :, 1] * ue[:, :, 1]).sum(1)
    gxy = (gp[:, :, 1] * ue[:, :, 0]).sum(1) + (gp[:, :, 0] * ue[:, :, 1]).sum(1)
    return exx, eyy, gxy


def assemble_force(geo, sxx, syy, sxy):
    """_assemble_force, fem_operators.py:661-679."""
    gp, A = geo.grad, geo.areas[:, None]
    fx = A * (sxx[:, None] * gp[:, :, 0] + sxy[:, None] * gp[:, :, 1])
    fy = A * (sxy[:, None] * gp[:, :, 0] + syy[:, None] * gp[:, :, 1])
    f = np.zeros((geo.n_nodes, 2))
    np.add.at(f[:, 0], geo.elements.reshape(-1), fx.reshape(-1))
    np.add.at(f[:, 1], geo.elements.reshape(-1), fy.reshape(-1))
    return f


def internal_force(geo, mat: Mat2D, u, d):
    """internal_force with compute_stress (fem_operators.py:598-653): g at the centroid mean of d."""
    exx, eyy, gxy = strain(geo, u)
    if d is None:
        return assemble_force(geo, *stress_split(mat, "linear", exx, eyy, gxy, None))
    g = mat.degradation(d[geo.elements].mean(1))
    return assemble_force(geo, *stress_split(mat, mat.stress_split or mat.split, exx, eyy, gxy, g))


def psi(geo, mat: Mat2D, u):
    """compute_psi_plus, one value per element."""
    return psi_plus(mat, *strain(geo, u))


def reaction_coeff(geo, H, gc_over_l0):
    """(2 H_e + Gc/l0) A_e / 12 (_prepare_cg, damage_solver.py:2168-2177)."""
    return (2.0 * np.asarray(H) + gc_over_l0) * geo.areas / 12.0


def damage_apply(geo, d, rc, gc_l0):
    """_Ax, damage_solver.py:1702-1755: Gc l0 K d + consistent reaction mass."""
    de = d[geo.elements]
    gp = geo.grad
    gx = (gp[:, :, 0] * de).sum(1)
    gy = (gp[:, :, 1] * de).sum(1)
    lap = geo.areas[:, None] * (gp[:, :, 0] * gx[:, None] + gp[:, :, 1] * gy[:, None])
    mass = rc[:, None] * (de + de.sum(1)[:, None])
    y = np.zeros(geo.n_nodes)
    np.add.at(y, geo.elements.reshape(-1), (gc_l0 * lap + mass).reshape(-1))
    return y


def damage_prepare(geo, H, gc_over_l0, gc_l0):
    """b = sum 2 H_e A_e / 3 and M_inv = 1 / (Gc l0 diag_lap + 2 rc_e) (damage_solver.py:2095-2265)."""
    rc = reaction_coeff(geo, H, gc_over_l0)
    b = np.zeros(geo.n_nodes)
    np.add.at(b, geo.elements.reshape(-1), np.repeat(2.0 * np.asarray(H) * geo.areas / 3.0, 3))
    gp = geo.grad
    diag_lap = geo.areas[:, None] * (gp[:, :, 0] ** 2 + gp[:, :, 1] ** 2)
    dg = np.zeros(geo.n_nodes)
    np.add.at(dg, geo.elements.reshape(-1), (gc_l0 * diag_lap + 2.0 * rc[:, None]).reshape(-1))
    return rc, b, 1.0 / (dg + 1e-30)


def damage_prepare_at1(geo, H, gc, l0, source=None):
    """AT1 with element history (damage_solver.py:1325-1329, 2060-2080): the AT2 system with
    Gc l0 -> 3 Gc l0 / 4, no Gc/l0 reaction, right-hand side (2 H_e - S) A_e / 3 with the source
    S = 3 Gc / (8 l0).  Returns (rc, b, M_inv, gc_l0)."""
    src = 3.0 * gc / (8.0 * l0) if source is None else source
    gc_l0 = 0.75 * gc * l0
    rc, b, mi = damage_prepare(geo, H, 0.0, gc_l0)
    np.add.at(b, geo.elements.reshape(-1), np.repeat(-src * geo.areas / 3.0, 3))
    return rc, b, mi, gc_l0


def damage_apply_nodal(geo, d, Hn, gc_over_l0, gc_l0):
    """_Ax_nodal (damage_solver.py:1840-1912): Gc l0 K d + the reaction mass of 2 H with H
    interpolated from the nodes (triple products A/10, A/30, A/60) + Gc/l0 M d."""
    de = d[geo.elements]
    he = np.asarray(Hn)[geo.elements]
    gp = geo.grad
    gx = (gp[:, :, 0] * de).sum(1)
    gy = (gp[:, :, 1] * de).sum(1)
    lap = geo.areas[:, None] * (gp[:, :, 0] * gx[:, None] + gp[:, :, 1] * gy[:, None])
    sh, sd, hd = he.sum(1), de.sum(1), (he * de).sum(1)
    mh = (geo.areas / 30.0)[:, None] * ((2.0 * he + sh[:, None]) * de + (he + sh[:, None]) * sd[:, None] +
                                        hd[:, None])
    mg = (gc_over_l0 * geo.areas / 12.0)[:, None] * (de + sd[:, None])
    y = np.zeros(geo.n_nodes)
    np.add.at(y, geo.elements.reshape(-1), (gc_l0 * lap + mh + mg).reshape(-1))
    return y


def damage_prepare_nodal(geo, Hn, gc_over_l0, gc_l0):
    """_prepare_cg_nodal (damage_solver.py:2303-2348): b_a = A/6 (H_a + S_H) and the Jacobi inverse
    of Gc l0 diag_lap + (2 H_a + S_H) A/15 + Gc/l0 A/6."""
    he = np.asarray(Hn)[geo.elements]
    sh = he.sum(1)
    b = np.zeros(geo.n_nodes)
    np.add.at(b, geo.elements.reshape(-1), ((geo.areas / 6.0)[:, None] * (he + sh[:, None])).reshape(-1))
    gp = geo.grad
    diag_lap = geo.areas[:, None] * (gp[:, :, 0] ** 2 + gp[:, :, 1] ** 2)
    md = (geo.areas / 15.0)[:, None] * (2.0 * he + sh[:, None]) + (gc_over_l0 * geo.areas / 6.0)[:, None]
    dg = np.zeros(geo.n_nodes)
    np.add.at(dg, geo.elements.reshape(-1), (gc_l0 * diag_lap + md).reshape(-1))
    return b, 1.0 / (dg + 1e-30)


def color_elements(elements, n_nodes):
    """Greedy colouring: no two elements of one colour share a node (first-fit, element order)."""
    el = np.asarray(elements, dtype=np.int64)
    node_colors = [set() for _ in range(n_nodes)]
    colors = np.zeros(el.shape[0], dtype=np.int64)
    for e, tri in enumerate(el):
        used = set().union(*(node_colors[v] for v in tri))
        c = 0
        while c in used:
            c += 1
        colors[e] = c
        for v in tri:
            node_colors[v].add(c)
    return colors

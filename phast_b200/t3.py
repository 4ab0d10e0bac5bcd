"""Unstructured linear triangles (T3) behind PhAST's ``FEMOperators`` and
``PhaseFieldDamageSolver`` interfaces.

PhAST's default 2D element is the T3 (src/phast/core/mesh.py:236-303,
core/fem_operators.py T3 branches, solvers/damage_solver.py element-H AT2 path).
The geometry (P1 gradients, areas, lumped mass, incircle sizes) is computed once
on the device; the elements are greedily coloured on the host so that the CUDA
kernels scatter element contributions colour by colour without atomics.
``FEMOperators`` / ``PhaseFieldDamageSolver`` construct these classes when the
mesh's ``element_type`` is ``'T3'``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr, raw, stream


def color_elements(elements, n_nodes):
    """Greedy first-fit colouring in element order: no colour touches a node twice."""
    el = np.asarray(elements, dtype=np.int64)
    used = np.zeros(n_nodes, dtype=np.uint64)
    colors = np.empty(el.shape[0], dtype=np.int64)
    for e in range(el.shape[0]):
        a, b, c = el[e]
        busy = int(used[a] | used[b] | used[c])
        k = 0
        while busy >> k & 1:
            k += 1
        if k >= 64:
            raise RuntimeError("T3 colouring needs more than 64 colours")
        colors[e] = k
        bit = np.uint64(1 << k)
        used[a] |= bit
        used[b] |= bit
        used[c] |= bit
    return colors


class T3FEMOperators:
    """GPU operators of a T3 mesh (core/fem_operators.py, triangle branches)."""

    def __init__(self, mesh, material):
        from .fem2d import q4_material_struct
        self.mesh = mesh
        self.material = material
        self.device = torch.device(getattr(mesh, "device", "cuda"))
        if self.device.type != "cuda":
            raise ValueError("the B200 backend needs the mesh on a CUDA device")
        self.dtype = torch.float64
        nodes = mesh.nodes.detach().to(self.device, torch.float64)
        el = mesh.elements.detach().to(self.device, torch.long)
        if el.ndim != 2 or el.shape[1] != 3:
            raise ValueError("T3 connectivity must have shape (E, 3)")
        self.n_nodes, self.n_elems = int(nodes.shape[0]), int(el.shape[0])
        p0, p1, p2 = nodes[el[:, 0]], nodes[el[:, 1]], nodes[el[:, 2]]
        v01, v02, v12 = p1 - p0, p2 - p0, p2 - p1
        s2a = v01[:, 0] * v02[:, 1] - v01[:, 1] * v02[:, 0]
        self.areas = (0.5 * s2a.abs()).contiguous()
        sgn = torch.sign(s2a)
        sgn[sgn == 0] = 1.0
        inv = 1.0 / torch.where(s2a.abs() > 1e-10, s2a, sgn * 1e-10)  # mesh.py:252-258
        g = torch.empty(self.n_elems, 3, 2, dtype=torch.float64, device=self.device)
        g[:, 0, 0] = (p1[:, 1] - p2[:, 1]) * inv
        g[:, 0, 1] = (p2[:, 0] - p1[:, 0]) * inv
        g[:, 1, 0] = (p2[:, 1] - p0[:, 1]) * inv
        g[:, 1, 1] = (p0[:, 0] - p2[:, 0]) * inv
        g[:, 2, 0] = (p0[:, 1] - p1[:, 1]) * inv
        g[:, 2, 1] = (p1[:, 0] - p0[:, 0]) * inv
        self.grad_phi = g.contiguous()
        perim = v01.norm(dim=1) + v12.norm(dim=1) + v02.norm(dim=1)
        self.elem_h = 4.0 * self.areas / (perim + 1e-30)
        self.h_min = float(self.elem_h.min())
        self.M_scalar = torch.zeros(self.n_nodes, dtype=torch.float64, device=self.device)
        self.M_scalar.scatter_add_(0, el.reshape(-1), (self.areas / 3.0).unsqueeze(1).expand(-1, 3).reshape(-1))
        self.M_vec = material.rho * self.M_scalar.unsqueeze(1).expand(-1, 2).flatten()
        self.M_vec_inv = 1.0 / (self.M_vec + 1e-30)
        self.dt_cfl = self.h_min / material.c_p
        self.diff_E_field = None
        colors = color_elements(el.cpu().numpy(), self.n_nodes)
        order = np.argsort(colors, kind="stable")
        self.n_colors = int(colors.max()) + 1
        off = np.searchsorted(colors[order], np.arange(self.n_colors + 1))
        self._elem32 = el.to(torch.int32).contiguous()
        self._order = torch.as_tensor(order.astype(np.int32), device=self.device)
        self._color_off = (C.c_int * (self.n_colors + 1))(*[int(v) for v in off])
        # the colour kernels trust the colouring: check it once, on the host, before any launch
        el_h = np.ascontiguousarray(el.cpu().numpy().astype(np.int32))
        ord_h = np.ascontiguousarray(order.astype(np.int32))
        IP = C.POINTER(C.c_int)
        _lib.call("phastb_t3_check_mesh", self.n_nodes, self.n_elems, el_h.ctypes.data_as(IP),
                  ord_h.ctypes.data_as(IP), self.n_colors, self._color_off)
        self.t3 = _lib.T3Mesh(self.n_nodes, self.n_elems, self.n_colors, 0, ptr(self._elem32), ptr(self._order),
                              self._color_off, ptr(self.grad_phi), ptr(self.areas))
        self._mat = q4_material_struct(material, torch.float64)

    def mat(self, dtype=None):
        return self._mat

    def _nodal(self, t, comps, name):
        shape = (self.n_nodes, comps) if comps > 1 else (self.n_nodes,)
        if tuple(t.shape) != shape:
            raise ValueError(f"{name} must have shape {shape}, got {tuple(t.shape)}")
        _lib.require_cuda(t, name)
        return t.to(torch.float64).contiguous()

    def internal_force(self, u, d):
        """f = sum_e A_e B_e^T sigma(u, d_e), d_e the element mean (fem_operators.py:598-680)."""
        u = self._nodal(u, 2, "u")
        dd = None if d is None else self._nodal(d, 1, "d")
        f = torch.empty_like(u)
        call("phastb_t3_internal_force", self.t3, self._mat, ptr(u), ptr(dd), ptr(f), stream())
        return f

    def internal_force_linear(self, u):
        return self.internal_force(u, None)

    def compute_psi_plus(self, u, strain=None, d=None):
        """psi+ per element for the material's energy split (fem_operators.py:951-1025)."""
        u = self._nodal(u, 2, "u")
        psi = torch.empty(self.n_elems, dtype=torch.float64, device=self.device)
        call("phastb_t3_psi_history", self.t3, self._mat, ptr(u), None, None, ptr(psi), stream())
        return psi

    def psi_history(self, u, H_in=None, H_out=None):
        """H_out = max(H_in, psi+(u)) per element (StaggeredSolver._H_update)."""
        u = self._nodal(u, 2, "u")
        H = torch.empty(self.n_elems, dtype=torch.float64, device=self.device) if H_out is None else H_out
        hin = None if H_in is None else H_in.to(torch.float64).contiguous()
        call("phastb_t3_psi_history", self.t3, self._mat, ptr(u), ptr(hin), ptr(H), None, stream())
        return H

    def compute_reaction_force(self, u, d, node_indices, component=1, f_ext=None):
        """Sum of f_int (- f_ext) over nodes (fem_operators.py:1502-1530); returns a float."""
        f = self.internal_force(u, d)
        idx = torch.as_tensor(node_indices, dtype=torch.long).to(self.device)
        r = f[idx, component].sum()
        if f_ext is not None:
            r = r - f_ext.to(torch.float64)[idx, component].sum()
        return float(r)

    # -- adjoint pieces (isotropic split) -------------------------------------------
    def psi_grad_t(self, u, w):
        """sum_e w_e (d psi+_e / du): the transpose of the element energy map, (N, 2)."""
        u = self._nodal(u, 2, "u")
        w = w.to(torch.float64).contiguous()
        f = torch.empty_like(u)
        call("phastb_t3_psi_grad_t", self.t3, self._mat, ptr(u), ptr(w), ptr(f), stream())
        return f

    def force_dd_t(self, u, z, d):
        """d/dd [z . f_int(u, d)], (N,)."""
        u, z, d = self._nodal(u, 2, "u"), self._nodal(z, 2, "z"), self._nodal(d, 1, "d")
        out = torch.empty_like(d)
        call("phastb_t3_force_dd_t", self.t3, self._mat, ptr(u), ptr(z), ptr(d), ptr(out), stream())
        return out


class T3DamageSolver:
    """Bound-projected PCG damage solve on a T3 mesh: AT2 with element or nodal history
    (``nodal_H``), AT1 with element history (the combinations the reference supports,
    damage_solver.py:1225-1236)."""

    def __init__(self, fem, tol=1e-5, max_iter=5000, bounds_method="projected_cg", nodal_H=False):
        if bounds_method != "projected_cg":
            raise NotImplementedError("the B200 backend implements bounds_method='projected_cg'")
        mat = fem.material
        self._pf_model = str(getattr(mat, "pf_model", "AT2")).upper()
        if self._pf_model not in ("AT2", "AT1"):
            raise NotImplementedError("T3 damage supports pf_model='AT2' and 'AT1'")
        if nodal_H and self._pf_model != "AT2":
            raise NotImplementedError(f"pf_model={self._pf_model!r} with nodal_H=True is not implemented "
                                      "(the nodal-history system is AT2's)")
        self.nodal_H = bool(nodal_H)
        self.fem = fem
        self.material = mat
        self.tol = float(tol)
        self.max_iter = int(max_iter)
        self._Gc, self._l0 = float(mat.Gc), float(mat.l0)
        self.check_every = 10
        self.last_iter = 0
        self.last_converged = True
        self.n_solves = 0
        self._ws = _lib.Workspace(fem.device)

    def _coeffs(self, Gc=None, l0=None, Gc_field=None):
        if self._pf_model != "AT2" or self.nodal_H:
            if Gc is not None or l0 is not None or Gc_field is not None:
                raise NotImplementedError("material overrides are implemented for element-history AT2")
        Gc_s = self._Gc if Gc is None else float(Gc)
        l0_s = self._l0 if l0 is None else float(l0)
        gcl0_e = gco_e = None
        if Gc_field is not None:
            gf = torch.as_tensor(Gc_field, dtype=torch.float64, device=self.fem.device).reshape(-1)
            if gf.numel() != self.fem.n_elems:
                raise ValueError("Gc_field must have one value per element")
            gcl0_e, gco_e = (gf * l0_s).contiguous(), (gf / l0_s).contiguous()
        return Gc_s * l0_s, Gc_s / l0_s, gcl0_e, gco_e

    def _model(self):
        """The C-ABI model of AT1 or nodal-history AT2 (damage_solver.py:1316-1340), else None."""
        if self._pf_model == "AT2" and not self.nodal_H:
            return None
        m = _lib.T3DamageModel()
        m.nodal_h = int(self.nodal_H)
        if self._pf_model == "AT1":
            m.gcl0, m.gc_over_l0 = 0.75 * self._Gc * self._l0, 0.0
            m.source = float(self.material.at1_source) if hasattr(self.material, "at1_source") else \
                3.0 * self._Gc / (8.0 * self._l0)
        else:
            m.gcl0, m.gc_over_l0, m.source = self._Gc * self._l0, self._Gc / self._l0, 0.0
        return m

    def _history(self, H):
        H = H.detach().to(torch.float64).contiguous()
        want = (self.fem.n_nodes,) if self.nodal_H else (self.fem.n_elems,)
        if tuple(H.shape) != want:
            raise ValueError(f"T3 damage expects {'nodal' if self.nodal_H else 'element'} H of shape {want}")
        return H

    def _Ax(self, d, reaction_H, Gc=None, l0=None, Gc_field=None):
        """(Gc l0 K + M(rc)) d with rc_e = (2 H_e + Gc/l0) A_e / 12 (damage_solver.py:1702-1755)."""
        gcl0, gco, gcl0_e, gco_e = self._coeffs(Gc, l0, Gc_field)
        d = d.to(torch.float64).contiguous()
        H = reaction_H.to(torch.float64).contiguous()
        y = torch.empty_like(d)
        model = self._model()
        if model is not None:
            call("phastb_t3_damage_apply_ex", self.fem.t3, C.byref(model), ptr(d), ptr(self._history(H)), ptr(y),
                 stream())
            return y
        call("phastb_t3_damage_apply", self.fem.t3, ptr(d), ptr(H), gco, ptr(gco_e), gcl0, ptr(gcl0_e), ptr(y),
             stream())
        return y

    def _apply_full(self, H_input, x, Gc=None, l0=None, Gc_field=None):
        """A x of the AT2 system (unmasked) with the given material overrides."""
        return self._Ax(x.detach(), H_input.detach(), Gc, l0, Gc_field)

    def linear_solve(self, H_input, rhs, Gc=None, l0=None, Gc_field=None, fixed=None, fixed_values=None, x0=None,
                     rtol=1e-11, max_iter=None):
        """Solve the unbounded AT2 system A x = rhs with ``fixed`` rows held at ``fixed_values``
        (_pcg_solve_adjoint_system, damage_solver.py:423-480)."""
        if self._model() is not None:
            raise NotImplementedError("the damage adjoint is implemented for element-history AT2")
        gcl0, gco, gcl0_e, gco_e = self._coeffs(Gc, l0, Gc_field)
        H = H_input.detach().to(torch.float64).contiguous()
        n = self.fem.n_nodes
        r = rhs.detach().to(torch.float64).contiguous()
        fx = None if fixed is None else fixed.to(torch.uint8).contiguous()
        fv = None if fixed_values is None else fixed_values.detach().to(torch.float64).contiguous()
        xi = None if x0 is None else x0.detach().to(torch.float64).contiguous()
        out = torch.empty(n, dtype=torch.float64, device=r.device)
        info = (C.c_int * 2)()
        rinfo = (C.c_double * 2)()
        wp, wn = self._ws.get(_lib.load().phastb_t3_damage_linear_workspace_bytes(n))
        call("phastb_t3_damage_linear_solve", self.fem.t3, ptr(H), gco, ptr(gco_e), gcl0, ptr(gcl0_e), ptr(r),
             ptr(fx), ptr(fv), ptr(xi), float(rtol), int(max_iter or max(self.max_iter, 1000)), self.check_every,
             ptr(out), info, rinfo, wp, wn, stream())
        self.last_linear_info = (int(info[0]), int(info[1]), float(rinfo[0]), float(rinfo[1]))
        if info[1] not in (0, 1):
            raise RuntimeError(f"adjoint damage PCG failed (reason {int(info[1])})")
        return out

    def adjoint_grads(self, lam, d, Gc_field=None, l0=None):
        """(dJ/dGc_e (E,), dJ/dH_e (E,)) for the adjoint ``lam`` of the damage solve at ``d``."""
        if self._model() is not None:
            raise NotImplementedError("the damage adjoint is implemented for element-history AT2")
        l0_s = self._l0 if l0 is None else float(l0)
        E, dev = self.fem.n_elems, d.device
        g_gc = torch.empty(E, dtype=torch.float64, device=dev)
        g_h = torch.empty(E, dtype=torch.float64, device=dev)
        lam = lam.to(torch.float64).contiguous()
        d = d.to(torch.float64).contiguous()
        call("phastb_t3_damage_adjoint_grads", self.fem.t3, ptr(lam), ptr(d), l0_s, ptr(g_gc), ptr(g_h), None, None,
             stream())
        return g_gc, g_h

    def prepare(self, H, Gc=None, l0=None, Gc_field=None):
        gcl0, gco, gcl0_e, gco_e = self._coeffs(Gc, l0, Gc_field)
        H = H.to(torch.float64).contiguous()
        b = torch.empty(self.fem.n_nodes, dtype=torch.float64, device=H.device)
        m = torch.empty_like(b)
        model = self._model()
        if model is not None:
            call("phastb_t3_damage_prepare_ex", self.fem.t3, C.byref(model), ptr(self._history(H)), ptr(b), ptr(m),
                 stream())
            return b, m
        call("phastb_t3_damage_prepare", self.fem.t3, ptr(H), gco, ptr(gco_e), gcl0, ptr(gcl0_e), ptr(b), ptr(m),
             stream())
        return b, m

    def solve(self, H_input, d_prev, Gc=None, l0=None, Gc_field=None, pf_dirichlet_mask=None,
              pf_dirichlet_values=None, initial_guess=None):
        """d in [d_prev, 1] by projected CG (damage_solver.py:2493-2640, 3528-3775)."""
        self.n_solves += 1
        gcl0, gco, gcl0_e, gco_e = self._coeffs(Gc, l0, Gc_field)
        H = self._history(H_input)
        dp = d_prev.detach().to(torch.float64).contiguous()
        di = None if initial_guess is None else initial_guess.detach().to(torch.float64).contiguous()
        fixed = vals = None
        if pf_dirichlet_mask is not None and bool(pf_dirichlet_mask.any()):
            if pf_dirichlet_values is None:
                raise ValueError("pf_dirichlet_values must be supplied with mask")
            fixed = pf_dirichlet_mask.to(device=dp.device, dtype=torch.uint8).contiguous()
            vals = pf_dirichlet_values.to(device=dp.device, dtype=torch.float64).contiguous()
        n = self.fem.n_nodes
        out = torch.empty(n, dtype=torch.float64, device=dp.device)
        info = (C.c_int * 2)()
        wp, wn = self._ws.get(_lib.load().phastb_t3_damage_solve_workspace_bytes(n))
        model = self._model()
        if model is not None:
            st = raw("phastb_t3_damage_solve_ex", self.fem.t3, C.byref(model), ptr(H), ptr(dp), ptr(di), ptr(fixed),
                     ptr(vals), self.tol, self.max_iter, self.check_every, ptr(out), info, wp, wn, stream())
            _lib.check(st, "phastb_t3_damage_solve_ex")
        else:
            st = raw("phastb_t3_damage_solve", self.fem.t3, ptr(H), gco, ptr(gco_e), gcl0, ptr(gcl0_e), ptr(dp),
                     ptr(di), ptr(fixed), ptr(vals), self.tol, self.max_iter, self.check_every, ptr(out), info, wp,
                     wn, stream())
            _lib.check(st, "phastb_t3_damage_solve")
        self.last_iter = int(info[0])
        self.last_converged = info[1] == 0
        return out.to(d_prev.dtype)

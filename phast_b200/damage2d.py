"""AT2 damage solve behind PhAST's ``PhaseFieldDamageSolver`` interface.

Mirrors ``phast.solvers.damage_solver.PhaseFieldDamageSolver`` (native Q4 AT2
branch, src/phast/solvers/damage_solver.py:1157-3775): ``solve`` runs the
bound-projected PCG of ``_solve_projected_cg`` entirely on the device with the
iteration state in GPU memory; the host looks at the state once per
``check_every`` iterations instead of at every dot product.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import call, ptr, raw, stream


class PhaseFieldDamageSolver:
    """GPU projected-CG AT2 damage solver for structured Q4 grids (T3 meshes: ``phast_b200.t3``)."""

    def __new__(cls, fem, *args, **kwargs):
        from .t3 import T3DamageSolver, T3FEMOperators
        if isinstance(fem, T3FEMOperators):
            keep = {k: kwargs[k] for k in ("tol", "max_iter", "bounds_method", "nodal_H") if k in kwargs}
            return T3DamageSolver(fem, *args[:2], **keep)
        return super().__new__(cls)

    def __init__(self, fem, tol=1e-5, max_iter=5000, ctx=None, use_multigrid=True, bounds_method="post_clamp",
                 preconditioner=None, nodal_H=False):
        if bounds_method not in ("post_clamp", "projected_cg", "direct"):
            raise ValueError(f"bounds_method must be 'post_clamp', 'projected_cg', or 'direct', got '{bounds_method}'")
        if bounds_method != "projected_cg":
            raise NotImplementedError("the B200 backend implements bounds_method='projected_cg'")
        mat = fem.material
        if getattr(mat, "pf_model", "AT2") != "AT2" or nodal_H:
            raise NotImplementedError("native Q4 damage supports pf_model='AT2' with Gauss-point H")
        if getattr(mat, "degradation_type", "standard") != "standard":
            raise NotImplementedError("only the standard AT2 degradation is implemented")
        self.fem = fem
        self.material = mat
        self.mesh = fem.mesh
        self.tol = float(tol)
        self.max_iter = int(max_iter)
        self._bounds_method = bounds_method
        self._pf_model = "AT2"
        self._Gc = float(mat.Gc)
        self._l0 = float(mat.l0)
        self._Gc_l0 = self._Gc * self._l0
        self._Gc_over_l0 = self._Gc / self._l0
        self._Gc_l0_e = None
        self._Gc_over_l0_e = None
        if getattr(mat, "gamma_correction", False):
            raise NotImplementedError("gamma_correction is not implemented for structured Q4 grids")
        self.differentiable = False
        self.damage_viscosity = 0.0
        self.damage_dt = None
        self.last_iter = 0
        self.last_converged = True
        self.last_reason = 0
        self.n_solves = 0
        self.check_every = 10  # Jacobi branch (damage_solver.py:3564)
        self._ws = _lib.Workspace(fem.device)

    # -- operator -------------------------------------------------------------
    def _normalize_q4_H(self, H):
        E = self.fem.n_elems
        if H.shape == (E,):
            H = H.unsqueeze(1).expand(E, 4)
        if tuple(H.shape) != (E, 4):
            raise ValueError(f"Native Q4 AT2 damage expects H with shape ({E},) or ({E}, 4), got {tuple(H.shape)}")
        return H.to(torch.float64).contiguous()

    def _Ax_q4(self, d, reaction_density):
        """(Gc l0 K + M(reaction_density)) d (damage_solver.py:1797-1838)."""
        rd = self._normalize_q4_H(reaction_density)
        d = d.to(torch.float64).contiguous()
        y = torch.empty_like(d)
        gl = self._Gc_l0_e
        call("phastb_q4_damage_apply", self.fem.grid, ptr(d), ptr(rd), 1.0, 0.0, None, self._Gc_l0, ptr(gl), ptr(y),
             stream())
        return y

    def _prepare(self, H):
        Hq = self._normalize_q4_H(H)
        n = self.fem.n_nodes
        b = torch.empty(n, dtype=torch.float64, device=Hq.device)
        m_inv = torch.empty_like(b)
        call("phastb_q4_damage_prepare", self.fem.grid, ptr(Hq), self._Gc_over_l0, ptr(self._Gc_over_l0_e),
             self._Gc_l0, ptr(self._Gc_l0_e), ptr(b), ptr(m_inv), stream())
        return b, m_inv

    def compute_residual(self, H_input, d):
        """A d - b of the AT2 system (damage_solver.py:1988-2093, Q4 AT2 branch)."""
        Hq = self._normalize_q4_H(H_input)
        b, _ = self._prepare(Hq)
        y = torch.empty_like(b)
        dd = d.to(torch.float64).contiguous()
        call("phastb_q4_damage_apply", self.fem.grid, ptr(dd), ptr(Hq), 2.0, self._Gc_over_l0,
             ptr(self._Gc_over_l0_e), self._Gc_l0, ptr(self._Gc_l0_e), ptr(y), stream())
        return y - b

    # -- solve ------------------------------------------------------------------
    def solve(self, H_input, d_prev, Gc=None, l0=None, Gc_field=None, pf_dirichlet_mask=None,
              pf_dirichlet_values=None, initial_guess=None):
        """Projected-CG AT2 solve with d in [d_prev, 1] (damage_solver.py:2493-2640, 3528-3775).

        When autograd is on and H_input, d_prev, Gc, l0 or Gc_field requires a
        gradient, the solve is differentiated by the adjoint method on the frozen
        active set (``_Q4DamageAdjoint``); PhAST raises NotImplementedError for
        differentiable Q4 solves (damage_solver.py:2550-2557) and differentiates
        its T3 path the same way (damage_solver.py:483-1154).
        """
        tracked = [t for t in (H_input, d_prev, Gc, l0, Gc_field) if isinstance(t, torch.Tensor) and t.requires_grad]
        if tracked and torch.is_grad_enabled():
            if Gc is not None and Gc_field is not None:
                raise ValueError("Pass either Gc (scalar) or Gc_field (per-element), not both.")
            return _Q4DamageAdjoint.apply(self, H_input, d_prev, Gc, l0, Gc_field, pf_dirichlet_mask,
                                          pf_dirichlet_values, initial_guess)
        return self._solve_forward(H_input, d_prev, Gc, l0, Gc_field, pf_dirichlet_mask, pf_dirichlet_values,
                                   initial_guess)

    def _material(self, Gc=None, l0=None, Gc_field=None):
        """(Gc l0, Gc / l0) scalars and per-element fields for the overrides."""
        Gc_s = self._Gc if Gc is None else float(Gc)
        l0_s = self._l0 if l0 is None else float(l0)
        gcl0_e = gco_e = None
        if Gc_field is not None:
            gf = torch.as_tensor(Gc_field, dtype=torch.float64, device=self.fem.device).detach().reshape(-1)
            if gf.numel() != self.fem.n_elems:
                raise ValueError("Gc_field must have one value per element")
            gcl0_e = (gf * l0_s).contiguous()
            gco_e = (gf / l0_s).contiguous()
        return Gc_s, l0_s, Gc_s * l0_s, Gc_s / l0_s, gcl0_e, gco_e

    def _apply_full(self, H_input, x, Gc=None, l0=None, Gc_field=None):
        """A x of the AT2 system (unmasked) with the given material overrides."""
        _, _, gcl0, gco, gcl0_e, gco_e = self._material(Gc, l0, Gc_field)
        Hq = self._normalize_q4_H(H_input.detach())
        xx = x.detach().to(torch.float64).contiguous()
        y = torch.empty_like(xx)
        call("phastb_q4_damage_apply", self.fem.grid, ptr(xx), ptr(Hq), 2.0, gco, ptr(gco_e), gcl0, ptr(gcl0_e),
             ptr(y), stream())
        return y

    def linear_solve(self, H_input, rhs, Gc=None, l0=None, Gc_field=None, fixed=None, fixed_values=None, x0=None,
                     rtol=1e-11, max_iter=None):
        """Solve the unbounded AT2 system A x = rhs with ``fixed`` rows held at ``fixed_values``.

        The adjoint system of the damage step (A is symmetric); mirrors
        _pcg_solve_adjoint_system (damage_solver.py:423-480).
        """
        _, _, gcl0, gco, gcl0_e, gco_e = self._material(Gc, l0, Gc_field)
        Hq = self._normalize_q4_H(H_input.detach())
        n = self.fem.n_nodes
        r = rhs.detach().to(torch.float64).contiguous()
        fx = None if fixed is None else fixed.to(torch.uint8).contiguous()
        fv = None if fixed_values is None else fixed_values.detach().to(torch.float64).contiguous()
        xi = None if x0 is None else x0.detach().to(torch.float64).contiguous()
        out = torch.empty(n, dtype=torch.float64, device=r.device)
        info = (C.c_int * 2)()
        rinfo = (C.c_double * 2)()
        wp, wn = self._ws.get(_lib.load().phastb_q4_damage_linear_workspace_bytes(n))
        call("phastb_q4_damage_linear_solve", self.fem.grid, ptr(Hq), gco, ptr(gco_e), gcl0, ptr(gcl0_e), ptr(r),
             ptr(fx), ptr(fv), ptr(xi), float(rtol), int(max_iter or max(self.max_iter, 1000)), self.check_every,
             ptr(out), info, rinfo, wp, wn, stream())
        self.last_linear_info = (int(info[0]), int(info[1]), float(rinfo[0]), float(rinfo[1]))
        if info[1] not in (0, 1):
            raise RuntimeError(f"adjoint damage PCG failed (reason {int(info[1])})")
        return out

    def adjoint_grads(self, lam, d, Gc_field=None, l0=None):
        """(dJ/dGc_e (E,), dJ/dH (E, 4)) for the adjoint ``lam`` of the damage solve at ``d``."""
        _, l0_s, *_ = self._material(None, l0, Gc_field)
        E, dev = self.fem.n_elems, d.device
        g_gc = torch.empty(E, dtype=torch.float64, device=dev)
        g_h = torch.empty(E, 4, dtype=torch.float64, device=dev)
        lam = lam.to(torch.float64).contiguous()
        d = d.to(torch.float64).contiguous()
        call("phastb_q4_damage_adjoint_grads", self.fem.grid, ptr(lam), ptr(d), l0_s, ptr(g_gc), ptr(g_h), None, None,
             stream())
        return g_gc, g_h

    def _solve_forward(self, H_input, d_prev, Gc=None, l0=None, Gc_field=None, pf_dirichlet_mask=None,
                       pf_dirichlet_values=None, initial_guess=None):
        self.n_solves += 1
        if Gc is not None and Gc_field is not None:
            raise ValueError("Pass either Gc (scalar) or Gc_field (per-element), not both.")
        _, _, gcl0, gco, gcl0_e, gco_e = self._material(Gc, l0, Gc_field)
        orig_dtype = d_prev.dtype
        if not torch.isfinite(d_prev).all():
            self.last_iter = 0
            self.last_converged = False
            return d_prev.clone()
        Hq = self._normalize_q4_H(H_input.detach())
        dp = d_prev.detach().to(torch.float64).contiguous()
        di = None if initial_guess is None else initial_guess.detach().to(torch.float64).contiguous()
        fixed = vals = None
        if pf_dirichlet_mask is not None:
            m = pf_dirichlet_mask.to(device=dp.device, dtype=torch.bool)
            if bool(m.any()):
                if pf_dirichlet_values is None:
                    raise ValueError("pf_dirichlet_values must be supplied with mask")
                fixed = m.to(torch.uint8).contiguous()
                vals = pf_dirichlet_values.to(device=dp.device, dtype=torch.float64).contiguous()
        n = self.fem.n_nodes
        out = torch.empty(n, dtype=torch.float64, device=dp.device)
        info = (C.c_int * 2)()
        wp, wn = self._ws.get(_lib.load().phastb_q4_damage_solve_workspace_bytes(n))
        st = raw("phastb_q4_damage_solve", self.fem.grid, ptr(Hq), gco, ptr(gco_e), gcl0, ptr(gcl0_e), ptr(dp),
                 ptr(di), ptr(fixed), ptr(vals), self.tol, self.max_iter, self.check_every, ptr(out), info, wp, wn,
                 stream())
        _lib.check(st, "phastb_q4_damage_solve")
        self.last_iter = int(info[0])
        self.last_reason = int(info[1])
        self.last_converged = info[1] == 0
        if info[1] == 3:
            print(f"  [PhaseFieldDamageSolver diverged at iter {self.last_iter}]", flush=True)
        return out.to(orig_dtype)


def classify_active_set(d_new, d_prev, fixed=None, upper_bound=1.0, atol=1e-12):
    """(lower, upper, fixed, interior) masks after projection onto [d_prev, 1].

    classify_damage_active_set, damage_solver.py:70-106: the upper bound and
    pinned nodes take precedence over the lower (irreversibility) bound.
    """
    upper = d_new >= (upper_bound - atol)
    fx = torch.zeros_like(upper) if fixed is None else fixed.to(device=d_new.device, dtype=torch.bool)
    lower = (d_new <= d_prev + atol) & ~upper & ~fx
    upper = upper & ~fx
    interior = ~(lower | upper | fx)
    return lower, upper, fx, interior


class _Q4DamageAdjoint(torch.autograd.Function):
    """Implicit differentiation of the bound-projected AT2 solve on its frozen active set.

    Forward: the device PPCG solve.  Backward: with the active set (bound-active
    and pinned nodes) frozen, the solution satisfies A_FF d_F = b_F - A_FA d_A,
    so for an upstream gradient g the adjoint lam solves A_FF lam_F = g_F
    (lam_A = 0) -- one Jacobi PCG on the device -- and

        dL/dGc_e     = -(l0 lam^T K_e d + lam^T M_e d / l0)
        dL/dl0       = -sum_e (Gc_e lam^T K_e d - Gc_e / l0^2 lam^T M_e d)
        dL/dH_{e,q}  = 2 w lam_q (1 - d_q)
        dL/dd_prev   = g_i - (A lam)_i on the nodes i held at their lower bound

    (the AT2 formulas of _AdjointDamageSolveScalar/_AdjointDamageSolveField,
    damage_solver.py:483-1037, with the Q4 Gauss rule; where PhAST passes g
    through to d_prev unchanged, the coupling of a held node to its free
    neighbours, -(A lam)_i, is kept here, which is the exact derivative).
    """

    @staticmethod
    def forward(ctx, solver, H_input, d_prev, Gc, l0, Gc_field, mask, values, initial_guess):
        d = solver._solve_forward(H_input, d_prev, Gc, l0, Gc_field, mask, values, initial_guess)
        ctx.solver = solver
        ctx.h_shape = tuple(H_input.shape)
        ctx.gc_scalar = isinstance(Gc, torch.Tensor)
        ctx.l0_tensor = isinstance(l0, torch.Tensor)
        ctx.has_field = Gc_field is not None
        ctx.Gc = None if Gc is None else float(Gc)
        ctx.l0 = None if l0 is None else float(l0)
        m = None if mask is None else mask.to(device=d.device, dtype=torch.bool)
        gf = None if Gc_field is None else torch.as_tensor(Gc_field, device=d.device).detach().to(torch.float64)
        ctx.save_for_backward(H_input.detach(), d_prev.detach(), d.detach(),
                              m if m is not None else torch.empty(0, dtype=torch.bool, device=d.device),
                              gf if gf is not None else torch.empty(0, dtype=torch.float64, device=d.device))
        return d

    @staticmethod
    def backward(ctx, grad_out):
        solver = ctx.solver
        H, d_prev, d, m, gf = ctx.saved_tensors
        mask = m if m.numel() else None
        gfield = gf if gf.numel() else None
        Gc_s, l0_s, *_ = solver._material(ctx.Gc, ctx.l0, gfield)
        g = grad_out.detach().to(torch.float64)
        lower, upper, fx, interior = classify_active_set(d.to(torch.float64), d_prev.to(torch.float64), mask)
        frozen = ~interior
        lam = solver.linear_solve(H, g * interior, Gc=ctx.Gc, l0=ctx.l0, Gc_field=gfield, fixed=frozen,
                                  fixed_values=None, rtol=1e-11)
        E = solver.fem.n_elems
        dev = d.device
        g_gc = torch.empty(E, dtype=torch.float64, device=dev)
        g_h = torch.empty(E, 4, dtype=torch.float64, device=dev)
        lkd = torch.empty(E, dtype=torch.float64, device=dev)
        lmd = torch.empty(E, dtype=torch.float64, device=dev)
        dd = d.to(torch.float64).contiguous()
        call("phastb_q4_damage_adjoint_grads", solver.fem.grid, ptr(lam), ptr(dd), l0_s, ptr(g_gc), ptr(g_h), ptr(lkd),
             ptr(lmd), stream())
        grad_H = g_h if ctx.h_shape == (E, 4) else g_h.sum(1)
        grad_H = grad_H.to(H.dtype).reshape(ctx.h_shape)
        grad_dprev = torch.zeros_like(g)
        if bool(lower.any()):
            Alam = solver._apply_full(H, lam, ctx.Gc, ctx.l0, gfield)
            grad_dprev = (g - Alam) * lower
        grad_dprev = grad_dprev.to(d_prev.dtype)
        gc_e = gfield if gfield is not None else torch.full((E,), Gc_s, dtype=torch.float64, device=dev)
        grad_l0 = -(gc_e * lkd).sum() + (gc_e / l0_s ** 2 * lmd).sum()
        grad_Gc = g_gc.sum() if ctx.gc_scalar else None
        grad_field = g_gc if ctx.has_field else None
        return (None, grad_H, grad_dprev, grad_Gc, grad_l0 if ctx.l0_tensor else None, grad_field, None, None, None)

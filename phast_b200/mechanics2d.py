"""2D mechanics solvers behind PhAST's ``ExplicitDynamics`` / ``QuasiStaticSolver``.

``ExplicitDynamics.step`` is one fused kernel (predictor, internal force of the
predicted field, corrector, Dirichlet zeroing) -- mechanics_solver.py:86-239.
``QuasiStaticSolver.solve`` is Newton with matrix-free CG on K(d) and the
residual line search of ``_accept_newton_step`` -- mechanics_solver.py:1597-2043;
the Newton loop, the CG iterations and the line search all run in
``libphastb.so``.
"""
from __future__ import annotations

import ctypes as C
import math

import torch

from . import _lib
from ._lib import call, ptr, raw, stream
from .fem2d import _dtype_code, stress_split_of


class ExplicitDynamics:
    """Central difference with lumped mass (mechanics_solver.py:86-239)."""

    def __init__(self, fem, dt=None, dt_safety=1.0, differentiable=False, damping_ratio_max=0.0):
        if differentiable:
            raise NotImplementedError("use phast_b200.adjoint for gradients through the explicit loop")
        if damping_ratio_max and damping_ratio_max > 0.0:
            raise NotImplementedError("Kelvin-Voigt damping is not implemented by the B200 backend")
        self.fem = fem
        self.differentiable = False
        self.damping_ratio_max = 0.0
        self.dt_cfl = fem.dt_cfl * dt_safety
        self.dt = self.dt_cfl if dt is None else dt
        self.last_iter = 1
        self._minv = {}

    def _m_inv(self, dtype):
        if dtype not in self._minv:
            mi = 1.0 / (self.fem.material.rho * self.fem.M_scalar + 1e-30)
            self._minv[dtype] = mi.to(dtype).contiguous()
        return self._minv[dtype]

    def step_into(self, u, v, a, d, f_ext, bc_mask, bc_vals, u_out, v_out, a_out, H_in=None, H_out=None):
        """One step written into caller buffers; optionally fuses H_out = max(H_in, psi+(u_new))."""
        fem = self.fem
        dt = u.dtype
        # converted copies are held in locals until the launch is enqueued: a temporary whose
        # last reference dies inside the argument list goes back to the caching allocator,
        # which may hand its block to the next conversion before the kernel reads it
        mask = (bc_mask if bc_mask.dtype == torch.uint8 else bc_mask.to(torch.uint8)).contiguous()
        d_k = d.to(dt).contiguous()
        f_k = f_ext.to(dt).contiguous()
        vals_k = bc_vals.to(dt).contiguous()
        call("phastb_q4_explicit_step", fem.grid, fem.mat(dt), _dtype_code(u), float(self.dt), ptr(self._m_inv(dt)),
             ptr(u), ptr(v), ptr(a), ptr(d_k), ptr(f_k), ptr(mask), ptr(vals_k), ptr(u_out), ptr(v_out), ptr(a_out),
             ptr(H_in), ptr(H_out), stream())

    def step(self, u, v, a, d, f_ext, bc_mask, bc_vals, rigid_connectors=None):
        """Predictor + corrector; returns new (u, v, a) (mechanics_solver.py:204-239)."""
        if rigid_connectors:
            raise NotImplementedError("rigid connectors are not implemented by the B200 backend")
        self.last_iter = 1
        u_n, v_n, a_n = torch.empty_like(u), torch.empty_like(v), torch.empty_like(a)
        self.step_into(u.contiguous(), v.contiguous(), a.contiguous(), d, f_ext, bc_mask, bc_vals, u_n, v_n, a_n)
        return u_n, v_n, a_n

    def predictor(self, u, v, a, bc_mask, bc_vals):
        u_new = u + self.dt * v + 0.5 * self.dt * self.dt * a
        return torch.where(bc_mask, bc_vals, u_new)

    def rollout(self, u, v, a, d, f_ext, bc_mask, bc_vals, n_steps, checkpoint_every=10):
        """``n_steps`` central-difference steps at fixed damage; returns the final (u, v, a).

        Differentiable (FP64) with respect to u, v, a, f_ext and d when any of
        them requires a gradient: the backward pass runs the hand-written reverse
        step (phastb_q4_explicit_adjoint_step) and recomputes each segment of
        ``checkpoint_every`` steps from its stored start state, so memory grows
        with n_steps / checkpoint_every, not with n_steps (the chunked
        recomputation of ChunkedExplicitDynamicsAutograd, mechanics_solver.py:4057-4137).
        """
        n_steps, k = int(n_steps), int(checkpoint_every)
        if n_steps < 0 or k < 1:
            raise ValueError("n_steps must be >= 0 and checkpoint_every >= 1")
        tracked = any(isinstance(t, torch.Tensor) and t.requires_grad for t in (u, v, a, f_ext, d))
        if tracked and torch.is_grad_enabled():
            return _ExplicitRollout.apply(self, u, v, a, d, f_ext, bc_mask, bc_vals, n_steps, k)
        with torch.no_grad():
            return self._run(u.detach(), v.detach(), a.detach(), d.detach(), f_ext.detach(), bc_mask, bc_vals,
                             n_steps)[0]

    def _run(self, u, v, a, d, f_ext, bc_mask, bc_vals, n_steps, keep_every=0):
        """Forward steps; with keep_every > 0 also the start states of the segments."""
        u, v, a = u.contiguous().clone(), v.contiguous().clone(), a.contiguous().clone()
        un, vn, an = torch.empty_like(u), torch.empty_like(v), torch.empty_like(a)
        dd, ff = d.contiguous(), f_ext.contiguous()
        kept = []
        for s in range(n_steps):
            if keep_every and s % keep_every == 0:
                kept.append((u.clone(), v.clone(), a.clone()))
            self.step_into(u, v, a, dd, ff, bc_mask, bc_vals, un, vn, an)
            u, un = un, u
            v, vn = vn, v
            a, an = an, a
        return (u, v, a), kept


class QuasiStaticSolver:
    """Newton-Raphson with matrix-free CG (mechanics_solver.py:816-2043).

    The CG operator is the consistent tangent at the Newton iterate for the spectral, Amor
    and star-convex splits (the reference's autograd JVP, mechanics_solver.py:1705-1733) and
    the degraded stiffness for the linear ones, both one kernel per CG step.
    """

    def __init__(self, fem, tol=1e-6, max_iter=50, cg_tol=1e-8, cg_max_iter=5000, backend="auto",
                 sparse_dof_threshold=200000, inner_solver=None, consistent_tangent=None, line_search=True,
                 line_search_max_steps=8, line_search_min_alpha=1e-4, line_search_c=1e-4, tol_rel=None,
                 plasticity_operator=None, cohesive_operator=None):
        if plasticity_operator is not None or cohesive_operator is not None:
            raise NotImplementedError("plasticity / cohesive mechanics are not implemented by the B200 backend")
        if tol_rel is not None:
            raise NotImplementedError("relative Newton tolerance is not implemented by the B200 backend")
        split = stress_split_of(fem.material)
        if consistent_tangent is False and split in ("spectral", "amor", "star_convex"):
            raise NotImplementedError("the secant (frozen-state) linearisation is not implemented by the B200 "
                                      "backend; the consistent tangent is used")
        self.fem = fem
        self.tol = float(tol)
        self.max_iter = int(max_iter)
        self.cg_tol = float(cg_tol)
        self.cg_max_iter = int(cg_max_iter)
        self.backend = backend
        self.line_search = bool(line_search)
        self.line_search_max_steps = int(line_search_max_steps)
        self.line_search_min_alpha = float(line_search_min_alpha)
        self.line_search_c = float(line_search_c)
        self.last_iter = 0
        self.last_cg_iters = 0
        self.last_backend = "cg"
        self._ws = _lib.Workspace(fem.device)

    def _newton(self, d, f_ext, mask_u8, bc_vals, u, tol, cg_tol, max_iter, line_search, cg_max_iter=None):
        """One device Newton-CG solve into ``u`` (FP64, contiguous); returns (status, info)."""
        fem = self.fem
        t3 = getattr(fem, "t3", None)
        n = fem.n_nodes
        info = (C.c_int * 3)()
        lib = _lib.load()
        if t3 is not None:
            name, geo, wb = "phastb_t3_qs_solve", t3, lib.phastb_t3_qs_workspace_bytes(n)
        else:
            name, geo, wb = "phastb_q4_qs_solve", fem.grid, lib.phastb_q4_qs_workspace_bytes(n)
        wp, wn = self._ws.get(wb)
        st = raw(name, geo, fem.mat(torch.float64), ptr(d), ptr(f_ext), ptr(mask_u8), ptr(bc_vals), ptr(u), float(tol),
                 float(cg_tol), int(cg_max_iter or self.cg_max_iter), int(max_iter), int(line_search), self.line_search_max_steps,
                 self.line_search_min_alpha, self.line_search_c, info, wp, wn, stream())
        if st not in (_lib.OK, _lib.NONCONVERGED, _lib.NONFINITE, _lib.BREAKDOWN):
            _lib.check(st, name)
        return st, info

    def solve(self, d, f_ext, bc_mask, bc_vals, u_init=None, rigid_connectors=None):
        """Equilibrium f_int(u, d) = f_ext; returns (u, converged, n_iter) (mechanics_solver.py:1597-1783)."""
        if rigid_connectors:
            raise NotImplementedError("rigid connectors are not implemented by the B200 backend")
        fem = self.fem
        n = fem.n_nodes
        u = (torch.zeros(n, 2, dtype=torch.float64, device=fem.device) if u_init is None
             else u_init.to(torch.float64).clone().contiguous())
        dd = d.to(torch.float64).contiguous()
        fe = None if f_ext is None else f_ext.to(torch.float64).contiguous()
        mask = bc_mask.to(torch.uint8).contiguous()
        vals = bc_vals.to(torch.float64).contiguous()
        _, info = self._newton(dd, fe, mask, vals, u, self.tol, self.cg_tol, self.max_iter, self.line_search)
        self.last_iter = int(info[0])
        self.last_cg_iters = int(info[2])
        converged = bool(info[1])
        return u.to(d.dtype if d.dtype.is_floating_point else torch.float64), converged, int(info[0])

    def solve_stiffness(self, d, rhs, bc_mask, rtol=1e-12, max_refine=30):
        """z with K(d)_ff z_f = rhs_f and z = 0 on prescribed dofs, to a residual of ``rtol``
        relative to |rhs_f| (the Newton entry with zero prescribed values and no line search:
        one CG solve plus refinement steps).  The adjoint of the equilibrium solve."""
        mask = bc_mask.to(device=self.fem.device, dtype=torch.uint8).contiguous()
        r = rhs.to(torch.float64) * (mask == 0).to(torch.float64)
        r = r.contiguous()
        z = torch.zeros_like(r)
        nrm = float(torch.linalg.vector_norm(r))
        if nrm == 0.0:
            return z
        dd = d.to(torch.float64).contiguous()
        # The system is linear: solve for the unit-norm right-hand side and scale back, so the
        # CG thresholds and curvature guards see numbers of order one whatever the size of rhs
        # (a reaction gradient is small); the inner CG's threshold sits below the target, and one
        # long CG per refinement keeps its Krylov space (a restarted short CG stalls on large
        # cracked meshes).
        r = (r / nrm).contiguous()
        st, info = self._newton(dd, r, mask, torch.zeros_like(r), z, rtol, min(1e-10, 0.5 * rtol), max_refine, False,
                                cg_max_iter=max(self.cg_max_iter, 200000))
        if st != _lib.OK or not info[1]:
            raise RuntimeError(f"stiffness solve did not converge (status {st}, {int(info[0])} refinements)")
        return z * nrm


class _ExplicitRollout(torch.autograd.Function):
    """Reverse-mode differentiation of n explicit steps with checkpoint-and-recompute."""

    @staticmethod
    def forward(ctx, dyn, u, v, a, d, f_ext, bc_mask, bc_vals, n_steps, k):
        if u.dtype != torch.float64:
            raise NotImplementedError("the differentiable explicit rollout runs in FP64")
        with torch.no_grad():
            (uN, vN, aN), kept = dyn._run(u.detach(), v.detach(), a.detach(), d.detach().to(u.dtype),
                                           f_ext.detach().to(u.dtype), bc_mask, bc_vals, n_steps, keep_every=k)
        ctx.dyn, ctx.n, ctx.k, ctx.kept = dyn, n_steps, k, kept
        ctx.save_for_backward(d.detach().to(u.dtype).contiguous(), f_ext.detach().to(u.dtype).contiguous(),
                              bc_mask, bc_vals)
        ctx.d_dtype, ctx.f_dtype = d.dtype, f_ext.dtype
        return uN, vN, aN

    @staticmethod
    def backward(ctx, gu, gv, ga):
        dyn, n, k = ctx.dyn, ctx.n, ctx.k
        d, f_ext, bc_mask, bc_vals = ctx.saved_tensors
        fem = dyn.fem
        mask = (bc_mask if bc_mask.dtype == torch.uint8 else bc_mask.to(torch.uint8)).contiguous()
        z = lambda t: torch.zeros_like(f_ext) if t is None else t.detach().contiguous().to(torch.float64)
        ub, vb, ab = z(gu), z(gv), z(ga)
        fb = torch.zeros_like(f_ext)
        db = torch.zeros(fem.n_nodes, dtype=torch.float64, device=f_ext.device)
        nb = [torch.empty_like(ub) for _ in range(3)]
        scratch = torch.empty(4 * fem.n_nodes, dtype=torch.float64, device=f_ext.device)
        mat = fem.mat(torch.float64)
        minv = dyn._m_inv(torch.float64)
        n_seg = len(ctx.kept)
        for seg in range(n_seg - 1, -1, -1):
            s0, s1 = seg * k, min((seg + 1) * k, n)
            # recompute the segment's states u_{s0+1} .. u_{s1} (the u' of each step)
            u, v, a = (t.clone() for t in ctx.kept[seg])
            outs = []
            with torch.no_grad():
                for _ in range(s1 - s0):
                    un, vn, an = torch.empty_like(u), torch.empty_like(v), torch.empty_like(a)
                    dyn.step_into(u, v, a, d, f_ext, bc_mask, bc_vals, un, vn, an)
                    outs.append(un)
                    u, v, a = un, vn, an
            for j in range(s1 - s0 - 1, -1, -1):
                call("phastb_q4_explicit_adjoint_step", fem.grid, mat, float(dyn.dt), ptr(minv), ptr(d), ptr(mask),
                     ptr(outs[j]), ptr(ub), ptr(vb), ptr(ab), ptr(nb[0]), ptr(nb[1]), ptr(nb[2]), ptr(fb), ptr(db),
                     ptr(scratch), stream())
                ub, nb[0] = nb[0], ub
                vb, nb[1] = nb[1], vb
                ab, nb[2] = nb[2], ab
        ctx.kept = None
        return (None, ub, vb, ab, db.to(ctx.d_dtype), fb.to(ctx.f_dtype), None, None, None, None)

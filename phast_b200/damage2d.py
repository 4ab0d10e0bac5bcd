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
    """GPU projected-CG AT2 damage solver for structured Q4 grids."""

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

    def compute_residual(self, H, d):
        """A d - b of the AT2 system (damage_solver.py:1988-2093, Q4 AT2 branch)."""
        Hq = self._normalize_q4_H(H)
        b, _ = self._prepare(Hq)
        y = torch.empty_like(b)
        dd = d.to(torch.float64).contiguous()
        call("phastb_q4_damage_apply", self.fem.grid, ptr(dd), ptr(Hq), 2.0, self._Gc_over_l0,
             ptr(self._Gc_over_l0_e), self._Gc_l0, ptr(self._Gc_l0_e), ptr(y), stream())
        return y - b

    # -- solve ------------------------------------------------------------------
    def solve(self, H_input, d_prev, Gc=None, l0=None, Gc_field=None, pf_dirichlet_mask=None,
              pf_dirichlet_values=None, initial_guess=None):
        """Projected-CG AT2 solve with d in [d_prev, 1] (damage_solver.py:2493-2640, 3528-3775)."""
        self.n_solves += 1
        for t in (Gc, l0, Gc_field):
            if isinstance(t, torch.Tensor) and t.requires_grad:
                raise NotImplementedError(
                    "Differentiable native Q4 damage solves are not implemented yet. Use forward Q4 AT2 solves "
                    "without gradient-tracked material overrides, or convert Q4 cells to T3 for adjoint damage "
                    "workflows.")
        if Gc is not None and Gc_field is not None:
            raise ValueError("Pass either Gc (scalar) or Gc_field (per-element), not both.")
        Gc_s = self._Gc if Gc is None else float(Gc)
        l0_s = self._l0 if l0 is None else float(l0)
        gcl0, gco = Gc_s * l0_s, Gc_s / l0_s
        gcl0_e = gco_e = None
        if Gc_field is not None:
            gf = torch.as_tensor(Gc_field, dtype=torch.float64, device=self.fem.device).reshape(-1)
            if gf.numel() != self.fem.n_elems:
                raise ValueError("Gc_field must have one value per element")
            gcl0_e = (gf * l0_s).contiguous()
            gco_e = (gf / l0_s).contiguous()
        orig_dtype = d_prev.dtype
        if not torch.isfinite(d_prev).all():
            self.last_iter = 0
            self.last_converged = False
            return d_prev.clone()
        Hq = self._normalize_q4_H(H_input)
        dp = d_prev.to(torch.float64).contiguous()
        di = None if initial_guess is None else initial_guess.to(torch.float64).contiguous()
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

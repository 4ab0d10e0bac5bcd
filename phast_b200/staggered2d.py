"""2D staggered driver behind PhAST's ``StaggeredSolver`` interface.

Mirrors ``phast.solvers.staggered_solver.StaggeredSolver.step_full``
(src/phast/solvers/staggered_solver.py:1103-1344) for the two solver types of
the hot path: ``'explicit'`` (one fused central-difference + history kernel,
then the damage solve every ``damage_every`` steps, always in the first five)
and ``'quasi_static'`` (stagger loop of Newton-CG mechanics, history, damage
solve, relative-L2 convergence on u and d with ``min_stag = 2``).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import torch

from . import _lib
from ._lib import call, ptr, stream
from .damage2d import PhaseFieldDamageSolver
from .fem2d import FEMOperators
from .mechanics2d import ExplicitDynamics, QuasiStaticSolver


@dataclass
class SolverConfig:
    """``phast.solvers.staggered_solver.SolverConfig`` (staggered_solver.py:45-162): the same
    fields in the same order with the same defaults, and its rule that the quasi-static solver
    types default to the Jacobi preconditioner.  ``dtype`` (last, this backend's own) selects
    FP32 state for the explicit step.  Options the GPU path does not run (generalized-alpha,
    adaptive time steps, mesh refinement or stagger tolerance, smooth-max history updates, the
    fresh-damage corrector) are refused by ``StaggeredSolver`` with ``NotImplementedError``."""
    solver_type: str = "explicit"
    time_integrator: str = "central_difference"
    rho_inf: float = 0.5
    dt: Optional[float] = None
    dt_safety: float = 1.0
    num_steps: int = 200
    damage_tol: float = 1e-5
    damage_max_iter: int = 5000
    static_tol: float = 1e-8
    static_max_iter: int = 5000
    H_cap: Optional[float] = None
    softmax_H_beta: Optional[float] = None
    H_update_method: str = "hard_max"
    H_update_scale: Optional[float] = None
    stagger_tol: float = 1e-6
    max_stagger: int = 500
    stagger_criterion: str = "relative"
    stagger_norm: str = "l2"
    use_multigrid: bool = True
    bounds_method: str = "post_clamp"
    preconditioner: Optional[str] = None
    adaptive_refine: bool = False
    refine_every: int = 10
    refine_d_threshold: float = 0.5
    refine_grad_d_threshold: float = 0.3
    anderson_depth: int = 0
    adaptive_stagger_tol: bool = False
    differentiable: bool = False
    fail_on_mechanics_nonconvergence: bool = True
    fail_on_stagger_nonconvergence: bool = True
    damage_viscosity: float = 0.0
    damping_ratio_max: float = 0.0
    enable_damage: bool = True
    backend: str = "auto"
    newton_line_search: bool = True
    line_search_max_steps: int = 8
    line_search_min_alpha: float = 1e-4
    line_search_c: float = 1e-4
    adaptive_dt: bool = False
    adaptive_dt_d_threshold: float = 0.01
    adaptive_dt_min_factor: float = 0.1
    adaptive_dt_grow_rate: float = 1.1
    dt_growth_threshold: float = 0.001
    dt_cutback_threshold: float = 0.01
    dt_floor: float = 1e-12
    damage_every: int = 3
    fresh_d_in_corrector: bool = False
    dump_every: int = 10
    h5_every: int = 1
    viz_format: str = "vtu"
    print_every: int = 10
    dtype: torch.dtype = torch.float64

    def __post_init__(self):
        if self.preconditioner is None and self.solver_type in ("static", "quasi_static", "quasi_static_legacy",
                                                                "lbfgs", "monolithic"):
            self.preconditioner = "jacobi"


class BoundaryConditions:
    """Dirichlet and phase-field Dirichlet data (physics/boundary_conditions.py:325-620)."""

    def __init__(self, n_nodes, device=None, dtype=torch.float64):
        self.n_nodes = int(n_nodes)
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.dtype = dtype
        self.bcs = []
        self.pf_dirichlet_bcs = []
        self.load_factor = 1.0

    def add(self, node_indices, component, value):
        self.bcs.append((torch.as_tensor(node_indices, dtype=torch.long), int(component), float(value)))
        return self

    def fix(self, node_indices, component):
        return self.add(node_indices, component, 0.0)

    def add_pf_dirichlet(self, node_indices, value=1.0):
        idx = torch.as_tensor(node_indices, dtype=torch.long).flatten().unique()
        self.pf_dirichlet_bcs.append((idx, float(value)))
        return self

    def get_masks_and_values(self):
        mask = torch.zeros(self.n_nodes, 2, dtype=torch.bool)
        vals = torch.zeros(self.n_nodes, 2, dtype=self.dtype)
        for idx, c, v in self.bcs:
            mask[idx, c] = True
            vals[idx, c] = v * self.load_factor
        return mask.to(self.device), vals.to(self.device)

    def get_pf_dirichlet_mask_values(self):
        mask = torch.zeros(self.n_nodes, dtype=torch.bool)
        vals = torch.zeros(self.n_nodes, dtype=self.dtype)
        for idx, v in self.pf_dirichlet_bcs:
            mask[idx] = True
            vals[idx] = v
        return mask.to(self.device), vals.to(self.device)


class AndersonAccelerator:
    """Type II Anderson mixing of the damage fixed point (_AndersonAccelerator,
    staggered_solver.py:165-255): the last ``m + 1`` pairs in a device ring, one C-ABI call per
    staggered pass (``phastb_anderson_step``)."""

    def __init__(self, n, m=5, device="cuda", reg=1e-10):
        self.n, self.m, self.reg = int(n), int(m), float(reg)
        self.hist = torch.empty(2 * (self.m + 1) * self.n, dtype=torch.float64, device=device)
        self._ws = _lib.Workspace(torch.device(device))
        self.count = self.head = 0
        self.used = 0

    def reset(self):
        """Clear the history (each new load step)."""
        self.count = self.head = 0

    def step(self, d_in, d_out, d_prev_step=None):
        """The next iterate: the mix clamped to [d_prev_step, 1], or ``d_out`` when there is no
        history, the least-squares system is singular or the mix fails the residual safeguard."""
        mix = torch.empty_like(d_out)
        used = (C.c_int * 1)()
        wp, wn = self._ws.get(_lib.load().phastb_anderson_workspace_bytes(self.m))
        call("phastb_anderson_step", self.n, self.m, self.count, self.head, ptr(self.hist), ptr(d_in.contiguous()),
             ptr(d_out.contiguous()), ptr(None if d_prev_step is None else d_prev_step.contiguous()), self.reg,
             ptr(mix), used, wp, wn, stream())
        self.head = (self.head + 1) % (self.m + 1)
        self.count = min(self.count + 1, self.m + 1)
        self.used += int(used[0])
        return mix


class StaggeredSolver:
    """GPU staggered phase-field step (staggered_solver.py:269-1344)."""

    def __init__(self, mesh, material, bcs, config=None, ctx=None):
        self.config = config or SolverConfig()
        cfg = self.config
        if cfg.damage_viscosity or cfg.H_cap is not None or cfg.H_update_method != "hard_max":
            raise NotImplementedError("damage viscosity and non-hard-max H updates are not implemented by the B200 "
                                      "backend")
        if cfg.anderson_depth and not 1 <= int(cfg.anderson_depth) <= 6:
            raise NotImplementedError("the B200 backend runs Anderson mixing of depth 1 to 6")
        if cfg.stagger_criterion != "relative" or cfg.stagger_norm != "l2":
            raise NotImplementedError("only the relative-L2 stagger criterion is implemented")
        if cfg.softmax_H_beta is not None:
            raise NotImplementedError("the smooth-max history update (softmax_H_beta) is not implemented by the B200 "
                                      "backend")
        if cfg.solver_type == "explicit" and cfg.time_integrator not in ("central_difference", "verlet", "newmark"):
            raise NotImplementedError(f"time_integrator {cfg.time_integrator!r}: the B200 backend runs the central "
                                      "difference step")
        for name in ("adaptive_refine", "adaptive_stagger_tol", "adaptive_dt", "fresh_d_in_corrector"):
            if getattr(cfg, name):
                raise NotImplementedError(f"{name}=True is not implemented by the B200 backend")
        if getattr(material, "plasticity_model", "none") != "none":
            raise NotImplementedError("plasticity coupling is not implemented by the B200 backend")
        if getattr(material, "driving_force", "strain_energy") != "strain_energy":
            raise NotImplementedError("only the strain-energy driving force is implemented")
        if (getattr(material, "sigma_ts", None) or 0.0) > 0.0:
            raise NotImplementedError("the sigma_ts nucleation scaling of the driving force is not implemented by the "
                                      "B200 backend")
        self.mesh, self.material, self.bcs = mesh, material, bcs
        self.fem = FEMOperators(mesh, material)
        fem = self.fem
        self.device = fem.device
        self.dtype = cfg.dtype if cfg.solver_type == "explicit" else torch.float64
        self.damage_solver = PhaseFieldDamageSolver(fem, tol=cfg.damage_tol, max_iter=cfg.damage_max_iter,
                                                    use_multigrid=cfg.use_multigrid,
                                                    bounds_method=cfg.bounds_method, preconditioner=cfg.preconditioner)
        if cfg.solver_type == "explicit":
            self.mechanics = ExplicitDynamics(fem, dt=cfg.dt, dt_safety=cfg.dt_safety,
                                              damping_ratio_max=cfg.damping_ratio_max)
            self.dt = self.mechanics.dt
        elif cfg.solver_type == "quasi_static":
            self.mechanics = QuasiStaticSolver(fem, tol=cfg.static_tol, max_iter=cfg.static_max_iter,
                                               backend=cfg.backend, line_search=cfg.newton_line_search,
                                               line_search_max_steps=cfg.line_search_max_steps,
                                               line_search_min_alpha=cfg.line_search_min_alpha,
                                               line_search_c=cfg.line_search_c)
            self.dt = None
        else:
            raise NotImplementedError(f"solver_type {cfg.solver_type!r} is not implemented by the B200 backend")
        N, E = fem.n_nodes, fem.n_elems
        z = lambda *s: torch.zeros(*s, dtype=self.dtype, device=self.device)
        # history per Gauss point: four per Q4 element, one per T3 element
        hq = (E,) if getattr(fem, "t3", None) is not None else (E, 4)
        self.u, self.v, self.a = z(N, 2), z(N, 2), z(N, 2)
        self.d = torch.zeros(N, dtype=torch.float64, device=self.device)
        self.H_elem = z(*hq)
        self.f_ext = z(N, 2)
        self._nxt = [z(N, 2), z(N, 2), z(N, 2), z(*hq)]
        self._step_count = 0
        self._explicit_step_count = 0
        self._last_stagger_iter = 0
        # when a list, every quasi-static staggered pass appends its iterate (u, d, H) to it
        self.stagger_trace = None

    # -- pieces ------------------------------------------------------------------
    def _pf(self):
        if getattr(self.bcs, "pf_dirichlet_bcs", None):
            return self.bcs.get_pf_dirichlet_mask_values()
        return None, None

    def _apply_pf_dirichlet(self):
        m, v = self._pf()
        if m is not None:
            self.d = torch.where(m, v.to(self.d.dtype), self.d)

    def step_mechanics(self):
        bc_mask, bc_vals = self.bcs.get_masks_and_values()
        if self.config.solver_type == "explicit":
            self.u, self.v, self.a = self.mechanics.step(self.u, self.v, self.a, self.d, self.f_ext, bc_mask, bc_vals)
        else:
            u_new, conv, nit = self.mechanics.solve(self.d, self.f_ext, bc_mask, bc_vals, u_init=self.u)
            if not conv and self.config.fail_on_mechanics_nonconvergence:
                raise RuntimeError(f"Quasi-static mechanics solve did not converge after {nit} Newton iterations.")
            self.u = u_new

    def step_compute_driving_force(self, strain=None):
        H_new = torch.empty_like(self.H_elem)
        self.fem.psi_history(self.u.contiguous(), self.H_elem.contiguous(), H_new)
        self.H_elem = H_new
        return H_new

    def set_damage(self, d_new):
        """Replace the damage field with a copy of ``d_new`` (staggered_solver.py:1409-1411); the
        kernels read it through raw pointers, so its shape, dtype and device are checked."""
        if not isinstance(d_new, torch.Tensor) or tuple(d_new.shape) != tuple(self.d.shape):
            raise ValueError(f"d_new must be a tensor of shape {tuple(self.d.shape)}")
        if d_new.device != self.d.device:
            raise ValueError(f"d_new must be on {self.d.device}")
        self.d = d_new.to(self.d.dtype).clone().contiguous()

    def step_solve_damage(self, d_prev_step=None):
        pf_mask, pf_vals = self._pf()
        d_prev_arg = d_prev_step if d_prev_step is not None else self.d
        init = self.d if d_prev_step is not None else None
        # a per-element Gc field set as diff_Gc_field (staggered_solver.py:904-936)
        gc_field = getattr(self, "diff_Gc_field", None)
        self.d = self.damage_solver.solve(self.H_elem, d_prev_arg, Gc_field=gc_field, pf_dirichlet_mask=pf_mask,
                                          pf_dirichlet_values=pf_vals, initial_guess=init)
        self._apply_pf_dirichlet()

    # -- the staggered step ----------------------------------------------------------
    def step_full(self):
        cfg = self.config
        if cfg.solver_type == "explicit":
            # fused: mechanics step + history update of the new displacement
            bc_mask, bc_vals = self.bcs.get_masks_and_values()
            u_n, v_n, a_n, H_n = self._nxt
            self.mechanics.step_into(self.u, self.v, self.a, self.d, self.f_ext, bc_mask, bc_vals, u_n, v_n, a_n,
                                     H_in=self.H_elem if cfg.enable_damage else None,
                                     H_out=H_n if cfg.enable_damage else None)
            self._nxt = [self.u, self.v, self.a, self.H_elem]
            self.u, self.v, self.a = u_n, v_n, a_n
            if cfg.enable_damage:
                self.H_elem = H_n
                self._explicit_step_count += 1
                k = self._explicit_step_count
                if cfg.damage_every <= 1 or k <= 5 or k % cfg.damage_every == 0:
                    self.step_solve_damage()
            self._step_count += 1
            self._last_stagger_iter = 1
            return self.H_elem
        tol = cfg.stagger_tol
        d_prev_step = self.d.clone()
        aa = None
        if cfg.anderson_depth > 0:
            if getattr(self, "_aa", None) is None:
                self._aa = AndersonAccelerator(self.d.numel(), int(cfg.anderson_depth), self.device)
            else:
                self._aa.reset()
            aa = self._aa
        stag = 0
        for stag in range(cfg.max_stagger):
            need = stag >= 1
            d_old = self.d.clone() if (need or aa is not None) else self.d
            u_old = self.u.clone() if need else self.u
            self.step_mechanics()
            self.step_compute_driving_force()
            self.step_solve_damage(d_prev_step=d_prev_step)
            if aa is not None:
                # the mixed field is the next iterate and the one the convergence test measures
                self.d = aa.step(d_old, self.d, d_prev_step)
            if self.stagger_trace is not None:
                self.stagger_trace.append((self.u.clone(), self.d.clone(), self.H_elem.clone()))
            if need:
                d_change = float(torch.linalg.vector_norm(self.d - d_old) / (torch.linalg.vector_norm(self.d) + 1e-30))
                u_change = float(torch.linalg.vector_norm(self.u - u_old) / (torch.linalg.vector_norm(self.u) + 1e-30))
                if d_change < tol and u_change < tol:
                    break
        else:
            if cfg.fail_on_stagger_nonconvergence:
                raise RuntimeError(f"Stagger loop did not converge after {cfg.max_stagger} iterations")
        self._step_count += 1
        self._last_stagger_iter = stag + 1
        return self.H_elem

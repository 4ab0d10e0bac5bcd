"""Gradient of the peak reaction force of a quasi-static staggered run with respect to a
per-element Gc field (Q4 or T3, isotropic split, AT2), by a hand-written reverse pass.

The forward run is PhAST's quasi-static staggered scheme as this package executes it
(``StaggeredSolver.step_full``, staggered_solver.py:1103-1344): at every load step each
staggered pass j solves the mechanics with the damage of the previous pass,
u_j = U(d_{j-1}) (K(d_{j-1}) u = 0 with the prescribed displacements), raises the
history H_j = max(H_{j-1}, psi0(u_j)), and solves the bound-projected damage problem
d_j = D(H_j, d_start, Gc) on [d_start, 1] (d_start: the damage at the start of the step).
The objective is J = max_k R_k, R_k = sum of f_int(u_k, d_k)_y over the top nodes
(compute_reaction_force, fem_operators.py:1502-1530, kept as a tensor quantity here).

The reverse pass differentiates exactly these operations, pass by pass -- the quantity
PhAST's autograd would differentiate through its own unrolled loop
(SparseSolveAutograd for the mechanics, mechanics_solver.py:1301;
_AdjointDamageSolveField for the damage, damage_solver.py:866-1037) -- with:

* the damage solve on its frozen active set: lam solves A_FF lam_F = g_F (one device
  PCG), giving the Gc-field, history and lower-bound gradients (the damage solver's
  ``linear_solve`` and ``adjoint_grads``);
* the history max: the gradient of H_j goes to psi0(u_j) on the Gauss points where psi0
  won and to H_{j-1} elsewhere; (d psi0/du)^T w is the operators' ``psi_grad_t``;
* the mechanics solve: U^T w = -(d (K(d) u)/dd)^T z with K_ff z = w_f, one stiffness
  solve (``QuasiStaticSolver.solve_stiffness``) and the operators' ``force_dd_t``.

Where no damage node sits on a bound other than the pinned (phase-field Dirichlet) ones,
the frozen-active-set derivative and PhAST's solve-then-clamp adjoint
(``_masked_adjoint_inputs`` / ``_pcg_solve_adjoint_system``, damage_solver.py:400-480) are
the same quantity; with bound-active nodes this module gives the exact derivative of the
projected solve (the held nodes' coupling -(A lam)_i to the lower bound included).

Memory: states are checkpointed every ``checkpoint_every`` load steps in the forward run;
the reverse pass recomputes one segment at a time, recording every staggered pass of it.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from .damage2d import classify_active_set
from .fem2d import stress_split_of


@dataclass
class GradientResult:
    objective: float
    peak_step: int
    reactions: np.ndarray
    grad: torch.Tensor                       # dJ/dGc, (E,)
    passes: list = field(default_factory=list)  # staggered passes per load step


class PeakReactionGradient:
    """dJ/dGc_e for J = max_k R_k over ``n_steps`` load steps of a quasi-static ``StaggeredSolver``.

    ``solver``: a ``phast_b200.StaggeredSolver`` with ``solver_type='quasi_static'`` on a
    structured Q4 or a T3 mesh with the isotropic split; its ``bcs`` prescribe the top displacement
    through ``load_factor``.  ``load(k)`` gives the load factor of step k (1-based);
    ``top`` the node ids of the loaded edge.  The solver's state is reset to its current
    values (u, d, H) at every ``forward`` call.
    """

    def __init__(self, solver, top, load, n_steps, checkpoint_every=10, adjoint_rtol=1e-12):
        cfg = solver.config
        if cfg.solver_type != "quasi_static":
            raise NotImplementedError("the peak-reaction gradient is built for quasi-static staggered runs")
        fem = solver.fem
        mat = solver.material
        if getattr(mat, "energy_split", "isotropic") != "isotropic" or stress_split_of(mat) != "isotropic":
            raise NotImplementedError("the mechanics adjoint kernels cover the isotropic split")
        self.s = solver
        self.fem = fem
        self.top = torch.as_tensor(top, dtype=torch.long, device=fem.device)
        self.load = load
        self.n_steps = int(n_steps)
        self.k = max(1, int(checkpoint_every))
        self.rtol = float(adjoint_rtol)
        self.start = (solver.u.clone(), solver.d.clone(), solver.H_elem.clone())
        bc_mask, _ = solver.bcs.get_masks_and_values()
        self.bc_mask = bc_mask.to(fem.device)
        self.e_top = torch.zeros(fem.n_nodes, 2, dtype=torch.float64, device=fem.device)
        self.e_top[self.top, 1] = 1.0
        pf_mask, _ = (solver.bcs.get_pf_dirichlet_mask_values() if getattr(solver.bcs, "pf_dirichlet_bcs", None)
                      else (None, None))
        self.pf_mask = None if pf_mask is None else pf_mask.to(fem.device)

    # -- forward ---------------------------------------------------------------------------
    def _set_state(self, st):
        s = self.s
        s.u, s.d, s.H_elem = st[0].clone(), st[1].clone(), st[2].clone()

    def _step(self, k, trace=None):
        s = self.s
        s.bcs.load_factor = self.load(k)
        s.stagger_trace = trace
        try:
            s.step_full()
        finally:
            s.stagger_trace = None
        return s.fem.compute_reaction_force(s.u, s.d, self.top, component=1)

    def forward(self, Gc_field):
        """Runs the load path with ``Gc_field``; returns the reactions and keeps the checkpoints."""
        s = self.s
        s.diff_Gc_field = torch.as_tensor(Gc_field, dtype=torch.float64, device=self.fem.device).reshape(-1)
        self._set_state(self.start)
        self.checkpoints = {0: self.start}
        R = []
        for k in range(1, self.n_steps + 1):
            R.append(self._step(k))
            if k % self.k == 0:
                self.checkpoints[k] = (s.u.clone(), s.d.clone(), s.H_elem.clone())
        return np.array(R)

    # -- reverse pieces ----------------------------------------------------------------------
    def _U_t(self, u, d, w):
        """U^T w: -(d(K(d) u)/dd)^T z with K_ff z = w_f (z = 0 on prescribed dofs)."""
        z = self.s.mechanics.solve_stiffness(d, w, self.bc_mask, rtol=self.rtol)
        if not bool(torch.any(z != 0)):
            return torch.zeros(self.fem.n_nodes, dtype=torch.float64, device=u.device)
        return -self.fem.force_dd_t(u, z, d)

    def _damage_vjp(self, H, d_start, d, g, Gc_field):
        """(dJ/dH, dJ/dd_start (N,), dJ/dGc (E,)) of d = D(H, d_start, Gc) for the output gradient g."""
        ds = self.s.damage_solver
        lower, upper, fx, interior = classify_active_set(d, d_start, self.pf_mask)
        lam = ds.linear_solve(H, g * interior, Gc_field=Gc_field, fixed=~interior, rtol=self.rtol)
        g_gc, g_h = ds.adjoint_grads(lam, d, Gc_field=Gc_field)
        g_start = torch.zeros_like(g)
        if bool(lower.any()):
            g_start = (g - ds._apply_full(H, lam, Gc_field=Gc_field)) * lower
        return g_h, g_start, g_gc

    def _step_reverse(self, start, passes, g_u, g_d, g_H, Gc_field, grad):
        """Reverse of one load step from its start state and recorded passes; returns the
        gradients (d, H) of the start state and accumulates dJ/dGc into ``grad``."""
        u0, d_start, H0 = start
        g_dstart = torch.zeros_like(d_start)
        # the outputs of the step are the last pass's iterate
        for j in range(len(passes) - 1, -1, -1):
            u_j, d_j, H_j = passes[j]
            d_prev_pass = passes[j - 1][1] if j > 0 else d_start
            H_prev_pass = passes[j - 1][2] if j > 0 else H0
            # d_j = D(H_j, d_start, Gc)
            gh, gs, ggc = self._damage_vjp(H_j, d_start, d_j, g_d, Gc_field)
            grad += ggc
            g_dstart += gs
            g_H = g_H + gh
            # H_j = max(H_{j-1}, psi0(u_j))
            psi = self.fem.compute_psi_plus(u_j)
            won = (psi > H_prev_pass).to(torch.float64)
            g_u = g_u + self.fem.psi_grad_t(u_j, won * g_H)
            g_H = (1.0 - won) * g_H
            # u_j = U(d_{j-1})
            g_d = self._U_t(u_j, d_prev_pass, g_u)
            g_u = torch.zeros_like(g_u)
        # the first pass's damage input is the start state's damage
        g_dstart = g_dstart + g_d
        return g_dstart, g_H

    def gradient(self, Gc_field):
        """J = max_k R_k and dJ/dGc (E,) by the reverse pass with checkpoint-and-recompute."""
        Gc_field = torch.as_tensor(Gc_field, dtype=torch.float64, device=self.fem.device).reshape(-1)
        R = self.forward(Gc_field)
        kstar = int(np.argmax(R)) + 1
        grad = torch.zeros(self.fem.n_elems, dtype=torch.float64, device=self.fem.device)
        N = self.fem.n_nodes
        g_d = torch.zeros(N, dtype=torch.float64, device=grad.device)
        g_H = torch.zeros_like(self.start[2], dtype=torch.float64)
        passes_per_step = {}
        seg_end = kstar
        while seg_end >= 1:
            seg_start = ((seg_end - 1) // self.k) * self.k
            self._set_state(self.checkpoints[seg_start])
            states, traces = {seg_start: self.checkpoints[seg_start]}, {}
            for k in range(seg_start + 1, seg_end + 1):
                trace = []
                self._step(k, trace)
                traces[k] = trace
                states[k] = (self.s.u.clone(), self.s.d.clone(), self.s.H_elem.clone())
            for k in range(seg_end, seg_start, -1):
                u_k, d_k, _ = states[k]
                g_u = torch.zeros(N, 2, dtype=torch.float64, device=grad.device)
                if k == kstar:
                    # R = e_top . K(d) u: dR/du = K(d) e_top, dR/dd = d(e_top . K(d) u)/dd
                    g_u = self.fem.internal_force(self.e_top, d_k).to(torch.float64)
                    g_d = g_d + self.fem.force_dd_t(u_k, self.e_top, d_k)
                passes_per_step[k] = len(traces[k])
                g_d, g_H = self._step_reverse(states[k - 1], traces[k], g_u, g_d, g_H, Gc_field, grad)
            seg_end = seg_start
        self._set_state(self.start)
        return GradientResult(float(R[kstar - 1]), kstar, R, grad,
                              [passes_per_step[k] for k in sorted(passes_per_step)])

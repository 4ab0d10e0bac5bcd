"""Anderson mixing (type II) of the 2D staggered damage fixed point in numpy.

TEST ORACLE ONLY.  Restates PhAST's ``_AndersonAccelerator`` (src/phast/solvers/
staggered_solver.py:165-255): the history of the last depth + 1 pairs (d_in, G(d_in)),
the regularised normal equations of the residual differences, the extrapolated field,
the 1.5x residual safeguard and the clamp to [floor, 1].
"""
from __future__ import annotations

from collections import deque

import numpy as np


class AndersonAccelerator:
    def __init__(self, m=5, reg=1e-10):
        self.m, self.reg = m, reg
        self.g_hist = deque(maxlen=m + 1)
        self.f_hist = deque(maxlen=m + 1)

    def reset(self):
        self.g_hist.clear()
        self.f_hist.clear()

    def step(self, d_in, d_out, floor=None):
        """The mixed field (staggered_solver.py:194-255)."""
        f = d_out - d_in
        self.g_hist.append(d_out.copy())
        self.f_hist.append(f.copy())
        mk = len(self.f_hist) - 1
        if mk == 0:
            return d_out
        dF = np.stack([self.f_hist[i + 1] - self.f_hist[i] for i in range(mk)], axis=1)
        FtF = dF.T @ dF + self.reg * np.eye(mk)
        Ftf = dF.T @ self.f_hist[-1]
        try:
            gamma = np.linalg.solve(FtF, Ftf)
        except np.linalg.LinAlgError:
            return d_out
        dG = np.stack([self.g_hist[i + 1] - self.g_hist[i] for i in range(mk)], axis=1)
        d_aa = d_out - dG @ gamma
        if np.linalg.norm(d_aa - d_in) > 1.5 * np.linalg.norm(f):
            return d_out
        d_aa = np.maximum(d_aa, floor) if floor is not None else np.maximum(d_aa, 0.0)
        return np.minimum(d_aa, 1.0)

"""Writes tests/golden/checkpoint_ref.pt: a checkpoint written by the reference's own
``save_checkpoint`` (src/phast/solid3d/staggered.py:1638-1663) of a seeded state with the
shapes of a 3x3x3 periodic cell, so the test reads the reference's file with this package's
``load_checkpoint`` and compares the two packages' file layouts.

Usage: python tests/golden/make_golden_checkpoint.py <path to the reference's src directory>
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

N_RED, N_ELEM = 27, 27
META = {"case": "golden", "targets": [0.001, 0.002], "seed": 7}


def seeded_fields():
    rng = np.random.default_rng(7)
    return dict(step=5, increment=4, external_work=0.125,
                x=rng.normal(size=3 * N_RED + 6), d=rng.uniform(0, 1, N_RED), H=rng.uniform(0, 2, (N_ELEM, 8)),
                macro_strain=rng.normal(size=6) * 1e-3, macro_stress=rng.normal(size=6),
                d_prev_step=rng.uniform(0, 0.5, N_RED))


def main(src):
    import torch
    from make_golden import _import_reference
    _import_reference(src)
    from phast.solid3d.staggered import SolverState, save_checkpoint
    f = seeded_fields()
    state = SolverState(**{k: (torch.as_tensor(v, dtype=torch.float64) if isinstance(v, np.ndarray) else v)
                           for k, v in f.items()})
    save_checkpoint(os.path.join(HERE, "checkpoint_ref.pt"), state, meta=META)


if __name__ == "__main__":
    main(sys.argv[1])

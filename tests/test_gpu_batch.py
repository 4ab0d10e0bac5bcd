"""Particle-in-cube cells advanced concurrently on several streams give the same
records as one at a time (needs a B200)."""
import numpy as np
import pytest

from phast_b200.solid3d import batch

pytestmark = pytest.mark.gpu


def test_concurrent_streams_match_sequential():
    cells = batch.particle_cells(seed=5, n_cells=5, sizes=(8, 12, 16))
    idx = list(range(len(cells)))
    seq = batch.run_cells(cells, idx, 2, streams=1)
    par = batch.run_cells(cells, idx, 2, streams=3)
    assert [r.index for r in par] == idx
    for a, b in zip(seq, par):
        sa, sb = np.asarray(a.sigma), np.asarray(b.sigma)
        assert np.linalg.norm(sa - sb) <= 1e-9 * np.linalg.norm(sa)
        assert abs(a.max_damage - b.max_damage) <= 1e-9
    # the load is uniaxial strain in x: sigma_xx grows with the ramp in every cell
    for r in seq:
        s = np.asarray(r.sigma)
        assert s[1, 0] > s[0, 0] > 0

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


def test_batch_cells_against_oracle():
    """Two cells of the batch (8^3 and 12^3, particle + interface shell + matrix) against the numpy
    oracle's staggered increments (the reference's algorithm restated): macro stress per increment
    and the damage field of the last one."""
    from oracle import h8

    cells = batch.particle_cells(seed=5, n_cells=5, sizes=(8, 12, 16))
    picks = [i for i, c in enumerate(cells) if c.n in (8, 12)][:2]
    assert picks
    load = batch.batch_load()
    recs = batch.run_cells(cells, picks, 2)
    for rec in recs:
        cell = cells[rec.index]
        op = batch.build_operator(cell, load)
        C = [h8.isotropic_C(p.E, p.nu) for p in batch.BATCH_PHASES]
        ref = h8.VoxelOperator(op.shape, op.h, op.slot_np, np.stack([c[0] for c in C]), np.array([c[1] for c in C]),
                               np.array([c[2] for c in C]), np.array([p.Gc for p in batch.BATCH_PHASES]),
                               np.array([2, 2, 2]), op.ell, op.kappa, op.pinned_node, 0, (1, 2, 3, 4, 5))
        x = np.zeros(ref.n_mech)
        d = np.zeros(ref.n_red)
        H = np.zeros((ref.n_elements, 8))
        prev = 0.0
        for k in range(2):
            target = load.targets[k]
            x, d, H, _, _, _, sig = h8.increment(ref, h8.Cfg3D(), x, d, H, prev, target)
            prev = target
            got = np.asarray(rec.sigma[k])
            assert np.linalg.norm(got - sig) <= 1e-7 * np.linalg.norm(sig)

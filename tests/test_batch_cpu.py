"""Particle-in-cube batch: seeded geometry, cost-balanced sharding and the gather of
per-cell records across ranks (world size 2 over gloo, no GPU)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from phast_b200.solid3d import batch


def test_particle_cells_are_seeded_and_in_range():
    a = batch.particle_cells(seed=3, n_cells=12)
    b = batch.particle_cells(seed=3, n_cells=12)
    for ca, cb in zip(a, b):
        assert ca.n == cb.n and np.array_equal(ca.phase, cb.phase)
    for c in a:
        assert c.n in (32, 40, 48, 56, 64)
        assert 4 <= len(c.radii) <= 12
        assert np.all(c.radii >= 0.08 * c.n - 1e-12) and np.all(c.radii <= 0.15 * c.n + 1e-12)
        # periodic minimum-image separation of the spheres including their shells
        for i in range(len(c.radii)):
            for j in range(i):
                dv = np.abs(c.centres[i] - c.centres[j])
                dv = np.minimum(dv, c.n - dv)
                assert np.linalg.norm(dv) >= c.radii[i] + c.radii[j] + 1.0 - 1e-9
        counts = np.bincount(c.phase.ravel(), minlength=3)
        assert counts[batch.INCLUSION] > 0 and counts[batch.INTERFACE] > 0
        assert c.phase.shape == (c.n, c.n, c.n)


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_cells_partitions_and_balances(world):
    costs = [c.voxels for c in batch.particle_cells(seed=0, n_cells=40)]
    parts = batch.shard_cells(costs, world)
    assert len(parts) == world
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    lower = max(max(costs), sum(costs) / world)  # no partition beats this
    assert max(loads) <= 4.0 / 3.0 * lower + 1e-9


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n_cells, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cells = batch.particle_cells(seed=1, n_cells=n_cells, sizes=(8, 12, 16))
        parts = batch.shard_cells([c.voxels for c in cells], world)
        # stand-in for the per-cell solve: a record computed from the cell alone
        local = [batch.CellRecord(i, cells[i].n, 1, [[float(cells[i].phase.sum()), rank]], 0.0, 0, 0, 0.0)
                 for i in parts[rank]]
        got = batch.gather_records(local, rank, world)
        if rank == 0:
            out.put([(r.index, r.n, r.sigma[0][0], r.sigma[0][1]) for r in got])
    finally:
        dist.destroy_process_group()


def test_gather_records_two_ranks_gloo():
    world, n_cells = 2, 9
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n_cells, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    cells = batch.particle_cells(seed=1, n_cells=n_cells, sizes=(8, 12, 16))
    parts = batch.shard_cells([c.voxels for c in cells], world)
    owner = {i: r for r, p in enumerate(parts) for i in p}
    assert [r[0] for r in res] == list(range(n_cells))
    for idx, n, s, rank in res:
        assert n == cells[idx].n and s == float(cells[idx].phase.sum()) and rank == owner[idx]


def test_packed_batch_plan_without_gpu():
    """The host plan of a packed batch: packed offsets per cell, brick counts, and refusals."""
    import ctypes as C

    from phast_b200 import _lib
    lib = _lib.load()
    shapes = [(32, 32, 32), (40, 40, 40), (16, 24, 8)]
    grids = (_lib.VoxelGrid * 3)(*[_lib.VoxelGrid(nx, ny, nz, 1, 1, 1, 1.0 / nx, 1.0 / ny, 1.0 / nz)
                                   for nx, ny, nz in shapes])
    ell = (C.c_double * 3)(0.1, 0.05, 0.2)
    ds = (C.c_double * 3)(1.0, 2.0, 3.0)
    h = lib.phastb_batch_create(3, grids, ell, ds, 8, 8, 4)
    assert h
    try:
        out = (C.c_longlong * (7 + 9))()
        assert lib.phastb_batch_sizes(C.c_void_p(h), out) == 0
        n_red = [nx * ny * nz for nx, ny, nz in shapes]
        assert out[0] == sum(n_red) and out[1] == sum(3 * n + 6 for n in n_red) and out[2] == sum(n_red)
        bricks = sum(-(-nx // 8) * -(-ny // 8) * -(-nz // 4) for nx, ny, nz in shapes)
        assert out[3] == bricks
        offs = [tuple(out[7 + 3 * c:10 + 3 * c]) for c in range(3)]
        assert offs[0] == (0, 0, 0)
        assert offs[1] == (n_red[0], 3 * n_red[0] + 6, n_red[0])
        assert offs[2] == (n_red[0] + n_red[1], 3 * (n_red[0] + n_red[1]) + 12, n_red[0] + n_red[1])
    finally:
        lib.phastb_batch_destroy(C.c_void_p(h))
    # an unsupported brick shape, a brick deeper than a cell, a non-positive scale: no plan
    assert not lib.phastb_batch_create(3, grids, ell, ds, 32, 4, 4)
    assert not lib.phastb_batch_create(3, grids, ell, ds, 8, 8, 16)
    bad = (C.c_double * 3)(1.0, 0.0, 3.0)
    assert not lib.phastb_batch_create(3, grids, ell, bad, 8, 8, 4)

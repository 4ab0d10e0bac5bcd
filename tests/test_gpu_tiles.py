"""Tile shapes of the fused voxel elastic action against the oracle (needs a B200).

The action kernel owns ox x oy x kz node bricks and recomputes one halo row of
elements; every tile shape, ragged tiles at the grid edge, grids smaller than a
tile and non-periodic axes must give the oracle's action.
"""
import numpy as np
import pytest
import torch

from conftest import rel
from oracle.h8 import VoxelOperator, isotropic_C

pytestmark = pytest.mark.gpu

GRIDS = [
    ((6, 6, 6), (True, True, True)),
    ((10, 7, 5), (True, True, True)),
    ((5, 4, 3), (False, False, False)),
    ((9, 5, 4), (True, False, True)),
    ((17, 3, 2), (True, True, False)),
]
SHAPES = [None, (16, 12, 16), (14, 14, 8), (24, 8, 4), (8, 8, 2), (4, 4, 4), (3, 2, 1), (1, 1, 1), (16, 8, 0), (5, 3, 0)]


def build(shape, periodic, seed):
    from phast_b200 import solid3d as s3
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    h = (1.0 / nx, 1.1 / ny, 0.9 / nz)
    slot = rng.integers(0, 2, nx * ny * nz)
    phases = [s3.PhaseMaterial("mi_matrix", "isotropic", 0.5, "spectral", 3000.0, 0.35), s3.PhaseMaterial("fibre", "isotropic", 0.4, "spectral", 70000.0, 0.3)]
    load = s3.LoadCase("zz", 2, (0.01,), (), (0, 1, 3, 4, 5))
    op = s3.PeriodicVoxelPhaseFieldOperator.from_slots(s3.VoxelGrid(shape, h, periodic=periodic), slot, phases, 0.1, 1e-6,
                                            load, pinned_node=0)
    Cs, lams, mus = zip(*(isotropic_C(p.E, p.nu) for p in phases))
    ref = VoxelOperator(shape, h, slot, np.stack(Cs), np.array(lams), np.array(mus), np.array([0.5, 0.4]),
                        np.zeros(2, dtype=np.int64), 0.1, 1e-6, 0, 2, (0, 1, 3, 4, 5), periodic=periodic)
    x = rng.standard_normal(op.n_mech) * 1e-3
    d = rng.uniform(0.0, 0.9, op.n_red)
    return op, ref, x, d


@pytest.mark.parametrize("shape,periodic", GRIDS)
def test_tile_shapes_match_oracle(shape, periodic):
    op, ref, x, d = build(shape, periodic, 7)
    want = ref.mech_action(x, ref.degradation(d))
    want1 = ref.mech_action(x)
    xg, dg = torch.as_tensor(x, device="cuda"), torch.as_tensor(d, device="cuda")
    for dt, tol in ((torch.float64, 1e-12), (torch.float32, 3e-5)):
        saved = op.tile_shape(dt)
        try:
            for ts in SHAPES:
                if ts is not None:
                    op.tile_shape(dt, ts)
                got = op.mech_action(xg.to(dt), d=dg.to(dt)).double().cpu().numpy()
                assert rel(got, want) < tol, (dt, ts)
                got1 = op.mech_action(xg.to(dt)).double().cpu().numpy()
                assert rel(got1, want1) < tol, (dt, ts)
        finally:
            op.tile_shape(dt, saved)


def test_autotune_records_a_valid_shape():
    op, ref, x, d = build((12, 10, 8), (True, True, True), 3)
    want = ref.mech_action(x, ref.degradation(d))
    for dt, tol in ((torch.float64, 1e-12), (torch.float32, 3e-5)):
        shape, ms = op.autotune(dt)
        assert ms > 0 and shape[0] >= 1 and shape[1] >= 1 and shape[2] >= 0  # kz = 0: depth chosen per launch
        assert (shape[0] + 1) * (shape[1] + 1) <= 256
        assert op.tile_shape(dt) == shape
        got = op.mech_action(torch.as_tensor(x, device="cuda", dtype=dt),
                             d=torch.as_tensor(d, device="cuda", dtype=dt))
        assert rel(got.double().cpu().numpy(), want) < tol

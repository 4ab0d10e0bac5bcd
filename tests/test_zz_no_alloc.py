"""The allocation-free elastic action, called through the C ABI (needs a B200).

``phastb_h8_mech_apply_noalloc`` exists for callers that cannot allocate device
memory themselves (a host runtime bound through a thin FFI without a device
allocator, or an application whose GPU memory is owned by another framework's
pool).  It keeps its element scratch in a fixed device array inside the library,
so these tests check that it gives the same result as the regular entry point
``phastb_h8_mech_apply`` (which takes a caller workspace) and as the numpy
oracle of the reference's ``mech_action`` on two calls in a row -- the second
call must not see anything left over from the first -- and that it refuses
grids larger than its fixed capacity.  This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the FP64 tolerance of the other operator parity tests


def _cell(shape):
    from phast_b200 import solid3d as s3
    h = 1.0 / shape[2]
    phase = s3.sphere_pore_phase(shape, 0.25, 0, 1)
    phases = [s3.PhaseMaterial("mi_matrix", "isotropic", 0.5, "spectral", 3000.0, 0.35), s3.PhaseMaterial("pore", "isotropic", 0.5, "spectral", 3e-3, 0.35)]
    load = s3.LoadCase.ramp("zz", 2, 0.02, 50)
    return s3.PeriodicVoxelPhaseFieldOperator.from_slots(s3.VoxelGrid(shape, (h, h, h)), phase, phases, 2 * h, 1e-6, load)


def _noalloc(op, x, d, mask=None):
    from phast_b200 import _lib
    y = torch.empty_like(x)
    code = _lib.F64 if x.dtype == torch.float64 else _lib.F32
    st = _lib.load().phastb_h8_mech_apply_noalloc(op.vgrid, op.mat, _lib.ptr(op.slot), code, _lib.ptr(x), None,
                                                  _lib.ptr(d), _lib.ptr(mask), _lib.ptr(y), _lib.stream())
    assert st == _lib.OK, st
    return y


def _rel(a, b):
    return float(torch.linalg.vector_norm((a - b).double()) / torch.linalg.vector_norm(b.double()))


def test_noalloc_matches_regular_entry_point_on_two_calls():
    op = _cell((12, 10, 9))
    rng = np.random.default_rng(11)
    cases = []
    for _ in range(2):
        x = torch.as_tensor(rng.normal(size=op.n_mech) * 1e-3, device="cuda")
        d = torch.as_tensor(rng.uniform(0, 1, size=op.n_red), device="cuda")
        cases.append((x, d))
    mask = op.mech_fixed_mask().to(torch.uint8)
    for x, d in cases:  # two calls in a row, different inputs
        y = _noalloc(op, x, d)
        ref = op.mech_action(x, d=d)
        torch.cuda.synchronize()
        assert _rel(y, ref) < TOL
        ym = _noalloc(op, x, d, mask)
        refm = op.mech_action(x, d=d, mask=mask)
        assert _rel(ym, refm) < TOL
        assert bool((ym[mask.bool()] == 0).all())


def _oracle_op(op):
    from oracle import h8
    C = [h8.isotropic_C(float(p.E), float(p.nu)) for p in op.phases]
    drivers = np.array([0 if p.name == "pore" else 2 for p in op.phases])
    return h8.VoxelOperator(op.shape, op.h, op.slot_np, np.stack([c[0] for c in C]), np.array([c[1] for c in C]),
                            np.array([c[2] for c in C]), np.array([float(p.Gc) for p in op.phases]), drivers,
                            op.ell, op.kappa, op.pinned_node, int(op.load.controlled), tuple(op.load.fixed_zero))


def test_noalloc_matches_oracle_on_two_calls():
    op = _cell((12, 10, 9))
    ref = _oracle_op(op)
    rng = np.random.default_rng(13)
    for _ in range(2):  # two calls in a row, different inputs
        x = rng.normal(size=op.n_mech) * 1e-3
        d = rng.uniform(0, 1, size=op.n_red)
        y = _noalloc(op, torch.as_tensor(x, device="cuda"), torch.as_tensor(d, device="cuda"))
        want = ref.mech_action(x, ref.degradation(d))
        assert float(np.linalg.norm(y.cpu().numpy() - want) / np.linalg.norm(want)) < TOL


def test_noalloc_float32_matches_regular_entry_point():
    op = _cell((8, 8, 8))
    rng = np.random.default_rng(12)
    for _ in range(2):
        x = torch.as_tensor(rng.normal(size=op.n_mech) * 1e-3, device="cuda", dtype=torch.float32)
        d = torch.as_tensor(rng.uniform(0, 1, size=op.n_red), device="cuda", dtype=torch.float32)
        assert _rel(_noalloc(op, x, d), op.mech_action(x, d=d)) < 1e-6


def test_noalloc_refuses_grids_above_capacity():
    from phast_b200 import _lib
    op = _cell((40, 40, 40))  # 64000 voxels > 32768
    x = torch.zeros(op.n_mech, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    st = _lib.load().phastb_h8_mech_apply_noalloc(op.vgrid, op.mat, _lib.ptr(op.slot), _lib.F64, _lib.ptr(x), None,
                                                  None, None, _lib.ptr(y), _lib.stream())
    assert st == _lib.ERR_CAPACITY

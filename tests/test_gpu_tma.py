"""TMA staging of the elastic action's node layers (needs a B200).

With TMA the tile kernel stages every node layer of a brick with tensor copies
issued by one thread (u~ rows and d rows, 16-byte aligned starts) and patches the
halo nodes that wrap around periodic edges; without it every thread stages its
halo-tile nodes through registers.  The element and node arithmetic is the same,
so both stagings must give the same bits: these tests run the actions and a
multigrid-preconditioned FP32 solve (Chebyshev, coarse-level and dot-product
epilogues) once with PHASTB_TMA=0 and once with TMA in fresh processes and
compare them, on grids that take the TMA path (periodic and not) and one that
does not, and check the TMA results against the numpy oracle.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = [((16, 16, 16), (True, True, True)), ((12, 10, 9), (True, True, True)), ((7, 8, 5), (False, False, True)),
         ((9, 9, 9), (True, True, True)), ((32, 32, 32), (True, True, True))]

SCRIPT = r"""
import sys, numpy as np, torch
sys.path.insert(0, '.')
from phast_b200 import solid3d as s3, _lib
cases = %r
out = {}
for ci, (shape, per) in enumerate(cases):
    h = 1.0 / shape[2]
    phase = s3.sphere_pore_phase(shape, 0.25, 0, 1)
    phases = [s3.PhaseMaterial("mi_matrix", "isotropic", 0.5, "spectral", 3000.0, 0.35),
              s3.PhaseMaterial("pore", "isotropic", 0.5, "spectral", 3e-3, 0.35)]
    load = s3.LoadCase.ramp("zz", 2, 0.02, 50)
    op = s3.PeriodicVoxelPhaseFieldOperator.from_slots(s3.VoxelGrid(shape, (h, h, h), periodic=per), phase, phases,
                                                       2 * h, 1e-6, load)
    rng = np.random.default_rng(ci)
    x = torch.as_tensor(rng.normal(size=op.n_mech) * 1e-3, device="cuda")
    d = torch.as_tensor(rng.uniform(0, 1, size=op.n_red), device="cuda")
    for dt in (torch.float64, torch.float32):
        xx, dd = x.to(dt), d.to(dt)
        tag = f"{ci}_{str(dt)[-2:]}"
        out["tma_" + tag] = _lib.load().phastb_h8_tma_staging(op.vgrid, _lib.F64 if dt == torch.float64 else _lib.F32)
        out["yd_" + tag] = op.mech_action(xx, d=dd).double().cpu().numpy()
        out["yg_" + tag] = op.mech_action(xx, op.degradation(dd)).double().cpu().numpy()
        out["y1_" + tag] = op.mech_action(xx).double().cpu().numpy()
    if all(per) and shape[0] %% 4 == 0 and shape[0] >= 16:
        sol, info = s3.solve_constrained_form(op, s3.MechForm(precond="gmg", mixed=True), fixed_mask=op.mech_fixed_mask(),
                                              fixed_values=op.mech_fixed_values(0.004), d=d * 0.5, rtol=1e-8,
                                              maxiter=2000)
        out[f"sol_{ci}"] = sol.cpu().numpy()
        out[f"its_{ci}"] = np.array([info.iterations])
np.savez(sys.argv[1], **out)
""" % (CASES,)


def _run(tma, path):
    env = dict(os.environ, PHASTB_TMA="1" if tma else "0")
    subprocess.run([sys.executable, "-c", SCRIPT, path], check=True, cwd=ROOT, env=env, timeout=900)
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="module")
def runs():
    with tempfile.TemporaryDirectory() as tmp:
        yield _run(True, os.path.join(tmp, "tma.npz")), _run(False, os.path.join(tmp, "regs.npz"))


def test_tma_staging_is_taken_where_eligible(runs):
    t, r = runs
    # rx a multiple of 4 (FP32) / 2 (FP64) words: 16, 12, 8 (non-periodic 7 + 1) and 32 take TMA; 9 does not
    for ci, expect32, expect64 in [(0, 1, 1), (1, 1, 1), (2, 1, 1), (3, 0, 0), (4, 1, 1)]:
        assert int(t[f"tma_{ci}_32"]) == expect32 and int(t[f"tma_{ci}_64"]) == expect64
        assert int(r[f"tma_{ci}_32"]) == 0 and int(r[f"tma_{ci}_64"]) == 0


def test_tma_and_register_staging_give_the_same_bits(runs):
    """Nodal rows: the same arithmetic on the same staged values, so the same bits.  The six
    macro-strain rows and the solves also depend on how the per-block partial sums are grouped,
    which follows the launch grid; they are held to 1e-12 (FP64) / 1e-6 (FP32) and 1e-7."""
    t, r = runs
    for k in t:
        if k.startswith("y"):
            ny = t[k].shape[0] - 6
            assert np.array_equal(t[k][:ny], r[k][:ny]), k
            assert rel(t[k][ny:], r[k][ny:]) < (1e-12 if k.endswith("64") else 1e-6), k
        elif k.startswith("sol"):
            assert rel(t[k], r[k]) < 1e-7, k


def test_tma_actions_against_oracle(runs):
    from oracle import h8
    from phast_b200 import solid3d as s3
    t, _ = runs
    for ci, (shape, per) in enumerate(CASES[:3]):
        h = 1.0 / shape[2]
        phase = s3.sphere_pore_phase(shape, 0.25, 0, 1)
        C0, l0, m0 = h8.isotropic_C(3000.0, 0.35)
        C1, l1, m1 = h8.isotropic_C(3e-3, 0.35)
        # the operator's pinned node only enters the masks, not the action
        ref = h8.VoxelOperator(shape, (h, h, h), phase.reshape(-1).astype(np.int64), np.stack([C0, C1]),
                               np.array([l0, l1]), np.array([m0, m1]), np.array([0.5, 0.5]), np.array([2, 0]), 2 * h,
                               1e-6, 0, 2, (0, 1, 3, 4, 5), periodic=per)
        rng = np.random.default_rng(ci)
        x = rng.normal(size=ref.n_mech) * 1e-3
        d = rng.uniform(0, 1, size=ref.n_red)
        want = ref.mech_action(x, ref.degradation(d))
        assert rel(t[f"yd_{ci}_64"], want) < 1e-12
        assert rel(t[f"yd_{ci}_32"], want) < 1e-5

"""Multigrid and mixed-precision mechanics forms against the plain FP64 solve (needs a B200).

The forms change how the constrained system is solved, not the system: each must
reach the same FP64 residual criterion as PhAST's Jacobi PCG (rtol 1e-8 on ||b_f||).
Two fields that both meet it differ by up to cond(A) x rtol; the 1e-6-contrast pore
cell is badly conditioned, so the fields are compared at 1e-5 after a 1e-8 solve and
at 1e-7 after a 1e-10 solve.
"""
import numpy as np
import pytest
import torch

from conftest import golden, rel

pytestmark = pytest.mark.gpu

FORMS = [
    ("gmg", dict(precond="gmg")),
    ("mixed-jacobi", dict(mixed=True)),
    ("mixed-gmg", dict(precond="gmg", mixed=True)),
]


def cell(n, r=0.2):
    from phast_b200 import solid3d as s3
    h = 1.0 / n
    phase = s3.sphere_pore_phase((n, n, n), r, 0, 1)
    phases = [s3.PhaseMaterial("mi_matrix", "isotropic", 0.5, "spectral", 3000.0, 0.35), s3.PhaseMaterial("pore", "isotropic", 0.5, "spectral", 3e-3, 0.35)]
    return s3.PeriodicVoxelPhaseFieldOperator.from_slots(s3.VoxelGrid((n, n, n), (h, h, h)), phase, phases, 2 * h, 1e-6,
                                              s3.LoadCase.ramp("zz", 2, 0.02, 50))


def smooth_damage(op, seed):
    n = op.shape[0]
    rng = np.random.default_rng(seed)
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    d = 0.45 * (1 + np.sin(2 * np.pi * (i + rng.uniform()) / n) * np.cos(2 * np.pi * (k + rng.uniform()) / n))
    return torch.as_tensor(d.reshape(-1), device="cuda")


@pytest.mark.parametrize("name,kw", FORMS)
def test_forms_match_plain_solve(name, kw):
    from phast_b200 import solid3d as s3
    op = cell(16)
    d = smooth_damage(op, 3)
    mask, vals = op.mech_fixed_mask(), op.mech_fixed_values(0.01)
    x_ref, info_ref = s3.solve_constrained(op.mech_operator(d=d), diag=op.mech_diagonal(d=d), fixed_mask=mask, fixed_values=vals, rtol=1e-8, maxiter=20000)
    assert info_ref.converged
    x, info = s3.solve_constrained_form(op, s3.MechForm(**kw), fixed_mask=mask, fixed_values=vals, d=d, rtol=1e-8,
                                        maxiter=20000)
    assert info.converged, info
    assert info.relative_residual <= 1e-8 * 1.0001
    # the FP64 residual of the returned field, recomputed by the plain operator
    r = op.mech_action(x, d=d, mask=mask)
    assert float(torch.linalg.vector_norm(r)) <= 1.01e-8 * info.rhs_norm
    assert rel(x.cpu(), x_ref.cpu()) < 1e-5
    if kw.get("precond") == "gmg":
        assert info.iterations < info_ref.iterations / 4, (info.iterations, info_ref.iterations)
    x_ref, _ = s3.solve_constrained(op.mech_operator(d=d), diag=op.mech_diagonal(d=d), fixed_mask=mask, fixed_values=vals, rtol=1e-10, maxiter=40000)
    x, info = s3.solve_constrained_form(op, s3.MechForm(**kw), fixed_mask=mask, fixed_values=vals, d=d, rtol=1e-10,
                                        maxiter=20000)
    assert info.converged, info
    assert rel(x.cpu(), x_ref.cpu()) < 1e-7


def test_gmg_warm_start_and_uniaxial_stress_mask():
    """Free macro-stress components (E rows in the system) and a warm start."""
    from phast_b200 import solid3d as s3
    op = cell(16)
    op.load = s3.LoadCase("zz", 2, (0.01,), free=(0, 1, 3, 4, 5), fixed_zero=())
    d = smooth_damage(op, 5)
    mask, vals = op.mech_fixed_mask(), op.mech_fixed_values(0.01)
    x_ref, _ = s3.solve_constrained(op.mech_operator(d=d), diag=op.mech_diagonal(d=d), fixed_mask=mask, fixed_values=vals, rtol=1e-10, maxiter=40000)
    x0 = x_ref * (1 + 1e-3)
    for kw in (dict(precond="gmg"), dict(precond="gmg", mixed=True)):
        x, info = s3.solve_constrained_form(op, s3.MechForm(**kw), fixed_mask=mask, fixed_values=vals, d=d,
                                            x0=x0, rtol=1e-10, maxiter=20000)
        assert info.converged
        assert rel(x.cpu(), x_ref.cpu()) < 1e-7
        sig = op.macro_stress(x, d=d).cpu().numpy()
        assert np.abs(sig[[0, 1, 3, 4, 5]]).max() < 1e-6 * abs(sig[2])  # free components carry no stress


@pytest.mark.parametrize("name,kw", FORMS)
def test_staggered_increments_forms_golden(name, kw):
    """Three staggered increments of the 6^3 golden cell with each form (2 multigrid levels)."""
    from phast_b200 import solid3d as s3
    g = golden("h8_staggered")
    shape = tuple(int(v) for v in g["shape"])
    h = float(g["h"])
    slot = (g["phase"].reshape(-1) == 4).astype(np.int64)
    phases = [s3.PhaseMaterial("mi_matrix", "isotropic", 0.5, "spectral", 3000.0, 0.35), s3.PhaseMaterial("pore", "isotropic", 0.5, "spectral", 3e-3, 0.35)]
    load = s3.LoadCase("zz", 2, tuple(float(t) for t in g["targets"]), (), (0, 1, 3, 4, 5))
    op = s3.PeriodicVoxelPhaseFieldOperator.from_slots(s3.VoxelGrid(shape, (h, h, h)), slot, phases, 2 * h, 1e-6, load)
    form = s3.MechForm(levels=2, **kw)
    solver = s3.StaggeredSolver(op, form=form)
    state = solver.initial_state()
    for k, target in enumerate(g["targets"]):
        state, rec = solver.advance(state, float(target))
        assert rel(state.x.cpu(), g["x"][k]) < 1e-6
        assert rel(state.d.cpu(), g["d"][k]) < 1e-6
        assert rel(state.macro_stress.numpy(), g["sigma"][k]) < 1e-6


def test_device_side_loop_matches_chunked_loop():
    """PHASTB_DEVICE_LOOP=1 (conditional-WHILE graphs) gives the chunked loop's solution."""
    import os
    import subprocess
    import sys
    code = (
        "import sys; sys.path.insert(0, 'tests'); sys.path.insert(0, '.');"
        "import torch, numpy as np; from test_gpu_forms import cell, smooth_damage;"
        "from phast_b200 import solid3d as s3;"
        "op = cell(16); d = smooth_damage(op, 3); m, v = op.mech_fixed_mask(), op.mech_fixed_values(0.01);"
        "x, i = s3.solve_constrained(op.mech_operator(d=d), diag=op.mech_diagonal(d=d), fixed_mask=m, fixed_values=v, rtol=1e-10, maxiter=20000);"
        "y, j = s3.solve_constrained_form(op, s3.MechForm(precond='gmg', mixed=True), fixed_mask=m, fixed_values=v,"
        " d=d, rtol=1e-10, maxiter=20000);"
        "np.save(sys.argv[1], np.stack([x.cpu().numpy(), y.cpu().numpy()]))")
    import tempfile
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    outs = {}
    with tempfile.TemporaryDirectory() as tmp:
        for flag in ("0", "1"):
            path = os.path.join(tmp, f"loop_{flag}.npy")
            env = dict(os.environ, PHASTB_DEVICE_LOOP=flag)
            subprocess.run([sys.executable, "-c", code, path], check=True, cwd=root, env=env, timeout=600)
            outs[flag] = np.load(path)
    for k in range(2):
        a, b = outs["0"][k], outs["1"][k]
        assert np.linalg.norm(a - b) <= 1e-8 * np.linalg.norm(a)

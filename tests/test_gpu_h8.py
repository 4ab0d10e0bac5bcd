"""CUDA periodic-voxel path against the reference's golden vectors (needs a B200)."""
import numpy as np
import pytest
import torch

from conftest import golden, rel

pytestmark = pytest.mark.gpu

TOL = 1e-12


def cuda(x, dtype=torch.float64):
    return torch.as_tensor(np.asarray(x)).to("cuda", dtype)


def make_op(g, controlled=2):
    from phast_b200 import solid3d as s3
    shape = tuple(int(v) for v in g["shape"])
    h = float(g["h"])
    slot = (g["phase"].reshape(-1) == 4).astype(np.int64)
    phases = [s3.PhaseMaterial("mi_matrix", "isotropic", 0.5, "spectral", 3000.0, 0.35), s3.PhaseMaterial("pore", "isotropic", 0.5, "spectral", 3000.0 * 1e-6, 0.35)]
    load = s3.LoadCase("zz", controlled, (0.01,), (), tuple(i for i in range(6) if i != controlled))
    return s3.PeriodicVoxelPhaseFieldOperator.from_slots(s3.VoxelGrid(shape, (h, h, h)), slot, phases, 2 * h, 1e-6, load)


def test_h8_operator_golden():
    g = golden("h8_ops")
    op = make_op(g)
    assert op.pinned_node == int(g["pinned"])
    assert abs(op.damage_scale - float(g["damage_scale"])) <= 1e-12 * op.damage_scale
    x, d, H = cuda(g["x"]), cuda(g["d"]), cuda(g["H"])
    gq = op.degradation(d)
    assert rel(gq.cpu(), g["g"]) < TOL
    assert rel(op.mech_action(x, gq).cpu(), g["mech_g"]) < TOL
    assert rel(op.mech_action(x, d=d).cpu(), g["mech_g"]) < TOL
    assert rel(op.mech_action(x).cpu(), g["mech_1"]) < TOL
    assert rel(op.mech_diagonal(gq).cpu(), g["mdiag_g"]) < TOL
    assert rel(op.mech_diagonal().cpu(), g["mdiag_1"]) < TOL
    # closed-form eigenvalues (the reference's CUDA path) vs eigvalsh on CPU
    assert rel(op.driving_force(x).cpu(), g["Y"]) < 1e-9
    assert rel(op.damage_action(d, H).cpu(), g["dact"]) < TOL
    assert rel(op.damage_action(d).cpu(), g["dact0"]) < TOL
    assert rel(op.damage_rhs(H).cpu(), g["drhs"]) < TOL
    assert rel(op.damage_diagonal(H).cpu(), g["ddiag"]) < TOL
    assert rel(op.macro_stress(x, gq).cpu(), g["sigma"]) < TOL
    assert abs(float(op.elastic_energy(x, gq)) - g["energy"][0]) <= 1e-12 * abs(g["energy"][0])


def test_h8_float32_apply_close():
    g = golden("h8_ops")
    op = make_op(g)
    x, d = cuda(g["x"], torch.float32), cuda(g["d"], torch.float32)
    y = op.mech_action(x, d=d)
    assert y.dtype == torch.float32
    assert rel(y.double().cpu(), g["mech_g"]) < 1e-5


def test_h8_constrained_solve_golden():
    from phast_b200 import solid3d as s3
    g = golden("h8_ops")
    op = make_op(g)
    d = cuda(g["d"])
    x, info = s3.solve_constrained(op.mech_operator(d=d), diag=op.mech_diagonal(d=d), fixed_mask=op.mech_fixed_mask(),
                                   fixed_values=op.mech_fixed_values(0.01), rtol=1e-8, maxiter=5000, check_every=10)
    assert info.converged and info.iterations == int(g["x_solve_iters"][0])
    assert rel(x.cpu(), g["x_solve"]) < 1e-7


def test_h8_box_kkt_golden():
    from phast_b200 import solid3d as s3
    g = golden("h8_ops")
    op = make_op(g)
    lower = cuda(g["lower_kkt"])
    res = s3.solve_h8_scalar_box_kkt(op.damage_system(cuda(g["H_kkt"])), lower_bound=lower, upper_bound=1.0,
                                     initial=lower, linear_tolerance=1e-10, kkt_tolerance=1e-8,
                                     max_linear_iterations=4000, max_active_set_iterations=64)
    assert res.satisfies_kkt
    assert res.total_pcg_iterations == int(g["kkt_pcg"][0]) and res.active_set_iterations == int(g["kkt_sets"][0])
    assert rel(res.solution.cpu(), g["d_kkt"]) < 1e-12
    assert float((res.solution - lower).min()) >= 0.0 and float(res.solution.max()) <= 1.0


def test_h8_box_kkt_mixed_precision_golden():
    """PHASTB_DAMAGE_MIXED=1 (FP32 CG under FP64 refinement) meets the same FP64 threshold."""
    import os
    import subprocess
    import sys
    import tempfile
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import sys; sys.path.insert(0, 'tests'); sys.path.insert(0, '.'); import numpy as np;"
        "from conftest import golden; from test_gpu_h8 import make_op, cuda; from phast_b200 import solid3d as s3;"
        "g = golden('h8_ops'); op = make_op(g); lower = cuda(g['lower_kkt']);"
        "res = s3.solve_h8_scalar_box_kkt(op.damage_system(cuda(g['H_kkt'])), lower_bound=lower, upper_bound=1.0,"
        " initial=lower, linear_tolerance=1e-10, kkt_tolerance=1e-8, max_linear_iterations=4000,"
        " max_active_set_iterations=64);"
        "np.save(sys.argv[1], np.concatenate([res.solution.cpu().numpy(),"
        " [float(res.satisfies_kkt), float(res.active_set_iterations)]]))")
    g = golden("h8_ops")
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "kkt_mixed.npy")
        subprocess.run([sys.executable, "-c", code, path], check=True, cwd=root,
                       env=dict(os.environ, PHASTB_DAMAGE_MIXED="1"), timeout=600)
        out = np.load(path)
    d, ok, sets = out[:-2], out[-2], out[-1]
    assert ok == 1.0 and int(sets) == int(g["kkt_sets"][0])
    assert rel(d, g["d_kkt"]) < 1e-9
    assert float((d - g["lower_kkt"]).min()) >= 0.0 and float(d.max()) <= 1.0


def test_h8_staggered_increments_golden():
    from phast_b200 import solid3d as s3
    g = golden("h8_staggered")
    op = make_op(g)
    op.load = s3.LoadCase("zz", 2, tuple(float(t) for t in g["targets"]), (), (0, 1, 3, 4, 5))
    solver = s3.StaggeredSolver(op)
    state = solver.initial_state()
    for k, target in enumerate(g["targets"]):
        state, rec = solver.advance(state, float(target))
        assert rec.stagger_iters == int(g["stag"][k])
        assert rec.pcg_iters_mech == int(g["pcg_mech"][k]) and rec.pcg_iters_pf == int(g["pcg_pf"][k])
        assert rel(state.x.cpu(), g["x"][k]) < 1e-7
        assert rel(state.d.cpu(), g["d"][k]) < 1e-7
        assert rel(state.macro_stress.numpy(), g["sigma"][k]) < 1e-7

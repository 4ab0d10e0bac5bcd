"""Which PhAST solver options the backend runs (CPU): the PF-CZM law, the crack closure, Anderson
mixing and history-only irreversibility are run; what the GPU path does not run is named so that
building an operator or solver raises ``NotImplementedError`` instead of silently changing the
algorithm."""
import pytest

from phast_b200.solid3d.model import SolverConfig, unsupported_options
from phast_b200.solid3d.operator import pfczm_softening_parameters


@pytest.mark.parametrize("kw", [dict(), dict(damage_law="pfczm"), dict(crack_closure="axes"),
                                dict(anderson_depth=3), dict(anderson_depth=6, anderson_start=3),
                                dict(irreversibility="history_only"), dict(history="current")])
def test_run_options_are_accepted(kw):
    assert unsupported_options(SolverConfig(**kw)) == []


@pytest.mark.parametrize("kw,name", [(dict(anderson_depth=7), "anderson_depth"),
                                     (dict(energy_split_band="interface"), "energy_split_band")])
def test_other_options_are_named(kw, name):
    bad = unsupported_options(SolverConfig(**kw))
    assert len(bad) == 1 and bad[0].startswith(name)


def test_pfczm_softening_parameters():
    # Wu's linear and exponential softening (physics/pfczm.py:57-65)
    assert pfczm_softening_parameters("linear") == (-0.5, 0.0)
    a2, a3 = pfczm_softening_parameters("exponential")
    assert abs(a2 - (2.0 ** (5.0 / 3.0) - 3.0)) < 1e-15 and a3 == 0.0
    with pytest.raises(ValueError):
        pfczm_softening_parameters("cubic")


@pytest.mark.parametrize("kw", [dict(anderson_start=1), dict(anderson_start=True), dict(dtype="float32"),
                                dict(device="mps"), dict(device="tpu:0"), dict(num_threads=0),
                                dict(crack_closure="axes", anderson_depth=2),
                                dict(band_stress="variational"),
                                dict(pfczm_p=1.5, damage_law="pfczm"), dict(pfczm_p=float("nan"), damage_law="pfczm"),
                                dict(pfczm_p=2.5), dict(pfczm_softening="exponential"), dict(pfczm_max_newton=50),
                                dict(damage_law="pfczm", pfczm_max_newton=0),
                                dict(damage_law="pfczm", irreversibility="history_only"),
                                dict(damage_law="pfczm", pfczm_p=2.5),
                                dict(damage_law="pfczm", pfczm_softening="exponential")])
def test_invalid_combinations_raise(kw):
    # the reference's SolverConfig refuses the same settings (solid3d/model.py:840-895)
    with pytest.raises(ValueError):
        SolverConfig(**kw)


def test_valid_combinations_normalise():
    cfg = SolverConfig(damage_law="pfczm", pfczm_softening="exponential", pfczm_p=2.5, pfczm_max_newton=40)
    assert cfg.pfczm_p == 2.5 and cfg.pfczm_max_newton == 40
    cfg = SolverConfig(damage_law="pfczm", pfczm_p=2.0)
    assert cfg.pfczm_p == 2 and isinstance(cfg.pfczm_p, int)
    cfg = SolverConfig(energy_split_band="interface", band_stress="variational", anderson_depth=2.0, anderson_start=3.0)
    assert cfg.anderson_depth == 2 and isinstance(cfg.anderson_start, int)


@pytest.mark.parametrize("kw", [dict(plasticity_model="j2_isotropic", yield_stress=300.0),
                                dict(driving_force="principal_stress"), dict(sigma_ts=3.0)])
def test_2d_solver_refuses_couplings_it_does_not_run(kw):
    # refused before any mesh or device work, so this runs without a GPU
    from phast_b200.fem2d import Material
    from phast_b200.staggered2d import StaggeredSolver, SolverConfig as Config2D
    with pytest.raises(NotImplementedError):
        StaggeredSolver(None, Material(**kw), None, Config2D(solver_type="quasi_static"))


@pytest.mark.parametrize("kw", [dict(softmax_H_beta=10.0), dict(time_integrator="generalized_alpha"),
                                dict(time_integrator="gen_alpha"), dict(adaptive_refine=True),
                                dict(adaptive_stagger_tol=True), dict(adaptive_dt=True),
                                dict(fresh_d_in_corrector=True)])
def test_2d_solver_refuses_options_it_does_not_run(kw):
    from phast_b200.fem2d import Material
    from phast_b200.staggered2d import StaggeredSolver, SolverConfig as Config2D
    with pytest.raises(NotImplementedError):
        StaggeredSolver(None, Material(), None, Config2D(**kw))


def test_reduced_of_full_matches_reference_map():
    # the full-to-reduced node map behind expand_damage, against the reference's own map
    # (tests/golden/make_golden_periodic_map.py); the index arithmetic runs on the host
    import types
    from conftest import golden
    from phast_b200.solid3d.operator import PeriodicVoxelPhaseFieldOperator as Op
    g = golden("periodic_map")
    for n in range(int(g["n"][0])):
        shape, per = tuple(int(v) for v in g[f"shape_{n}"]), tuple(bool(v) for v in g[f"periodic_{n}"])
        red = tuple(s if p else s + 1 for s, p in zip(shape, per))
        assert red == tuple(int(v) for v in g[f"reduced_shape_{n}"])
        fake = types.SimpleNamespace(shape=shape, reduced_shape=red, device="cpu", _rof=None,
                                     vgrid=types.SimpleNamespace(px=int(per[0]), py=int(per[1]), pz=int(per[2])))
        assert (Op.reduced_of_full(fake).numpy() == g[f"rof_{n}"]).all(), n


def test_2d_set_damage_checks_and_copies():
    # the method only touches self.d, so a stand-in object with CPU tensors exercises it
    import types
    import torch
    from phast_b200.staggered2d import StaggeredSolver
    fake = types.SimpleNamespace(d=torch.zeros(5, dtype=torch.float64))
    new = torch.linspace(0, 1, 5, dtype=torch.float32)
    StaggeredSolver.set_damage(fake, new)
    assert fake.d.dtype == torch.float64 and torch.equal(fake.d, new.double()) and fake.d.data_ptr() != new.data_ptr()
    with pytest.raises(ValueError):
        StaggeredSolver.set_damage(fake, torch.zeros(4, dtype=torch.float64))
    with pytest.raises(ValueError):
        StaggeredSolver.set_damage(fake, [0.0] * 5)

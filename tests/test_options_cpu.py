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
                                     (dict(energy_split_band="interface"), "energy_split_band"),
                                     (dict(dtype="float32"), "dtype")])
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

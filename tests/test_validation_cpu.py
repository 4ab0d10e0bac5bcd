"""The 3D data classes, the 2D ``Material`` and the 2D ``SolverConfig`` accept and refuse the same constructor
arguments as the reference's (src/phast/solid3d/model.py:183-897, src/phast/physics/material.py:
80-257), with the same exception class and the same normalised fields: cases recorded from the
reference's own classes by ``tests/golden/make_golden_validation.py``."""
import importlib.util
import json
import os

import pytest

from conftest import GOLDEN
import types

import phast_b200.solid3d.model as _model3d
from phast_b200.fem2d import Material
from phast_b200.staggered2d import SolverConfig as Config2D

ours = types.SimpleNamespace(**vars(_model3d))
ours.Material, ours.Config2D = Material, Config2D

_spec = importlib.util.spec_from_file_location("make_golden_validation",
                                               os.path.join(GOLDEN, "make_golden_validation.py"))
_script = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(_script)

with open(os.path.join(GOLDEN, "validation.json")) as _f:
    CASES = json.load(_f)


def test_fixture_covers_the_script_cases():
    assert [dict(cls=c["cls"], kw=c["kw"]) for c in CASES] == json.loads(json.dumps(_script.CASES))


@pytest.mark.parametrize("case", CASES, ids=[f"{c['cls']}-{i}" for i, c in enumerate(CASES)])
def test_same_outcome_as_reference(case):
    assert _script.outcome(ours, case) == case["outcome"], case["kw"]

"""The drop-in boundary: this package's public signatures against the reference's (CPU).

``tests/golden/reference_signatures.json`` was written by
``tests/golden/make_signatures.py`` from the reference's own modules.  For
every mirrored function or method, every reference parameter must exist here
under the same name, of the same kind, in the same order and (for constant
defaults) with the same default; parameters this package adds must come after
them and have defaults.  For every mirrored data class the field names must be
the reference's, in order (followed by the few fields this package adds, listed below).
"""
import dataclasses
import inspect
import json
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
with open(os.path.join(ROOT, "tests", "golden", "reference_signatures.json")) as f:
    REF = json.load(f)

# defaults that differ on purpose: the device of a GPU backend
DEFAULT_EXCEPTIONS = set()
# fields this package adds after the reference's: the FP32 state of the 2D explicit step
EXTRA_FIELDS = {"phast.solvers.staggered_solver:SolverConfig": ["dtype"]}


def _ours(module, qualname):
    import phast_b200
    from phast_b200 import solid3d
    top = solid3d if module.startswith("phast.solid3d") or module == "phast.solvers.box_kkt_h8" else phast_b200
    obj = top
    for part in qualname.split("."):
        obj = getattr(obj, part)
    return obj


@pytest.mark.parametrize("key", sorted(REF["functions"]))
def test_signature_matches_reference(key):
    module, qualname = key.split(":")
    ours = list(inspect.signature(_ours(module, qualname)).parameters.values())
    ref = REF["functions"][key]
    assert len(ours) >= len(ref), f"{key}: fewer parameters than the reference"
    for p, r in zip(ours, ref):
        assert p.name == r["name"], f"{key}: parameter {p.name!r} where the reference has {r['name']!r}"
        assert p.kind.name == r["kind"], f"{key}: {p.name} is {p.kind.name}, the reference's is {r['kind']}"
        if "default" in r:
            assert p.default is not inspect.Parameter.empty, f"{key}: {p.name} needs a default"
            if r["default"] is not None and (key, p.name) not in DEFAULT_EXCEPTIONS:
                assert repr(p.default) == r["default"], f"{key}: default of {p.name} {p.default!r} != {r['default']}"
        else:
            assert p.default is inspect.Parameter.empty, f"{key}: {p.name} has a default the reference lacks"
    for p in ours[len(ref):]:
        assert p.default is not inspect.Parameter.empty or p.kind in (p.VAR_POSITIONAL, p.VAR_KEYWORD), \
            f"{key}: added parameter {p.name} needs a default"


@pytest.mark.parametrize("key", sorted(REF["dataclasses"]))
def test_dataclass_fields_match_reference(key):
    module, qualname = key.split(":")
    cls = _ours(module, qualname)
    assert [f.name for f in dataclasses.fields(cls)] == REF["dataclasses"][key] + EXTRA_FIELDS.get(key, [])

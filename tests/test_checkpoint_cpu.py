"""Checkpoints (CPU): this package reads a checkpoint the reference's ``save_checkpoint`` wrote
(``tests/golden/make_golden_checkpoint.py``) and writes files with the same layout, so a run
resumes across the two packages; bad files raise the reference's errors."""
import importlib.util
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from phast_b200.solid3d import SolverState, load_checkpoint, save_checkpoint

_spec = importlib.util.spec_from_file_location("make_golden_checkpoint",
                                               os.path.join(GOLDEN, "make_golden_checkpoint.py"))
_script = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(_script)
REF = os.path.join(GOLDEN, "checkpoint_ref.pt")


def _layout(obj):
    if isinstance(obj, dict):
        return {k: _layout(v) for k, v in obj.items()}
    if isinstance(obj, torch.Tensor):
        return ("tensor", obj.dtype, tuple(obj.shape), obj.device.type)
    return type(obj).__name__


def test_reads_the_reference_file():
    state, meta = load_checkpoint(REF)
    f = _script.seeded_fields()
    assert meta == _script.META
    assert (state.step, state.increment, state.external_work) == (f["step"], f["increment"], f["external_work"])
    for name in ("x", "d", "H", "macro_strain", "macro_stress", "d_prev_step"):
        assert np.array_equal(getattr(state, name).numpy(), f[name]), name


def test_writes_the_reference_layout(tmp_path):
    state, meta = load_checkpoint(REF)
    out = save_checkpoint(tmp_path / "sub" / "ours.pt", state, meta=meta)
    assert out.exists() and not (tmp_path / "sub" / "ours.pt.tmp").exists()
    ours = torch.load(out, map_location="cpu", weights_only=True)
    ref = torch.load(REF, map_location="cpu", weights_only=True)
    assert _layout(ours) == _layout(ref)
    assert ours["meta_json"] == ref["meta_json"]
    for name, value in ref["state"].items():
        if isinstance(value, torch.Tensor):
            assert torch.equal(ours["state"][name], value), name
        else:
            assert ours["state"][name] == value, name
    again, meta2 = load_checkpoint(out)
    assert meta2 == meta and torch.equal(again.x, state.x) and again.increment == state.increment


def test_bad_files_raise(tmp_path):
    torch.save({"format": "other"}, tmp_path / "a.pt")
    with pytest.raises(ValueError):
        load_checkpoint(tmp_path / "a.pt")
    payload = torch.load(REF, map_location="cpu", weights_only=True)
    payload["version"] = 2
    torch.save(payload, tmp_path / "b.pt")
    with pytest.raises(ValueError):
        load_checkpoint(tmp_path / "b.pt")
    payload["version"] = 1
    payload["state"]["d"] = payload["state"]["d"].float()
    torch.save(payload, tmp_path / "c.pt")
    with pytest.raises(ValueError):
        load_checkpoint(tmp_path / "c.pt")
    with pytest.raises(TypeError):
        save_checkpoint(tmp_path / "d.pt", {"x": 1})

"""The C-ABI library loads without a GPU and exports every symbol include/phastb.h declares."""
import os
import re

from conftest import ROOT


def declared_functions():
    text = open(os.path.join(ROOT, "include", "phastb.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(phastb_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported():
    from phast_b200 import _lib
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_header():
    from phast_b200 import _lib
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_version_and_sizes_callable_without_gpu():
    from phast_b200 import _lib
    lib = _lib.load()
    assert lib.phastb_version().startswith(b"phastb")
    assert lib.phastb_reduce_workspace_bytes() > 0
    assert lib.phastb_q4_damage_solve_workspace_bytes(100) > 800
    g = _lib.VoxelGrid(4, 4, 4, 1, 1, 1, 0.25, 0.25, 0.25)
    assert lib.phastb_h8_scratch_bytes(g, _lib.F64) >= 24 * 8 * 64


def test_bad_arguments_rejected_without_gpu():
    from phast_b200 import _lib
    lib = _lib.load()
    g = _lib.Q4Grid(0, 3, 1.0, 1.0)  # nx = 0 is invalid
    assert lib.phastb_q4_strain(g, 0, None, None, None, None, None) == _lib.ERR_ARG

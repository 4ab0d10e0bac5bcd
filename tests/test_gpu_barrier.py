"""The bounded grid barrier of the persistent damage CG (needs a B200).

The persistent kernel's blocks meet at a grid-wide barrier twice per CG
iteration; a wait that never ends must not hang the GPU.  The library's
self-test launches a small cooperative grid in which one block never arrives:
the others must give up after the stated limit of GPU time, set the error
flag and return, and the entry point must report PHASTB_ERR_CUDA -- the status
the damage solve turns into an error.  The same launch with every block
arriving passes both barriers.
"""
import ctypes as C
import time

import pytest

pytestmark = pytest.mark.gpu


def _run(blocks, skip, limit_s):
    from phast_b200 import _lib
    err, passed = C.c_int(-1), C.c_int(-1)
    t0 = time.perf_counter()
    st = _lib.load().phastb_test_grid_barrier(blocks, skip, limit_s, C.byref(err), C.byref(passed))
    return st, err.value, passed.value, time.perf_counter() - t0


def test_barrier_passes_when_every_block_arrives():
    from phast_b200 import _lib
    st, err, passed, _ = _run(8, -1, 0.5)
    assert st == _lib.OK and err == 0 and passed == 8


def test_barrier_wait_runs_out_and_reports_an_error():
    from phast_b200 import _lib
    st, err, passed, secs = _run(8, 3, 0.05)
    assert st == _lib.ERR_CUDA and err == 1 and passed == 0
    assert secs < 5.0
    # the context stays usable afterwards
    st2, err2, passed2, _ = _run(4, -1, 0.5)
    assert st2 == _lib.OK and err2 == 0 and passed2 == 4

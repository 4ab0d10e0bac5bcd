"""CPU oracle for the phase-field hot path (TEST INFRASTRUCTURE ONLY).

This package is a numpy restatement of PhAST's matrix-free hot path, written
from the reference's published behaviour.  Every function cites the file and
line of ``src/phast/...`` it follows.  It exists to check the CUDA path:

* ``tests/`` compare the CUDA kernels (through the C-ABI) with it;
* ``__graft_entry__.smoke()`` checks one small launch against it;
* ``bench.py`` times it as the ``cpu_baseline`` / ``--impl reference`` leg.

Nothing in ``phast_b200`` imports, calls or links anything here.  The oracle is
pinned against the reference itself: ``tests/golden/make_golden.py`` imported
the reference implementation (with stub modules for its I/O-only
dependencies) and wrote the fixtures in ``tests/golden/*.npz``;
``tests/test_oracle_golden.py`` checks this package against them.
"""

"""The recursive half-step cutback of ``StaggeredSolver.advance_increment`` (CPU, no kernels).

``advance`` is replaced by a stand-in that fails whenever the step it is asked
to take is longer than a threshold, so the recursion of
solid3d/staggered.py:1523-1582 can be followed exactly: the interval is halved
until the pieces converge or ``max_cutbacks`` is reached, accepted sub-steps are
reported in order, and a failure past the limit carries the last accepted state
and the sub-steps accepted so far.
"""
import pytest
import torch

from phast_b200.solid3d import IncrementRecord, SolverConfig, SolverState, StaggerConvergenceError, StaggeredSolver


def _solver(max_step, **cfg_kw):
    s = object.__new__(StaggeredSolver)
    s.cfg = SolverConfig(device="cpu", **cfg_kw)
    s._c = 2
    s.last_state = None
    calls = []

    def advance(state, target, *, increment=None, cutbacks=0):
        begin = float(state.macro_strain[2])
        calls.append((round(begin, 12), round(target, 12), cutbacks))
        if abs(target - begin) > max_step + 1e-15:
            raise StaggerConvergenceError("failed", state=state, target=target, increment=increment,
                                          cutbacks=cutbacks, reason="staggered iteration did not converge")
        strain = state.macro_strain.clone()
        strain[2] = target
        new = SolverState(state.step + 1, state.x, state.d, state.H, strain, state.macro_stress, 0.0, state.d,
                          state.increment)
        return new, IncrementRecord(step=new.step, increment=increment, cutbacks=cutbacks)

    s.advance = advance
    return s, calls


def _start():
    z = torch.zeros(1)
    return SolverState(0, z, z, z, torch.zeros(6, dtype=torch.float64), torch.zeros(6, dtype=torch.float64), 0.0, z, 0)


def test_full_increment_needs_no_cutback():
    s, calls = _solver(1.0)
    state, recs = s.advance_increment(_start(), 0.8)
    assert calls == [(0.0, 0.8, 0)] and [r.cutbacks for r in recs] == [0]
    assert state.increment == 1 and float(state.macro_strain[2]) == 0.8


def test_two_levels_of_halving_in_order():
    s, calls = _solver(0.25, max_cutbacks=2)
    seen = []
    state, recs = s.advance_increment(_start(), 0.8, on_increment=lambda st, r: seen.append(r.step))
    # 0.8 fails -> [0, 0.4] fails -> [0, 0.2], [0.2, 0.4] ok -> [0.4, 0.8] fails -> [0.4, 0.6], [0.6, 0.8] ok
    assert calls == [(0.0, 0.8, 0), (0.0, 0.4, 1), (0.0, 0.2, 2), (0.2, 0.4, 2), (0.4, 0.8, 1), (0.4, 0.6, 2),
                     (0.6, 0.8, 2)]
    assert [r.cutbacks for r in recs] == [2, 2, 2, 2] and seen == [1, 2, 3, 4]
    assert state.increment == 1 and state.step == 4 and float(state.macro_strain[2]) == pytest.approx(0.8)
    assert s.last_state is state


def test_failure_past_the_limit_carries_the_accepted_substeps():
    s, calls = _solver(0.25, max_cutbacks=1)
    with pytest.raises(StaggerConvergenceError) as info:
        s.advance_increment(_start(), 0.8)
    exc = info.value
    assert calls == [(0.0, 0.8, 0), (0.0, 0.4, 1)]
    assert exc.cutbacks == 1 and exc.attempts == 2 and exc.records == ()
    assert float(exc.state.macro_strain[2]) == 0.0 and exc.target == pytest.approx(0.4)


def test_raise_mode_never_cuts_back():
    s, calls = _solver(0.25, on_stagger_failure="raise", max_cutbacks=3)
    with pytest.raises(StaggerConvergenceError) as info:
        s.advance_increment(_start(), 0.8)
    assert calls == [(0.0, 0.8, 0)] and info.value.attempts == 1

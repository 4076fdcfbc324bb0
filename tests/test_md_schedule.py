"""The molecular-dynamics schedules (hmc.schedule) against the call sequences of
the reference's own integrate_om / integrate_lp (hmc.py:104-162), recorded from the
unmodified reference in tests/golden/md_schedules.json (make_golden.py
--case md_schedules): the same kicks (level, weight) and drifts (weight) in the
same order, with a closing kick that reuses the previous force summed into it."""
import json
import os

import pytest

from tests.conftest import GOLDEN
from tfleonardym_b200 import hmc


def _cases():
    with open(os.path.join(GOLDEN, "md_schedules.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("key", sorted(_cases()))
def test_schedule_matches_reference_call_sequence(key):
    fn, steps, dt = key.split("/")
    steps = [int(k) for k in steps.split("_")]
    scheme = {"integrate_om": "omelyan", "integrate_lp": "leapfrog"}[fn]
    ops = hmc.schedule(scheme, steps, float(dt))
    want = _cases()[key]
    assert len(ops) == len(want), (len(ops), len(want))
    for op, (kind, level, weight) in zip(ops, want):
        assert ("drift" if op.kind == hmc.DRIFT else "kick") == kind
        if kind == "kick":
            assert op.level == level
        assert abs(op.weight - weight) <= 1e-15 * max(1.0, abs(weight)), (op, weight)


def test_force_evaluations_per_level():
    # Omelyan: 1 + 2 n_l evaluations per call of level l, level l called 2 n_{l-1} times per call above
    ops = hmc.schedule("omelyan", [4, 3], 1.0)
    assert hmc.force_evaluations(ops) == {0: 1 + 2 * 4, 1: 2 * 4 * (1 + 2 * 3)}
    ops = hmc.schedule("leapfrog", [2, 3, 2], 1.0)
    assert hmc.force_evaluations(ops) == {0: 1 + 2, 1: 2 * (1 + 3), 2: 2 * 3 * (1 + 2)}


def test_schedule_is_time_reversible():
    """Forward then backward: the backward schedule is the forward one reversed with
    negated weights (the integrator is symmetric), so the composition is the identity
    in exact arithmetic."""
    fwd = hmc.schedule("omelyan", [3, 2], 1.0)
    bwd = hmc.schedule("omelyan", [3, 2], -1.0)
    assert len(fwd) == len(bwd)
    for a, b in zip(fwd, reversed(bwd)):
        assert a.kind == b.kind and a.level == b.level
        assert abs(a.weight + b.weight) < 1e-16

"""Warm-start bookkeeping for sequences of systems (host logic)."""

import numpy as np
import pytest

from polysolve_b200.sequence import WarmStart


def test_warm_start_modes():
    for mode in ("zero", "previous", "extrapolate"):
        ws = WarmStart(mode)
        assert ws.guess(3) is None
        ws.record(np.array([1.0, 2.0, 3.0]))
        g1 = ws.guess(3)
        ws.record(np.array([2.0, 3.0, 5.0]))
        g2 = ws.guess(3)
        if mode == "zero":
            assert g1 is None and g2 is None
        elif mode == "previous":
            np.testing.assert_array_equal(g1, [1.0, 2.0, 3.0])
            np.testing.assert_array_equal(g2, [2.0, 3.0, 5.0])
        else:
            np.testing.assert_array_equal(g1, [1.0, 2.0, 3.0])
            np.testing.assert_array_equal(g2, [3.0, 4.0, 7.0])


def test_warm_start_keeps_two_and_copies():
    ws = WarmStart("extrapolate")
    x = np.zeros(2)
    for k in range(5):
        x[:] = k
        ws.record(x)
    np.testing.assert_array_equal(ws.guess(2), [5.0, 5.0])
    ws.reset()
    assert ws.guess(2) is None
    with pytest.raises(ValueError):
        WarmStart("quadratic")
    learned = WarmStart("learned")  # the solver makes the guess itself
    learned.record(x)
    assert learned.guess(2) is None

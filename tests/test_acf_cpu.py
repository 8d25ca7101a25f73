"""The multiple-tau stress autocorrelator restatement (oracle), pinned on the
reference's own correlator tests (tests/test_correlator.cu:7-79) and on the
lag and count pattern its update implies (analysis/correlator.cu:33-92)."""
import math

import numpy as np

from oracle.pyoracle import StressACF


def test_constant_signal_is_one_at_every_lag():
    # test_correlator.cu:7-39: 64 pushes of (1, 0, 0, 0, 0, 0); every level-0
    # lag averages to 1.
    acf = StressACF(freq=1)
    for _ in range(64):
        acf.push([1.0, 0, 0, 0, 0, 0])
    lag, val, cnt = acf.rows()
    lvl0 = lag <= 16
    assert np.all(np.abs(val[lvl0, 0] - 1.0) < 1e-12)
    assert np.all(val[:, 1:] == 0.0)


def test_decaying_signal_decays():
    # test_correlator.cu:41-79: exp(-i / 10) for 256 samples; C(lag 0) > C(lag 1).
    acf = StressACF(freq=1)
    for i in range(256):
        acf.push([math.exp(-i / 10.0), 0, 0, 0, 0, 0])
    lag, val, cnt = acf.rows()
    assert val[0, 0] > val[1, 0]


def test_lag_and_count_pattern():
    # The insert position bounds the lags: after N = 16 m level-0 pushes lag k
    # holds m (16 - k) products; level 1 receives N / 16 block averages.
    acf = StressACF(freq=5)
    for i in range(64):
        acf.push([1.0, -1.0, 0.5, 2.0, 0.0, 3.0])
    lag, val, cnt = acf.rows()
    assert list(lag[:16]) == [5 * (k + 1) for k in range(16)]
    assert list(cnt[:16]) == [4 * (16 - k) for k in range(16)]
    # level 1: 4 samples -> lags 0..3 with counts 4, 3, 2, 1, lags 80, 160, ...
    assert list(lag[16:20]) == [80, 160, 240, 320]
    assert list(cnt[16:20]) == [4, 3, 2, 1]
    assert len(lag) == 20
    assert np.allclose(val[:, :], np.array([1.0, 1.0, 0.25, 4.0, 0.0, 9.0]))


def test_alternating_signal():
    acf = StressACF(freq=1)
    for i in range(32):
        acf.push([(-1.0) ** i] * 6)
    lag, val, cnt = acf.rows()
    for k in range(16):
        assert val[k, 0] == (-1.0) ** k
    # block averages of 16 alternating samples are 0
    assert np.all(val[16:, :] == 0.0)

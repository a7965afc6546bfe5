"""The device gamma tail Q(a, x) against 40-digit mpmath and scipy (B200).

Every gamma-approximation p-value (dcc.gamma, hsic.gamma) is Q(shape, x)
with shape = mean^2 / variance and x = statistic / scale.  On the 500 x 50
level batch the shapes lie in 2.6..6.4 and x / shape in 0.27..92; the grid
below covers shape 0.5..50 and x / shape 0.01..200.

Tolerance: relative max(1e-14, 4e-16 |ln Q|).  The second term is the
conditioning of Q itself: Q = exp(E) * (a sum near 1) with |E| ~ |ln Q|, and
E rounded to double moves Q by |E| * 2^-53 relative.  For every Q above
1.4e-11 the bound is 1e-14 relative.
"""
import math

import numpy as np
import pytest

import fastkpc_b200 as fk

pytestmark = pytest.mark.gpu


def _tol(q):
    return q * max(1e-14, 4e-16 * abs(math.log(q)))


def _grid():
    A = np.geomspace(0.5, 50.0, 40)
    R = np.geomspace(0.01, 200.0, 40)
    a = np.repeat(A, len(R))
    x = a * np.tile(R, len(A))
    # the series / continued-fraction switch at x = a + 1, integer shapes
    # (the fraction terminates) and x = 0
    extra_a = np.array([0.5, 1.0, 2.0, 3.0, 4.5, 7.0, 12.0, 30.0, 3.0, 3.0, 5.0, 5.0, 0.7])
    extra_x = np.array([1.5, 2.0, 3.0, 4.0, 5.5, 8.0, 13.0, 31.0, 4.0 - 1e-12, 4.0 + 1e-12, 0.0, 1e-300, 1e-8])
    return np.concatenate([a, extra_a]), np.concatenate([x, extra_x])


@pytest.fixture(scope="module")
def truth():
    mp = pytest.importorskip("mpmath")
    mp.mp.dps = 40
    a, x = _grid()
    q = np.array([float(mp.gammainc(ai, xi, mp.inf, regularized=True)) for ai, xi in zip(a, x)])
    return a, x, q


def test_gamma_tail_matches_mpmath(lib_built, truth):
    a, x, ref = truth
    q, ok = fk.gamma_q(a, x)
    assert ok.all()
    worst = 0.0
    for k in range(len(a)):
        if ref[k] < 1e-300:
            assert q[k] <= 1e-290
            continue
        err = abs(q[k] - ref[k])
        assert err <= _tol(ref[k]), (a[k], x[k], q[k], ref[k])
        worst = max(worst, err / ref[k])
    assert worst > 0.0  # the comparison ran on real values


def test_gamma_tail_matches_scipy_on_the_batch_range(lib_built):
    from scipy.special import gammaincc
    a = np.repeat(np.linspace(2.0, 8.0, 31), 31)
    x = a * np.tile(np.geomspace(0.2, 100.0, 31), 31)
    q, ok = fk.gamma_q(a, x)
    ref = gammaincc(a, x)
    assert ok.all()
    keep = ref > 1e-11
    assert np.all(np.abs(q[keep] - ref[keep]) <= 1e-14 * ref[keep])
    # the grid covers p-values around the decision level (alpha = 0.1)
    band = (ref > 0.01) & (ref < 0.5)
    assert band.sum() > 50


def test_gamma_tail_edges(lib_built):
    q, ok = fk.gamma_q([2.0, 1.0, 1e3, 1e4], [0.0, 3.0, 1e3, 1.02e4])
    assert ok.all()
    assert q[0] == 1.0
    assert abs(q[1] - math.exp(-3.0)) <= 4e-15 * math.exp(-3.0)  # Q(1, x) = e^-x
    from scipy.special import gammaincc
    assert abs(q[2] - gammaincc(1e3, 1e3)) <= 1e-12 * q[2]
    assert abs(q[3] - gammaincc(1e4, 1.02e4)) <= 1e-11 * q[3]
    # invalid shapes are reported, not evaluated
    q, ok = fk.gamma_q([0.0, -1.0, float("nan")], [1.0, 1.0, 1.0])
    assert not ok.any() and np.isnan(q).all()

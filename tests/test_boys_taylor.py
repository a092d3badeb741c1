"""The Boys-function scheme of the device RI integrals (molgw_b200/csrc/ri_ints.cu),
restated in NumPy and checked against high-precision values (mpmath):

* below T = 40: a table of F_m(T_i) at T_i = 0, 0.1, ..., 40 and the eight-term
  Taylor expansion F_m(T) = sum_k F_{m+k}(T_i) (T_i - T)^k / k! about the nearest
  point (|T_i - T| <= 0.05);
* from T = 40: F_0 = sqrt(pi/T)/2 and the upward recursion
  F_{m+1} = ((2m+1) F_m - e^-T) / (2T).

Both hold to a few ulps for m <= 12 (the highest order of three g shells), which
is what lets the device integrals match the oracle's to 1e-12."""
import math

import numpy as np
import pytest

mpmath = pytest.importorskip("mpmath")
mpmath.mp.dps = 40


def boys_exact(m, t):
    if t == 0.0:
        return mpmath.mpf(1) / (2 * m + 1)
    t = mpmath.mpf(t)
    return mpmath.gammainc(m + mpmath.mpf("0.5"), 0, t) / (2 * t ** (m + mpmath.mpf("0.5")))


@pytest.fixture(scope="module")
def table():
    rows, orders = 401, 20
    tab = np.empty((rows, orders))
    for i in range(rows):
        t = i * 0.1   # the double the device forms
        for m in range(orders):
            tab[i, m] = float(boys_exact(m, t))
    return tab


def taylor(tab, m, t):
    i = int(round(t * 10.0))
    d = i * 0.1 - t
    v = tab[i, m + 7]
    for k in range(7, 0, -1):
        v = tab[i, m + k - 1] + v * d / k
    return v


def upward(mmax, t):
    e, f, out = math.exp(-t), 0.5 * math.sqrt(math.pi / t), []
    for k in range(mmax + 1):
        out.append(f)
        f = ((2 * k + 1) * f - e) / (2.0 * t)
    return out


def test_taylor_below_40(table):
    rng = np.random.default_rng(7)
    ts = np.concatenate([rng.uniform(0.0, 40.0, 300), [0.0, 1e-12, 0.05, 0.049999, 39.96, 20.05]])
    worst = 0.0
    for t in ts:
        t = float(min(t, 39.999))
        for m in range(13):
            ref = float(boys_exact(m, t))
            worst = max(worst, abs(taylor(table, m, t) - ref) / ref)
    assert worst < 4e-15, worst


def test_upward_recursion_from_40():
    worst = 0.0
    for t in [40.0, 41.3, 55.0, 120.0, 1e3, 1e5]:
        vals = upward(12, t)
        for m in range(13):
            ref = float(boys_exact(m, t))
            worst = max(worst, abs(vals[m] - ref) / ref)
    assert worst < 4e-15, worst

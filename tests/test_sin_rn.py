"""The sine of the device Lanczos2/3 weights (sin_rn.cuh), evaluated on the host
through viprs_sin_rn (the same source).

viprs's InterpolationKernel (kernel.rs:133-214) calls the platform sin (glibc).
The device's sin is rounded to nearest; these tests pin it against exact
values (decimal Taylor series at 60 digits) and against glibc on the Lanczos
argument range: equal to glibc except where glibc itself is off by more than
half an ulp, which happens for about 0.1% of the arguments.
"""
import ctypes
import math
from decimal import Decimal, getcontext

import numpy as np
import pytest

from viprs_b200 import _native as N


def sin_rn(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(x)
    assert N.lib().viprs_sin_rn(x.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p),
                                x.size) == 0
    return out


def exact_sin(x):
    getcontext().prec = 60
    x = Decimal(float(x))
    term = s = x
    n = 1
    while abs(term) > Decimal(10) ** -58:
        term = -term * x * x / ((n + 1) * (n + 2))
        n += 2
        s += term
    return s


def ulp_err(got, x):
    """|got - sin(x)| in ulps of got."""
    e = abs(Decimal(float(got)) - exact_sin(x))
    return float(e / Decimal(math.ulp(got)))


def lanczos_args(n, seed):
    rng = np.random.default_rng(seed)
    p = math.pi * rng.uniform(0.0, 3.0, n)
    return np.concatenate([p, p / 2.0, p / 3.0])


def test_special_values():
    x = np.array([0.0, -0.0, 1e-300, 1e-9, math.pi, math.pi / 2, 2 * math.pi, 3 * math.pi, -math.pi, 0.5, 1.0])
    got = sin_rn(x)
    assert got[0] == 0.0 and math.copysign(1.0, got[1]) == -1.0
    assert got[2] == 1e-300 and got[3] == math.sin(1e-9)
    assert got[4] == 1.2246467991473532e-16
    assert got[5] == 1.0
    for xi, gi in zip(x[4:], got[4:]):
        assert ulp_err(gi, xi) <= 0.5


def test_rounded_to_nearest_sample():
    x = lanczos_args(300, 11)
    got = sin_rn(x)
    worst = max(ulp_err(g, xi) for g, xi in zip(got, x))
    assert worst <= 0.5 + 1e-9


def test_agrees_with_glibc_except_its_misroundings():
    x = lanczos_args(400_000, 12)
    got = sin_rn(x)
    ref = np.array([math.sin(v) for v in x])  # glibc's sin, as viprs calls it
    diff = got != ref
    assert diff.mean() < 3e-3
    # every disagreement is one ulp, and there this sine is the nearer one
    d = np.abs(got[diff] - ref[diff]) / np.array([math.ulp(v) for v in got[diff]])
    assert np.all(d <= 1.0)
    idx = np.flatnonzero(diff)[:40]
    for i in idx:
        assert ulp_err(got[i], x[i]) < 0.5 + 1e-9 < ulp_err(ref[i], x[i])


@pytest.mark.parametrize("k", range(4))
def test_near_multiples_of_half_pi(k):
    x = k * math.pi / 2 + np.linspace(-1e-6, 1e-6, 2001)
    x = x[x >= 0]
    got = sin_rn(x)
    for i in range(0, x.size, 97):
        assert ulp_err(got[i], x[i]) <= 0.5 + 1e-9

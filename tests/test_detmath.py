"""Deterministic elementary functions (felis_b200/csrc/detmath.h), host build.

The GPU path and the CPU restatement both evaluate these; their accuracy is
checked here against the C library (<= 2 ulp on the ranges the slice loop
uses).  Bit equality of the device build with the host build is part of the
GPU parity tests (whole-loop bit equality depends on it).
"""
import math

import numpy as np
import pytest


def ulp_err(a: float, b: float) -> float:
    if a == b:
        return 0.0
    return abs(a - b) / math.ulp(b if b != 0 else 1e-300)


@pytest.mark.parametrize("lo,hi", [(-math.pi / 4, math.pi / 4), (-8.0, 8.0), (0.0, 2 * math.pi), (-200.0, 200.0)])
def test_sincos_accuracy(fb, lo, hi):
    rng = np.random.default_rng(1)
    worst = 0.0
    for x in rng.uniform(lo, hi, 20000):
        s, c = fb.detmath_sincos(float(x))
        # absolute error in ulps of 1 (the functions are evaluated near |1|)
        worst = max(worst, abs(s - math.sin(x)) / math.ulp(1.0), abs(c - math.cos(x)) / math.ulp(1.0))
    assert worst <= 2.0, worst


def test_sincos_relative_small_args(fb):
    for x in [1e-300, 1e-20, 1e-8, 1e-3, 0.1, 0.5, 0.78, -0.3]:
        s, c = fb.detmath_sincos(x)
        assert ulp_err(s, math.sin(x)) <= 2.0
        assert ulp_err(c, math.cos(x)) <= 2.0


def test_sincos_symmetry_and_zero(fb):
    assert fb.detmath_sincos(0.0) == (0.0, 1.0)
    for x in np.linspace(0.01, 50, 500):
        s1, c1 = fb.detmath_sincos(float(x))
        s2, c2 = fb.detmath_sincos(float(-x))
        assert s2 == -s1 and c2 == c1


def test_atan_accuracy(fb):
    rng = np.random.default_rng(2)
    xs = np.concatenate([rng.uniform(-1, 1, 20000), rng.uniform(-50, 50, 5000), 10 ** rng.uniform(-12, 12, 5000)])
    worst = max(ulp_err(fb.detmath_atan(float(x)), math.atan(x)) for x in xs)
    assert worst <= 2.0, worst
    assert fb.detmath_atan(0.0) == 0.0
    assert abs(fb.detmath_atan(1e308) - math.pi / 2) <= math.ulp(math.pi / 2)
    assert math.isnan(fb.detmath_atan(float("nan")))


def test_atan2_accuracy(fb):
    rng = np.random.default_rng(3)
    worst = 0.0
    for y, x in rng.normal(size=(20000, 2)):
        worst = max(worst, ulp_err(fb.detmath_atan2(float(y), float(x)), math.atan2(y, x)))
    assert worst <= 2.5, worst
    for y, x in [(0.0, 1.0), (0.0, -1.0), (1.0, 0.0), (-1.0, 0.0), (-0.0, -1.0)]:
        assert fb.detmath_atan2(y, x) == math.atan2(y, x)

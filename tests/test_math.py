"""Accuracy of the deterministic elementary functions of include/ice_math.h, which the device's
plain form and the oracle both compute with, against the platform library (numpy / glibc)."""
import numpy as np
import pytest


def ulps(a, b):
    a = np.asarray(a, dtype=np.float64); b = np.asarray(b, dtype=np.float64)
    sp = np.spacing(np.maximum(np.abs(b), np.finfo(float).tiny))
    return np.abs(a - b) / sp


def vec(orc, fn, x, y=None):
    y = np.zeros_like(x) if y is None else y
    return np.array([orc.math(fn, float(a), float(b)) for a, b in zip(x, y)])


def test_exp(orc):
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.uniform(-700, 700, 4000), rng.uniform(-1, 1, 4000), rng.uniform(-1e-8, 1e-8, 500)])
    assert ulps(vec(orc, 0, x), np.exp(x)).max() <= 3
    assert orc.math(0, 0.0, 0) == 1.0 and orc.math(0, 800.0, 0) == np.inf and orc.math(0, -800.0, 0) == 0.0


def test_log(orc):
    rng = np.random.default_rng(2)
    x = np.concatenate([10 ** rng.uniform(-300, 300, 4000), rng.uniform(0.5, 2.0, 4000), [1.0, 2.0, 1e-310, 5e-324]])
    assert ulps(vec(orc, 1, x), np.log(x)).max() <= 3
    assert orc.math(1, 1.0, 0) == 0.0 and np.isnan(orc.math(1, -1.0, 0)) and orc.math(1, 0.0, 0) == -np.inf


def test_log10(orc):
    rng = np.random.default_rng(3)
    x = 10 ** rng.uniform(-30, 30, 3000)
    assert ulps(vec(orc, 5, x), np.log10(x)).max() <= 4


def test_pow_ranges_of_the_correlations(orc):
    rng = np.random.default_rng(4)
    # Reynolds, Prandtl, Schmidt, Mach numbers and temperatures to the exponents the sources use
    x = np.concatenate([10 ** rng.uniform(-6, 5, 3000), rng.uniform(200, 2000, 2000)])
    for y in (0.687, 1.0 / 3.0, 0.6, 0.55, 0.15, 0.33, 0.7, 4.63, 0.88, -1.16, 2.0 / 3.0, 0.5, 4.0, 8.0, 3.0, -1.0):
        got = vec(orc, 2, x, np.full_like(x, y))
        ref = np.power(x, y)
        bound = max(4.0, 2.0 * float(np.max(np.abs(y * np.log(x)))))
        assert ulps(got, ref).max() <= bound, y


def test_pow_special(orc):
    assert orc.math(2, -2.0, 3.0) == -8.0 and orc.math(2, -2.0, 2.0) == 4.0
    assert np.isnan(orc.math(2, -2.0, 0.5))
    assert orc.math(2, 0.0, 2.0) == 0.0 and orc.math(2, 0.0, -1.0) == np.inf
    assert orc.math(2, 5.0, 0.0) == 1.0 and orc.math(2, 9.0, 0.5) == 3.0


def test_tanh_and_expm1(orc):
    rng = np.random.default_rng(5)
    x = np.concatenate([rng.uniform(-25, 25, 3000), rng.uniform(-1e-3, 1e-3, 2000), rng.uniform(-1, 1, 2000)])
    assert ulps(vec(orc, 3, x), np.tanh(x)).max() <= 4
    assert ulps(vec(orc, 4, x), np.expm1(x)).max() <= 4

"""Accuracy of the shared FP64 elementary functions (b2e_math.h) against
high-precision values, through the oracle build that exports them."""
import math

import numpy as np
import pytest

from reforacle import PortOracle

mp = pytest.importorskip("mpmath")
mp.mp.prec = 200


def ulp_error(got, exact):
    ex = float(exact)
    return float(abs(mp.mpf(got) - exact) / math.ulp(ex)) if ex != 0 else 0.0


@pytest.mark.parametrize("fn,lo,hi,bound", [
    ("sin", -0.8, 0.8, 1.0), ("cos", -0.8, 0.8, 1.0), ("sin", -1e6, 1e6, 1.5), ("cos", -50.0, 50.0, 1.5),
    ("asin", -0.125, 0.125, 0.6), ("asin", -0.5, 0.5, 0.7), ("asin", -1.0, 1.0, 2.5), ("tan", -0.7, 0.7, 2.0),
    ("sin", -0.0625, 0.0625, 0.6), ("cos", -0.0625, 0.0625, 0.6), ("asin", -0.015625, 0.015625, 0.6),
    ("sin", 0.0625, 0.07, 0.6), ("cos", 0.0625, 0.07, 0.6), ("asin", 0.015625, 0.02, 0.6)])
def test_ulp_error(fn, lo, hi, bound):
    o = PortOracle("b2e")
    f = getattr(o.lib, f"b2e_oracle_{fn}")
    ref = {"sin": mp.sin, "cos": mp.cos, "asin": mp.asin, "tan": mp.tan}[fn]
    rng = np.random.default_rng(1)
    worst = 0.0
    for x in rng.uniform(lo, hi, 3000):
        worst = max(worst, ulp_error(f(float(x)), ref(mp.mpf(float(x)))))
    assert worst <= bound


def test_symmetry_and_special_values():
    o = PortOracle("b2e").lib
    for x in (1e-300, 1e-8, 0.3, 2.0, 1234.5):
        assert o.b2e_oracle_sin(-x) == -o.b2e_oracle_sin(x)
        assert o.b2e_oracle_cos(-x) == o.b2e_oracle_cos(x)
        assert o.b2e_oracle_asin(-min(x, 1.0)) == -o.b2e_oracle_asin(min(x, 1.0))
    assert o.b2e_oracle_sin(0.0) == 0.0 and o.b2e_oracle_cos(0.0) == 1.0 and o.b2e_oracle_tan(0.0) == 0.0
    assert math.isnan(o.b2e_oracle_asin(1.5)) and math.isnan(o.b2e_oracle_sin(float("nan")))


@pytest.mark.parametrize("lo,hi", [(1e-3, 10.0), (0.5, 2.0), (1e-300, 1e300), (0.99, 1.01)])
def test_log_ulp_error(lo, hi):
    o = PortOracle("b2e")
    import ctypes
    f = o.lib.b2e_oracle_log
    f.restype, f.argtypes = ctypes.c_double, [ctypes.c_double]
    rng = np.random.default_rng(7)
    xs = np.exp(rng.uniform(np.log(lo), np.log(hi), 3000))
    worst = max(ulp_error(f(float(x)), mp.log(mp.mpf(float(x)))) for x in xs)
    assert worst <= 0.75, worst
    assert f(1.0) == 0.0 and math.isinf(f(0.0)) and math.isnan(f(-1.0))


@pytest.mark.parametrize("y", [1.0 / 3.0, 2.0 / 3.0, 4.0 / 3.0, 2.0])
def test_pow_exponents_ulp_error(y):
    """pow for the exponents the CSR code evaluates per bin, against the
    exact value of x to the double nearest p/3 (not p/3 itself)."""
    o = PortOracle("b2e")
    import ctypes
    f = o.lib.b2e_oracle_pow
    f.restype, f.argtypes = ctypes.c_double, [ctypes.c_double, ctypes.c_double]
    rng = np.random.default_rng(8)
    xs = np.exp(rng.uniform(np.log(1e-12), np.log(1e6), 3000))
    worst = max(ulp_error(f(float(x), y), mp.power(mp.mpf(float(x)), mp.mpf(y))) for x in xs)
    assert worst <= 0.51, worst

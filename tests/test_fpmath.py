"""The exp and pow that the engine and the oracle share (pdac_b200/csrc/
fpmath.h): within about one unit in the last place of the C library's over
the ranges the per-step physics uses, and the IEEE special cases."""
import ctypes as C
import math

import numpy as np
import pytest

import pyoracle


def _fns():
    L = pyoracle.lib()
    L.pdac_oracle_fp_pow.argtypes = [C.c_double, C.c_double]
    L.pdac_oracle_fp_pow.restype = C.c_double
    L.pdac_oracle_fp_exp.argtypes = [C.c_double]
    L.pdac_oracle_fp_exp.restype = C.c_double
    return L.pdac_oracle_fp_pow, L.pdac_oracle_fp_exp


def _ulps(a, b):
    return abs(a - b) / math.ulp(b) if b != 0 else abs(a)


def test_exp_is_within_one_ulp():
    _, fexp = _fns()
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(-700, 700, 20000), rng.uniform(-3, 3, 20000), rng.uniform(-1e-3, 1e-3, 2000),
                         [0.0, 1.0, -1.0, 709.7, -708.0, 1e-300, -1e-300]])
    worst = max(_ulps(fexp(float(x)), math.exp(float(x))) for x in xs)
    assert worst <= 1.0, worst
    assert fexp(0.0) == 1.0
    assert fexp(800.0) == math.inf and fexp(-800.0) == 0.0
    assert math.isnan(fexp(math.nan))


@pytest.mark.parametrize("lo,hi,ys", [
    (1e-9, 1.0, [-2.65, 4.14, 1.28, 2.65]),          # void-fraction powers of the drag laws (drag.f)
    (1e-3, 1e6, [0.687, 0.2, 0.7, 1.0 / 3.0]),      # Reynolds and Prandtl powers (drag.f, hvs.f)
    (0.3, 300.0, [-0.14874, -0.25]),                 # viscosity collision integral (visc.f)
    (10.0, 10.0, np.linspace(-40.0, 5.0, 301)),      # 10**(...) of the particle repulsion and turbo.f
])
def test_pow_is_within_one_ulp(lo, hi, ys):
    fpow, _ = _fns()
    rng = np.random.default_rng(1)
    xs = np.exp(rng.uniform(math.log(lo), math.log(hi), 3000)) if hi > lo else np.array([lo])
    worst = 0.0
    for y in ys:
        for x in xs:
            worst = max(worst, _ulps(fpow(float(x), float(y)), math.pow(float(x), float(y))))
    assert worst <= 1.0, worst


def test_pow_special_cases():
    fpow, _ = _fns()
    assert fpow(0.0, 0.687) == 0.0
    assert fpow(0.0, -1.0) == math.inf
    assert fpow(5.0, 0.0) == 1.0 and fpow(1.0, 123.4) == 1.0
    assert math.isnan(fpow(-2.0, 0.5))
    assert fpow(-2.0, 3.0) == -8.0 and fpow(-2.0, 2.0) == 4.0
    assert fpow(math.inf, 2.0) == math.inf and fpow(math.inf, -2.0) == 0.0
    assert math.isnan(fpow(math.nan, 2.0))

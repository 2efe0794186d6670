"""Accuracy of plibm.h (the kernels' exp/pow) against the system libm."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hostemu")


@pytest.fixture(scope="module")
def shim():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    L = ctypes.CDLL(os.path.join(HERE, "libplibm_shim.so"))
    L.plibm_check.restype = ctypes.c_double
    L.plibm_check.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long,
                              ctypes.c_void_p, ctypes.c_void_p]
    return L


def _worst(L, mode, x, y=None):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(x if y is None else y, dtype=np.float64)
    p = np.empty_like(x)
    q = np.empty_like(x)
    w = L.plibm_check(mode, x.ctypes.data, y.ctypes.data, len(x), p.ctypes.data, q.ctypes.data)
    return w, p, q


RNG = np.random.default_rng(0)
N = 400_000


@pytest.mark.parametrize("lo,hi", [(-50, 50), (-745, 709), (-1e-6, 1e-6), (-0.35, 0.35)])
def test_exp_within_one_ulp(shim, lo, hi):
    w, _, _ = _worst(shim, 0, RNG.uniform(lo, hi, N))
    assert w <= 1.0


@pytest.mark.parametrize("xr,yr", [((-20, 6), (-4, 4)), ((-300, 300), (-1, 1)), ((-12, -2), (0.3, 0.7))])
def test_pow_within_two_ulp(shim, xr, yr):
    x = 10.0 ** RNG.uniform(*xr, N)
    y = RNG.uniform(*yr, N)
    w, _, _ = _worst(shim, 1, x, y)
    assert w <= 2.0


def test_pow_constant_exponents_of_cloudsc(shim):
    """The exponents CLOUDSC uses with bases in their physical ranges."""
    cases = [(0.4, (0.3, 3.0)), (0.5555555555555556, (1e-12, 1e-2)), (0.67, (0.0, 2e-3)),
             (1.5, (0.7, 1.2)), (3.0, (150.0, 320.0)), (0.666, (1e-14, 1e-2)), (0.5777, (0.0, 1.0)),
             (-1.79, (50.0, 300.0)), (1.47, (1e-10, 1e-2)), (0.15, (1e-10, 1e-2)), (1.15, (1e-10, 1e-2))]
    for y, (a, b) in cases:
        x = RNG.uniform(a, b, N)
        w, _, _ = _worst(shim, 1, x, np.full(N, y))
        assert w <= 2.0, (y, w)


def test_special_values(shim):
    x = np.array([0.0, 0.0, 0.0, 1.0, np.inf, np.inf, 2.0, np.nan])
    y = np.array([2.0, -1.0, 0.0, 3.7, 1.0, -1.0, 0.0, 1.0])
    _, p, q = _worst(shim, 1, x, y)
    assert p[0] == 0.0 and p[1] == np.inf and p[2] == 1.0 and p[3] == 1.0
    assert p[4] == np.inf and p[5] == 0.0 and p[6] == 1.0 and np.isnan(p[7])
    _, e, _ = _worst(shim, 0, np.array([0.0, 800.0, -800.0, np.nan, -np.inf, np.inf]))
    assert e[0] == 1.0 and e[1] == np.inf and e[2] == 0.0 and np.isnan(e[3])
    assert e[4] == 0.0 and e[5] == np.inf

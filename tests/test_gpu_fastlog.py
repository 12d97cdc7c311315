"""The device logarithm of the ACDI distance function (fastlog.cuh) against numpy.log.

psi = eps log((min(phi,1)+1e-16)/(1-min(phi,1)+1e-16)) (multi/main.f90:527-528) takes
arguments from ~1e-16 to ~1e16; the table-driven log must stay within 2 ulp there and over the
whole normal range, and keep log(0) = -inf, log(x<0) = NaN, log(NaN) = NaN, log(inf) = inf.
"""
import ctypes

import numpy as np
import pytest

from mhit36_mixedp_b200 import _lib

pytestmark = pytest.mark.gpu


def dev_log(x):
    lib = _lib.load()
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    p = ctypes.POINTER(ctypes.c_double)
    assert lib.mhit_debug_fastlog(x.ctypes.data_as(p), y.ctypes.data_as(p), x.size) == 0
    return y


def test_fastlog_accuracy(gpu):
    rng = np.random.default_rng(7)
    x = np.concatenate([
        10.0 ** rng.uniform(-300, 300, 200000),
        10.0 ** rng.uniform(-17, 17, 400000),
        1.0 + rng.uniform(-1e-3, 1e-3, 100000),          # near 1: result near 0
        rng.uniform(0.70, 1.42, 100000),                  # the reduced range itself
        np.array([1.0, 2.0, 0.5, np.sqrt(2.0), np.sqrt(0.5), 1e-16, 1e16, 2.0 ** -1022, np.finfo(float).max]),
    ])
    y = dev_log(x)
    ref = np.log(x)
    ulp = np.spacing(np.abs(ref))
    err_ulp = np.abs(y - ref) / np.maximum(ulp, np.finfo(float).tiny)
    assert np.max(err_ulp) <= 2.0, float(np.max(err_ulp))


def test_fastlog_special_values(gpu):
    x = np.array([0.0, -0.0, -1.0, -1e-300, np.nan, np.inf, 5e-324, 1e-310])
    y = dev_log(x)
    assert y[0] == -np.inf and y[1] == -np.inf
    assert np.isnan(y[2]) and np.isnan(y[3]) and np.isnan(y[4])
    assert y[5] == np.inf
    np.testing.assert_allclose(y[6:], np.log(x[6:]), rtol=1e-15)

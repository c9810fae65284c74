"""The reciprocal ("fast") form's arithmetic (csrc/cdm_fast.cuh) beside CUDA's
correctly rounded square root and division, through cdm_selftest_fastmath:

* sqrt_nr — the hardware approximation of 1/sqrt(x), two Newton-Raphson steps,
  Markstein's final correction — within one ulp of sqrt(x) over normal
  arguments from 1e-300 to 1e300, and equal to sqrt(x) on 0, -0, subnormals,
  inf, NaN and negative arguments (which take the IEEE square root);
* rcp_nr — the hardware reciprocal approximation, two Newton-Raphson steps —
  within one ulp of 1/x where 1/x is a normal number, and 1/(+-0) = +-inf,
  1/(+-inf) = +-0, NaN for NaN.
"""
import ctypes as C

import numpy as np
import pytest

from curvilineardiffusionmanuscript_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _probe(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty(4 * len(x), dtype=np.float64)
    dp = C.POINTER(C.c_double)
    rc = L.load().cdm_selftest_fastmath(0, x.ctypes.data_as(dp), len(x), out.ctypes.data_as(dp))
    assert rc == L.CDM_OK, L.last_error()
    return out.reshape(-1, 4)


def _ulps(got, ref):
    return np.abs(got - ref) / np.spacing(np.abs(ref))


def test_newton_square_root_within_one_ulp():
    rng = np.random.default_rng(5)
    x = np.concatenate([10.0 ** rng.uniform(-300.0, 300.0, 200000), rng.uniform(0.5, 2.0, 100000),
                        rng.uniform(1.0, 1e4, 100000), 1.0 + np.arange(1, 2001) * 2.0 ** -52,
                        [2.2250738585072014e-308, 1.7976931348623157e308, 1.0, 2.0, 4.0, np.pi ** 2]])
    r = _probe(x)
    err = _ulps(r[:, 0], r[:, 1])
    assert err.max() <= 1.0, (err.max(), x[np.argmax(err)])
    # most results are the correctly rounded ones
    assert np.mean(r[:, 0] == r[:, 1]) > 0.9


def test_newton_reciprocal_within_one_ulp():
    rng = np.random.default_rng(6)
    mag = 10.0 ** rng.uniform(-300.0, 300.0, 200000)
    x = np.concatenate([mag * np.where(rng.random(len(mag)) < 0.5, -1.0, 1.0), rng.uniform(0.5, 2.0, 100000),
                        [1.0, -1.0, 3.0, 0.1, 1e-300, 1e300]])
    r = _probe(x)
    err = _ulps(r[:, 2], r[:, 3])
    assert err.max() <= 1.0, (err.max(), x[np.argmax(err)])


def test_special_arguments_match_ieee():
    x = np.array([0.0, -0.0, 5e-324, 1e-310, np.inf, -np.inf, -1.0, -4.0, np.nan])
    r = _probe(x)
    # square root: the IEEE result, signed zeros included
    assert np.array_equal(r[:, 0].view(np.int64)[~np.isnan(r[:, 1])], r[:, 1].view(np.int64)[~np.isnan(r[:, 1])])
    assert np.array_equal(np.isnan(r[:, 0]), np.isnan(r[:, 1]))
    # reciprocal of zeros, infinities and NaN
    rz = _probe(np.array([0.0, -0.0, np.inf, -np.inf, np.nan]))
    assert rz[0, 2] == np.inf and rz[1, 2] == -np.inf
    assert rz[2, 2] == 0.0 and not np.signbit(rz[2, 2]) and rz[3, 2] == 0.0 and np.signbit(rz[3, 2])
    assert np.isnan(rz[4, 2])


def test_rejects_bad_arguments():
    out = np.empty(4)
    dp = C.POINTER(C.c_double)
    assert L.load().cdm_selftest_fastmath(0, None, 1, out.ctypes.data_as(dp)) == L.CDM_BAD_INPUT
    x = np.ones(1)
    assert L.load().cdm_selftest_fastmath(0, x.ctypes.data_as(dp), 0, out.ctypes.data_as(dp)) == L.CDM_BAD_INPUT

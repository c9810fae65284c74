"""The reciprocal ("fast") form's Newton-refined reciprocals (csrc/cdm_fast.cuh)
beside CUDA's correctly rounded division, through cdm_selftest_fastmath:

* rcp_nr — the hardware reciprocal approximation, two Newton-Raphson steps,
  the approximation's own result kept for 0 and inf — within one ulp of 1/x
  where 1/x is a normal number, 1/(+-0) = +-inf, 1/(+-inf) = +-0, NaN for NaN;
* rcp_pos — the same refinement without those fix-ups, used for arguments known
  to be positive, finite and normal — within one ulp of 1/x there.
"""
import ctypes as C

import numpy as np
import pytest

from curvilineardiffusionmanuscript_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _probe(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty(3 * len(x), dtype=np.float64)
    dp = C.POINTER(C.c_double)
    rc = L.load().cdm_selftest_fastmath(0, x.ctypes.data_as(dp), len(x), out.ctypes.data_as(dp))
    assert rc == L.CDM_OK, L.last_error()
    return out.reshape(-1, 3)


def _ulps(got, ref):
    return np.abs(got - ref) / np.spacing(np.abs(ref))


def test_newton_reciprocals_within_one_ulp():
    rng = np.random.default_rng(6)
    mag = 10.0 ** rng.uniform(-300.0, 300.0, 200000)
    pos = np.concatenate([mag, rng.uniform(0.5, 2.0, 100000), 1.0 + np.arange(1, 2001) * 2.0 ** -52,
                          [1.0, 3.0, 0.1, 1e-300, 1e300, np.pi]])
    sign = np.where(rng.random(len(pos)) < 0.5, -1.0, 1.0)
    r = _probe(pos * sign)
    err = _ulps(r[:, 0], r[:, 2])
    assert err.max() <= 1.0, (err.max(), (pos * sign)[np.argmax(err)])
    assert np.mean(r[:, 0] == r[:, 2]) > 0.9  # mostly the correctly rounded result
    rp = _probe(pos)
    err = _ulps(rp[:, 1], rp[:, 2])
    assert err.max() <= 1.0, (err.max(), pos[np.argmax(err)])


def test_special_arguments_of_the_general_reciprocal():
    r = _probe(np.array([0.0, -0.0, np.inf, -np.inf, np.nan]))
    assert r[0, 0] == np.inf and r[1, 0] == -np.inf
    assert r[2, 0] == 0.0 and not np.signbit(r[2, 0]) and r[3, 0] == 0.0 and np.signbit(r[3, 0])
    assert np.isnan(r[4, 0])


def test_rejects_bad_arguments():
    out = np.empty(3)
    dp = C.POINTER(C.c_double)
    assert L.load().cdm_selftest_fastmath(0, None, 1, out.ctypes.data_as(dp)) == L.CDM_BAD_INPUT
    x = np.ones(1)
    assert L.load().cdm_selftest_fastmath(0, x.ctypes.data_as(dp), 0, out.ctypes.data_as(dp)) == L.CDM_BAD_INPUT

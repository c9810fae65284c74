"""Twilight-zone path of the oracle (define_forcing_wavy, twilight_zone.jl:54-195).

* The forcing's exp and sinpi (a Cody–Waite/Taylor exp and an exactly reduced
  Taylor sinpi, the methods the CUDA library also evaluates) stay within 2 ulp
  of the correctly rounded values (mpmath at 200 bits).
* Known answer: the reference verifies its solver by this manufactured
  solution (wavy_manufactured_solution/run.jl).  With the forcing the exact
  solution exp(−(x² + y²)) is steady (no_t), so one implicit step from it
  measures the truncation error, which must fall as h² on the reference's grid.
"""
import math

import mpmath
import numpy as np
import pytest
import torch

from oracle.oracle import OracleSolver, exp_cw, sinpi
from curvilineardiffusionmanuscript_b200 import problems
from curvilineardiffusionmanuscript_b200.solver import NeumannBC

mpmath.mp.prec = 200


def ulp_err(got, exact):
    e = float(exact)
    if e == 0.0:
        return 0.0 if got == 0.0 else math.inf
    return abs(float(mpmath.mpf(got) - exact)) / math.ulp(abs(e))


def test_exp_within_two_ulp():
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(-745.0, 709.0, 1500), rng.uniform(-1.0, 1.0, 1500),
                         rng.uniform(-80.0, 0.0, 1500), [0.0, -0.0, 1.0, -1.0, 0.5 * math.log(2.0), 700.0]])
    worst = max(ulp_err(exp_cw(x), mpmath.exp(mpmath.mpf(x))) for x in xs)
    assert worst <= 2.0, worst
    assert exp_cw(1000.0) == math.inf and exp_cw(-1000.0) == 0.0 and math.isnan(exp_cw(math.nan))


def test_sinpi_within_two_ulp():
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.uniform(-1.0, 1.0, 2000), rng.uniform(-100.0, 100.0, 2000),
                         np.arange(-8, 8) + 0.25, np.arange(-8, 8) + 1e-9, [0.5, -0.5, 1.5, 1e-300]])
    worst = max(ulp_err(sinpi(x), mpmath.sinpi(mpmath.mpf(x))) for x in xs)
    assert worst <= 2.0, worst
    assert sinpi(3.0) == 0.0 and sinpi(0.5) == 1.0 and math.isnan(sinpi(math.inf))


def _truncation_error(n, dt=1e-3):
    pr = problems.tz_wavy_2d(n)
    m = pr.mesh
    o = OracleSolver(m, pr.bcs)
    o.set_source(pr.source)
    o.set_twilight_zone(*m.centroids, *m.cell_fwd, m.nnodes)
    T = pr.T0.numpy().copy()
    st, _ = o.step(T, pr.rho.numpy(), pr.cp, pr.kappa.k0, pr.kappa.n, dt, tz=True, no_t=True, rtol=1e-9, atol=0.0,
                   max_iter=200000)
    assert st["status"] == 0
    d = m.domain()
    return float(np.abs(T[d] - pr.T0.numpy()[d]).max()) / dt


def test_manufactured_solution_is_second_order_on_the_reference_grid():
    e = [_truncation_error(n) for n in (96, 192, 384)]
    orders = [math.log2(e[k] / e[k + 1]) for k in range(2)]
    assert orders[0] > 1.6 and 1.8 < orders[1] < 2.3, (e, orders)


def test_time_dependent_forcing_tracks_the_decay():
    """no_t = false: the exact solution decays as e^{−4t}; a few steps from it
    stay within the grid's truncation error of the exact values."""
    pr = problems.tz_wavy_2d(96)
    m = pr.mesh
    o = OracleSolver(m, pr.bcs)
    o.set_source(pr.source)
    o.set_twilight_zone(*m.centroids, *m.cell_fwd, m.nnodes)
    T = pr.T0.numpy().copy()
    t, dt = 0.0, 1e-4
    for _ in range(5):
        st, _ = o.step(T, pr.rho.numpy(), pr.cp, 1.0, 2.5, dt, t=t, tz=True, no_t=False, rtol=1e-9, atol=0.0,
                       max_iter=200000)
        assert st["status"] == 0
        t += dt
    x, y = m.centroids
    exact = problems.tz_exact(x, y, t).numpy()
    d = m.domain()
    assert np.abs(T[d] - exact[d]).max() < 1e-3
    # without the forcing the same steps leave the exact solution much further behind
    o2 = OracleSolver(m, pr.bcs)
    o2.set_source(pr.source)
    T2 = pr.T0.numpy().copy()
    for _ in range(5):
        o2.step(T2, pr.rho.numpy(), pr.cp, 1.0, 2.5, dt, rtol=1e-9, atol=0.0, max_iter=200000)
    assert np.abs(T2[d] - exact[d]).max() > 10 * np.abs(T[d] - exact[d]).max()


def test_forcing_is_rejected_without_inputs_or_in_3d():
    pr = problems.tz_wavy_2d(16)
    o = OracleSolver(pr.mesh, pr.bcs)
    st, _ = o.step(pr.T0.numpy().copy(), pr.rho.numpy(), 1.0, 1.0, 2.5, 1e-5, tz=True)
    assert st["status"] == 3

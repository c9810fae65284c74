"""Twilight-zone forcing on the GPU (tz = true of step!, update.jl:23-71,
residuals.jl:49-99) through the C ABI, against the oracle's literal
restatement of define_forcing_wavy (twilight_zone.jl:54-195).

The library evaluates the forcing's α-independent terms once per step and adds
α inside the operation-for-operation kernel in the reference's order, with the
same exp/sinpi methods as the oracle: fields, iteration counts and next_dt are
bit-identical, for both FP64 precisions (a tz step runs the exact kernel).
"""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle.oracle import OracleSolver
from curvilineardiffusionmanuscript_b200 import _lib as L
from curvilineardiffusionmanuscript_b200 import problems
from curvilineardiffusionmanuscript_b200.solver import (APTError, PseudoTransientBatch, PseudoTransientSolver,
                                                        step)
from helpers import small_case_3d

pytestmark = pytest.mark.gpu

KW = dict(rtol=1e-9, atol=1e-12, max_iter=50000)


def _oracle(pr):
    o = OracleSolver(pr.mesh, pr.bcs)
    o.set_source(pr.source)
    o.set_twilight_zone(*pr.mesh.centroids, *pr.mesh.cell_fwd, pr.mesh.nnodes)
    return o


@pytest.mark.parametrize("precision", ["fp64_exact", "fp64"])
@pytest.mark.parametrize("no_t", [False, True])
def test_forcing_bit_identical_to_the_oracle(precision, no_t):
    pr = problems.tz_wavy_2d(48)
    o = _oracle(pr)
    g = PseudoTransientSolver(pr.mesh, pr.bcs, precision=precision)
    g.set_source(pr.source)
    g.set_twilight_zone()
    To = pr.T0.numpy().copy()
    Tg = pr.T0.clone().cuda()
    rho = pr.rho.cuda()
    t, dt = 0.0, 2e-4
    for s in range(3):
        so, ndo = o.step(To, pr.rho.numpy(), pr.cp, 1.0, 2.5, dt, t=t, tz=True, no_t=no_t, **KW)
        sg, ndg = step(g, pr.mesh, Tg, rho, pr.cp, pr.kappa, dt, t=t, tz=True, tz_dim=2, no_t=no_t, **KW)
        assert so["status"] == 0 and sg["niter"] == so["niter"], (s, so["niter"], sg["niter"])
        assert np.array_equal(Tg.cpu().numpy(), To), (s, np.abs(Tg.cpu().numpy() - To).max())
        assert abs(ndg - ndo) <= 1e-14 * abs(ndo)
        assert abs(sg["abs_err"] - so["abs_err"]) <= 1e-12 * abs(so["abs_err"])
        t += dt


def test_forcing_on_host_arrays_and_without_it_afterwards():
    """tz is a per-step switch: a step without it after tz steps is the plain step."""
    pr = problems.tz_wavy_2d(40)
    o = _oracle(pr)
    g = PseudoTransientSolver(pr.mesh, pr.bcs, precision="fp64_exact")
    g.set_source(pr.source.numpy())
    g.set_twilight_zone()
    To, Tg = pr.T0.numpy().copy(), pr.T0.numpy().copy()
    for tz in (True, False, True):
        so, _ = o.step(To, pr.rho.numpy(), pr.cp, 1.0, 2.5, 1e-4, t=1e-4, tz=tz, no_t=False, **KW)
        sg, _ = step(g, pr.mesh, Tg, pr.rho.numpy(), pr.cp, pr.kappa, 1e-4, t=1e-4, tz=tz, no_t=False, **KW)
        assert sg["niter"] == so["niter"] and np.array_equal(Tg, To), tz


def test_batch_with_forcing_restores_the_tuned_schedule():
    """A batch tuned to the wavefront schedule runs a tz step on the exact
    kernel (bit-identical to the oracle) and returns to its tuning after it."""
    prs = [problems.tz_wavy_2d(n) for n in (32, 56)]
    b = PseudoTransientBatch([p.mesh for p in prs], [p.bcs for p in prs], precision="fp64")
    for i, p in enumerate(prs):
        b.set_source(i, p.source.cuda())
        b.set_twilight_zone(i)
    b.set_tuning(4, 16, 8)
    Ts = [p.T0.clone().cuda() for p in prs]
    args = ([p.rho.cuda() for p in prs], [1.0] * 2, [p.kappa for p in prs], [2e-4] * 2)
    st, _ = b.step(Ts, *args, t=0.0, tz=True, no_t=False, **KW)
    assert b.tuning() == {"variant": 4, "strip_h": 16, "iter_block": 8}
    for i, p in enumerate(prs):
        o = _oracle(p)
        T = p.T0.numpy().copy()
        so, _ = o.step(T, p.rho.numpy(), 1.0, 1.0, 2.5, 2e-4, t=0.0, tz=True, no_t=False, **KW)
        assert so["niter"] == st[i]["niter"] and np.array_equal(Ts[i].cpu().numpy(), T), i
    b.close()


def test_forcing_error_paths():
    pr = problems.tz_wavy_2d(24)
    g = PseudoTransientSolver(pr.mesh, pr.bcs)
    with pytest.raises(APTError) as ei:  # no mesh inputs given
        step(g, pr.mesh, pr.T0.clone().cuda(), pr.rho.cuda(), 1.0, pr.kappa, 1e-5, tz=True)
    assert ei.value.status == L.CDM_BAD_INPUT and "set_twilight_zone" in str(ei.value)
    gm = PseudoTransientSolver(pr.mesh, pr.bcs, precision="mixed")
    gm.set_twilight_zone()
    with pytest.raises(APTError) as ei:
        step(gm, pr.mesh, pr.T0.clone().cuda(), pr.rho.cuda(), 1.0, pr.kappa, 1e-5, tz=True)
    assert ei.value.status == L.CDM_BAD_INPUT and "FP64" in str(ei.value)
    # the forcing is two-dimensional: a 3D handle refuses its inputs
    p3 = small_case_3d()
    g3 = PseudoTransientSolver(p3.mesh, p3.bcs)
    z = torch.zeros(8, dtype=torch.float64, device="cuda")
    d = L.TzDesc()
    d.mem = L.CDM_MEM_DEVICE
    d.nnodes[0] = d.nnodes[1] = 9
    d.x = d.y = d.x_xi = d.x_eta = d.y_xi = d.y_eta = z.data_ptr()
    assert L.load().cdm_apt_set_twilight_zone(g3._h, C.byref(d)) == L.CDM_BAD_INPUT

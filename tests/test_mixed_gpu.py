"""GPU tests of the mixed-precision path: FP32 correction sweeps with FP64
residual and defect-correction restarts.

The FP32 path solves the same discrete equations to the same stopping rule, so
its solution differs from the FP64 oracle's by the stopping tolerance, not by
FP32 rounding: the stated bound is a relative L2 difference ≤ 1e-6 on the full
array at rel ≤ 1e-8, and the manufactured-solution error equals the FP64 one.
"""
import math

import numpy as np
import pytest
import torch

from helpers import rel_l2, small_case_2d
from oracle.oracle import OracleSolver
from curvilineardiffusionmanuscript_b200 import problems
from curvilineardiffusionmanuscript_b200.solver import (APTError, DirichletBC, NeumannBC, PeriodicBC,
                                                        PseudoTransientSolver, step)

pytestmark = pytest.mark.gpu
KW = dict(rtol=1e-8, atol=1e-8, max_iter=100000)


def run_mixed_vs_oracle(pr, nsteps, src=None, mean="harmonic"):
    o = OracleSolver(pr.mesh, pr.bcs, mean=mean)
    g = PseudoTransientSolver(pr.mesh, pr.bcs, precision="mixed", mean=mean)
    To = pr.T0.numpy().copy()
    Tg = pr.T0.clone().cuda()
    rho = pr.rho.cuda()
    t = 0.0
    out = []
    for _ in range(nsteps):
        if src is not None:
            S = src(t + pr.dt)
            o.set_source(S.numpy())
            g.set_source(S.cuda())
        so, _ = o.step(To, pr.rho.numpy(), pr.cp, pr.kappa.k0, pr.kappa.n, pr.dt, **KW)
        sg, _ = step(g, pr.mesh, Tg, rho, pr.cp, pr.kappa, pr.dt, **KW)
        t += pr.dt
        out.append((so, sg, To.copy(), Tg.cpu().numpy()))
    return out


def test_mixed_gaussian_128():
    for so, sg, To, Tg in run_mixed_vs_oracle(problems.gaussian_2d(128), 4):
        assert so["status"] == 0 and sg["status"] == 0
        assert sg["rel_err"] <= 1e-8 or sg["abs_err"] <= 1e-8
        assert sg["n_restarts"] >= 2
        assert rel_l2(Tg, To) <= 1e-6, rel_l2(Tg, To)


def test_mixed_mms_error_matches_fp64():
    pr = problems.mms_2d(256)
    out = run_mixed_vs_oracle(pr, 3, src=lambda t: problems.mms_source(pr, t))
    so, sg, To, Tg = out[-1]
    e_o = problems.mms_error(pr, torch.from_numpy(To), 3 * pr.dt)
    e_g = problems.mms_error(pr, torch.from_numpy(Tg), 3 * pr.dt)
    assert abs(e_g[0] - e_o[0]) <= 1e-6 * e_o[0] and abs(e_g[1] - e_o[1]) <= 1e-6 * e_o[1]
    assert rel_l2(Tg, To) <= 1e-8


@pytest.mark.parametrize("bcs", [[DirichletBC(1.5), NeumannBC(), PeriodicBC(), PeriodicBC()],
                                 [NeumannBC(), NeumannBC(), DirichletBC(0.5), NeumannBC()]])
def test_mixed_boundary_conditions(bcs):
    pr = small_case_2d(ni=150, nj=140, bcs=bcs, source=True)
    for so, sg, To, Tg in run_mixed_vs_oracle(pr, 2):
        assert so["status"] == 0 and sg["status"] == 0
        assert rel_l2(Tg, To) <= 1e-6


def test_mixed_arithmetic_mean():
    pr = small_case_2d(ni=120, nj=100, kn=2.5)
    for so, sg, To, Tg in run_mixed_vs_oracle(pr, 2, mean="arithmetic"):
        assert sg["status"] == 0 and rel_l2(Tg, To) <= 1e-6


def test_mixed_state_carries_into_fp64():
    """The damped-flux state written by the mixed path continues the FP64 iteration."""
    pr = problems.gaussian_2d(96)
    g = PseudoTransientSolver(pr.mesh, pr.bcs, precision="mixed")
    T = pr.T0.clone().cuda()
    step(g, pr.mesh, T, pr.rho.cuda(), pr.cp, pr.kappa, pr.dt, **KW)
    q, last = g.get_state()
    assert np.isfinite(q).all() and np.abs(q).max() > 0 and last > 0


def test_mixed_rejects_batches():
    """The mixed path runs single problems (2D or 3D); a batch asks for FP64."""
    from curvilineardiffusionmanuscript_b200.mesh import wavy_mesh_2d
    from curvilineardiffusionmanuscript_b200.solver import PseudoTransientBatch
    ms = [wavy_mesh_2d(16, 16), wavy_mesh_2d(24, 24)]
    with pytest.raises(APTError):
        PseudoTransientBatch(ms, [[NeumannBC()] * 4] * 2, precision="mixed")


# ----------------------------------------------------------------------- 3D
def test_mixed_3d_gaussian_matches_oracle():
    """3D FP32 plane-marching sweeps with FP64 3D restarts against the oracle."""
    from helpers import small_case_3d
    for so, sg, To, Tg in run_mixed_vs_oracle(small_case_3d(n=(20, 18, 16)), 3):
        assert so["status"] == 0 and sg["status"] == 0
        assert sg["n_restarts"] >= 2
        assert rel_l2(Tg, To) <= 1e-6, rel_l2(Tg, To)


@pytest.mark.parametrize("mean", ["harmonic", "arithmetic"])
def test_mixed_3d_boundary_conditions(mean):
    from helpers import small_case_3d
    from curvilineardiffusionmanuscript_b200.solver import FixedNegSymmetryBC
    pr = small_case_3d(n=(14, 11, 13), bcs=[DirichletBC(1.0), NeumannBC(), PeriodicBC(), PeriodicBC(),
                                             FixedNegSymmetryBC(), DirichletBC(3.0)])
    for so, sg, To, Tg in run_mixed_vs_oracle(pr, 2, mean=mean):
        assert so["status"] == 0 and sg["status"] == 0
        assert rel_l2(Tg, To) <= 1e-6, rel_l2(Tg, To)


def test_mixed_and_fp64_agree_on_large_3d_grid():
    """Several column tiles, k-strips and restart tiles (70 x 45 x 37)."""
    from helpers import small_case_3d
    pr = small_case_3d(n=(70, 45, 37))
    gm = PseudoTransientSolver(pr.mesh, pr.bcs, precision="mixed")
    gf = PseudoTransientSolver(pr.mesh, pr.bcs, precision="fp64")
    Tm, Tf = pr.T0.clone().cuda(), pr.T0.clone().cuda()
    rho = pr.rho.cuda()
    for _ in range(2):
        sm, _ = step(gm, pr.mesh, Tm, rho, pr.cp, pr.kappa, pr.dt, **KW)
        sf, _ = step(gf, pr.mesh, Tf, rho, pr.cp, pr.kappa, pr.dt, **KW)
        assert sm["status"] == 0 and sm["n_restarts"] >= 2
        assert rel_l2(Tm.cpu().numpy(), Tf.cpu().numpy()) <= 1e-6

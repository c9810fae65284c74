"""GPU parity: the CUDA APT path (through the C ABI) against the CPU oracle.

Bar (FP64 path): relative L2 difference ≤ 1e-10 and identical iteration
counts on the same seeded inputs.

* precision "fp64_exact" keeps the reference's operation order and contracts
  no multiply-add: the expected difference is exactly zero, and it is asserted;
* precision "fp64" (the default, reciprocal form) differs in the last bits:
  the 1e-10 bar and equal iteration counts are asserted.
"""
import math

import numpy as np
import pytest
import torch

from helpers import decaying_mode_error, rel_l2, richardson_order, small_case_2d, small_case_3d
from oracle.oracle import OracleSolver
from curvilineardiffusionmanuscript_b200 import problems
from curvilineardiffusionmanuscript_b200.solver import (APTError, DirichletBC, FixedNegSymmetryBC, NeumannBC,
                                                        PeriodicBC, PowerLawConductivity, PseudoTransientBatch,
                                                        PseudoTransientSolver, step)

pytestmark = pytest.mark.gpu
TOL = 1e-10


def run_pair(pr, nsteps=None, mean="harmonic", device_arrays=False, precision="fp64_exact", **kw):
    kw.setdefault("rtol", 0.0)
    kw.setdefault("atol", 1e-8)
    kw.setdefault("max_iter", 50000)
    nsteps = nsteps or pr.nsteps
    o = OracleSolver(pr.mesh, pr.bcs, mean=mean)
    g = PseudoTransientSolver(pr.mesh, pr.bcs, mean=mean, precision=precision)
    if pr.source is not None:
        o.set_source(pr.source.numpy())
        g.set_source(pr.source.clone())
    To = pr.T0.numpy().copy()
    if device_arrays:
        Tg = pr.T0.clone().cuda()
        rho = pr.rho.cuda()
    else:
        Tg = pr.T0.numpy().copy()
        rho = pr.rho.numpy()
    out = []
    for s in range(nsteps):
        so, ndo = o.step(To, pr.rho.numpy(), pr.cp, pr.kappa.k0, pr.kappa.n, pr.dt, **kw)
        sg, ndg = step(g, pr.mesh, Tg, rho, pr.cp, pr.kappa, pr.dt, **kw)
        Tgh = Tg.cpu().numpy() if device_arrays else Tg
        out.append((so, sg, ndo, ndg, To.copy(), Tgh.copy()))
    return o, g, out


def assert_parity(out, exact=True):
    for s, (so, sg, ndo, ndg, To, Tg) in enumerate(out):
        assert so["status"] == 0 and sg["status"] == 0
        assert so["niter"] == sg["niter"], (s, so["niter"], sg["niter"])
        assert rel_l2(Tg, To) <= TOL, (s, rel_l2(Tg, To))
        assert abs(ndg - ndo) <= 1e-14 * abs(ndo), (s, ndo, ndg)
        # near convergence the residual is a difference of large terms, so its
        # last digits follow the rounding of the path (fast form: a few percent)
        assert abs(sg["abs_err"] - so["abs_err"]) <= (1e-12 if exact else 1e-3) * abs(so["abs_err"]) + 1e-300
        if exact:
            assert np.array_equal(Tg, To), (s, np.abs(Tg - To).max())


def test_metric_cache_matches_oracle():
    pr = small_case_2d(ni=40, nj=33, amp=0.07)
    o = OracleSolver(pr.mesh, pr.bcs)
    g = PseudoTransientSolver(pr.mesh, pr.bcs)
    co, cg = o.metric_cache(), g.metric_cache()
    assert np.array_equal(co[:, 1:-1, 1:-1], cg[:, 1:-1, 1:-1])
    pr3 = small_case_3d()
    assert np.array_equal(OracleSolver(pr3.mesh, pr3.bcs).metric_cache()[:, 1:-1, 1:-1, 1:-1],
                          PseudoTransientSolver(pr3.mesh, pr3.bcs).metric_cache()[:, 1:-1, 1:-1, 1:-1])


def test_neumann_2d_small():
    _, _, out = run_pair(small_case_2d())
    assert_parity(out)


def test_gaussian_128_ten_steps():
    """The 128² Gaussian-pulse configuration (κ = T³, 10 steps of 1e-5, tol 1e-8)."""
    _, _, out = run_pair(problems.gaussian_2d(128))
    assert_parity(out)


def test_device_pointers():
    _, _, out = run_pair(small_case_2d(ni=37, nj=21), device_arrays=True)
    assert_parity(out)


@pytest.mark.parametrize("bcs", [
    [DirichletBC(1.5), NeumannBC(), PeriodicBC(), PeriodicBC()],
    [PeriodicBC(), PeriodicBC(), NeumannBC(), DirichletBC(0.5)],
    [FixedNegSymmetryBC(), NeumannBC(), NeumannBC(), DirichletBC(2.0)],
    [NeumannBC(), PeriodicBC(), NeumannBC(), NeumannBC()],
])
def test_boundary_conditions(bcs):
    _, _, out = run_pair(small_case_2d(ni=29, nj=19, bcs=bcs, source=True), apply_cutoff=True)
    assert_parity(out)


def test_arithmetic_mean_no_subcycle():
    _, _, out = run_pair(small_case_2d(kn=2.5), mean="arithmetic", subcycle_conductivity=False)
    assert_parity(out)


@pytest.mark.parametrize("kn", [0.0, 1.0, 1.5, 2.5, 3.0])
def test_conductivity_exponents(kn):
    _, _, out = run_pair(small_case_2d(ni=20, nj=20, kn=kn), nsteps=2)
    assert_parity(out)


def test_conductivity_general_exponent():
    """Non-half-integer exponents go through pow(), whose CUDA and glibc results
    may differ in the last bit: the 1e-10 bar and equal iteration counts hold,
    bitwise equality is not expected."""
    _, _, out = run_pair(small_case_2d(ni=20, nj=20, kn=0.7), nsteps=2)
    assert_parity(out, exact=False)


def test_every_k_checks():
    _, _, out = run_pair(small_case_2d(), check_every=5)
    assert_parity(out)


def test_rms_norm():
    """The CPU reference norm sqrt(Σr²/N) (residuals.jl:8-22) sums in a different
    order on the GPU, so a residual within rounding of the tolerance can stop
    one check later: iteration counts agree within one check interval and the
    solutions within the stopping tolerance."""
    _, _, out = run_pair(small_case_2d(), norm_kind="rms", check_every=5, nsteps=1)
    so, sg, _, _, To, Tg = out[0]
    assert so["status"] == 0 and sg["status"] == 0
    assert abs(so["niter"] - sg["niter"]) <= 5
    if so["niter"] == sg["niter"]:
        assert rel_l2(Tg, To) <= TOL
    else:
        assert rel_l2(Tg, To) <= 1e-8


def test_reference_tolerances_defaults():
    """rtol = 1e-5, atol = √eps (step! defaults) with the adaptive schedule."""
    pr = small_case_2d()
    _, _, out = run_pair(pr, nsteps=4, rtol=1e-5, atol=2.220446049250313e-16 ** 0.5)
    assert_parity(out)


def test_multi_halo_dirichlet():
    pr = small_case_2d(ni=18, nj=14, nhalo=3, bcs=[DirichletBC(1.2), DirichletBC(0.8), NeumannBC(), NeumannBC()])
    _, _, out = run_pair(pr)
    assert_parity(out)


def test_3d_small():
    _, _, out = run_pair(small_case_3d())
    assert_parity(out)


def test_3d_mixed_bcs():
    pr = small_case_3d(n=(12, 7, 9), bcs=[DirichletBC(1.0), NeumannBC(), PeriodicBC(), PeriodicBC(),
                                          NeumannBC(), DirichletBC(3.0)])
    _, _, out = run_pair(pr)
    assert_parity(out)


def test_state_roundtrip_matches_oracle():
    pr = small_case_2d()
    o, g, out = run_pair(pr, nsteps=2)
    qo, lo = o.get_state()
    qg, lg = g.get_state()
    assert lo == lg
    assert np.array_equal(qo, qg)
    # restore a checkpoint into a fresh solver: the next step is identical
    g2 = PseudoTransientSolver(pr.mesh, pr.bcs, precision="fp64_exact")
    g2.set_state(qg, lg)
    T1, T2 = out[-1][5].copy(), out[-1][5].copy()
    s1, _ = step(g, pr.mesh, T1, pr.rho.numpy(), pr.cp, pr.kappa, pr.dt, rtol=0.0, atol=1e-8)
    s2, _ = step(g2, pr.mesh, T2, pr.rho.numpy(), pr.cp, pr.kappa, pr.dt, rtol=0.0, atol=1e-8)
    assert s1["niter"] == s2["niter"] and np.array_equal(T1, T2)


def test_error_paths_match_reference():
    pr = small_case_2d()
    g = PseudoTransientSolver(pr.mesh, pr.bcs)
    T = pr.T0.numpy().copy()
    with pytest.raises(APTError) as ei:
        step(g, pr.mesh, T, pr.rho.numpy(), pr.cp, pr.kappa, pr.dt, rtol=0.0, atol=1e-8, max_iter=3)
    assert ei.value.status == 1 and ei.value.stats["niter"] == 4
    T = pr.T0.numpy().copy()
    T[5, 5] = np.nan
    g2 = PseudoTransientSolver(pr.mesh, pr.bcs)
    with pytest.raises(APTError) as ei:
        step(g2, pr.mesh, T, pr.rho.numpy(), pr.cp, pr.kappa, pr.dt)
    assert ei.value.status == 2 and ei.value.stats["niter"] == 1
    g3 = PseudoTransientSolver(pr.mesh, pr.bcs)
    S = np.zeros(pr.mesh.full_shape)
    S[3, 3] = np.inf
    g3.set_source(S)
    with pytest.raises(APTError) as ei:
        step(g3, pr.mesh, pr.T0.numpy().copy(), pr.rho.numpy(), pr.cp, pr.kappa, pr.dt)
    assert ei.value.status == 3
    with pytest.raises(APTError):
        step(g, pr.mesh, pr.T0.numpy().copy(), pr.rho.numpy(), pr.cp, pr.kappa, -1.0)


def test_run_twice_bitwise_identical():
    pr = small_case_2d(ni=50, nj=45)
    outs = []
    for _ in range(2):
        g = PseudoTransientSolver(pr.mesh, pr.bcs, precision="fp64")
        T = pr.T0.numpy().copy()
        for _ in range(2):
            step(g, pr.mesh, T, pr.rho.numpy(), pr.cp, pr.kappa, pr.dt, rtol=0.0, atol=1e-8, norm_kind="rms")
        outs.append(T)
    assert np.array_equal(outs[0], outs[1])


def test_batch_matches_individual_oracle_runs():
    probs = problems.batch_2d(nprob=6, nmin=20, nmax=70, seed=7)
    b = PseudoTransientBatch([p.mesh for p in probs], [p.bcs for p in probs], precision="fp64_exact")
    Ts = [p.T0.numpy().copy() for p in probs]
    for _ in range(2):
        stats, ndts = b.step(Ts, [p.rho.numpy() for p in probs], [p.cp for p in probs],
                             [p.kappa for p in probs], [p.dt for p in probs], rtol=0.0, atol=1e-8, max_iter=50000)
    for p, pr in enumerate(probs):
        o = OracleSolver(pr.mesh, pr.bcs)
        T = pr.T0.numpy().copy()
        for _ in range(2):
            so, _ = o.step(T, pr.rho.numpy(), pr.cp, pr.kappa.k0, pr.kappa.n, pr.dt, rtol=0.0, atol=1e-8,
                           max_iter=50000)
        assert so["niter"] == stats[p]["niter"], p
        assert np.array_equal(T, Ts[p]), p


def test_batch_autotune_changes_speed_not_results(tmp_path):
    """The autotuner times every (strip height, iteration block) candidate on the
    given inputs without changing them or the solver state; after tuning the
    exact batch still equals the oracle bit for bit, and the choice is cached."""
    probs = problems.batch_2d(nprob=6, nmin=20, nmax=70, seed=7)
    b = PseudoTransientBatch([p.mesh for p in probs], [p.bcs for p in probs], precision="fp64_exact")
    Ts = [p.T0.numpy().copy() for p in probs]
    T0 = [t.copy() for t in Ts]
    args = ([p.rho.numpy() for p in probs], [p.cp for p in probs], [p.kappa for p in probs], [p.dt for p in probs])
    kw = dict(rtol=0.0, atol=1e-8, max_iter=50000)
    cache = str(tmp_path / "tune.json")
    c = b.autotune(Ts, *args, cache_path=cache, **kw)
    assert 0 <= c < 18
    assert all(np.array_equal(a, t) for a, t in zip(Ts, T0))
    tun = b.tuning()
    if c < 12:
        assert tun == {"variant": 0, "strip_h": [8, 16, 32, 64][c // 3], "iter_block": [4, 8, 16][c % 3]}
    else:
        assert tun["variant"] == 2 + (c - 12) // 3 and tun["iter_block"] == [4, 8, 16][c % 3]
    for _ in range(2):
        stats, _ = b.step(Ts, *args, **kw)
    for p, pr in enumerate(probs):
        o = OracleSolver(pr.mesh, pr.bcs)
        T = pr.T0.numpy().copy()
        for _ in range(2):
            so, _ = o.step(T, pr.rho.numpy(), pr.cp, pr.kappa.k0, pr.kappa.n, pr.dt, **kw)
        assert so["niter"] == stats[p]["niter"], p
        assert np.array_equal(T, Ts[p]), p
    # a second batch of the same sizes reads the cached choice
    b2 = PseudoTransientBatch([p.mesh for p in probs], [p.bcs for p in probs], precision="fp64_exact")
    assert b2.autotune([p.T0.numpy().copy() for p in probs], *args, cache_path=cache, **kw) == c
    assert b2.tuning() == tun


@pytest.mark.parametrize("tuning", [(0, 0, 8), (0, 8, 4), (2, 0, 16), (3, 0, 1)])
def test_every_2d_kernel_variant_matches_the_oracle(tuning):
    """Marching kernel at two strip heights and both tile kernels, exact form:
    bit-identical to the oracle whatever the tuning."""
    probs = problems.batch_2d(nprob=4, nmin=20, nmax=90, seed=11)
    b = PseudoTransientBatch([p.mesh for p in probs], [p.bcs for p in probs], precision="fp64_exact")
    b.set_tuning(*tuning)
    assert b.tuning() == dict(zip(("variant", "strip_h", "iter_block"), tuning))
    Ts = [p.T0.numpy().copy() for p in probs]
    stats, _ = b.step(Ts, [p.rho.numpy() for p in probs], [p.cp for p in probs], [p.kappa for p in probs],
                      [p.dt for p in probs], rtol=0.0, atol=1e-8, max_iter=50000)
    for p, pr in enumerate(probs):
        o = OracleSolver(pr.mesh, pr.bcs)
        T = pr.T0.numpy().copy()
        so, _ = o.step(T, pr.rho.numpy(), pr.cp, pr.kappa.k0, pr.kappa.n, pr.dt, rtol=0.0, atol=1e-8,
                       max_iter=50000)
        assert so["niter"] == stats[p]["niter"] and np.array_equal(T, Ts[p]), p


def test_fast_form_tile_variant_matches_the_oracle():
    probs = problems.batch_2d(nprob=3, nmin=30, nmax=80, seed=12)
    b = PseudoTransientBatch([p.mesh for p in probs], [p.bcs for p in probs], precision="fp64")
    b.set_tuning(2, 0, 8)
    Ts = [p.T0.clone().cuda() for p in probs]
    stats, _ = b.step(Ts, [p.rho.cuda() for p in probs], [p.cp for p in probs], [p.kappa for p in probs],
                      [p.dt for p in probs], rtol=1e-8, atol=1e-8, max_iter=50000)
    for p, pr in enumerate(probs):
        o = OracleSolver(pr.mesh, pr.bcs)
        T = pr.T0.numpy().copy()
        so, _ = o.step(T, pr.rho.numpy(), pr.cp, pr.kappa.k0, pr.kappa.n, pr.dt, rtol=1e-8, atol=1e-8,
                       max_iter=50000)
        assert so["niter"] == stats[p]["niter"] and rel_l2(Ts[p].cpu().numpy(), T) <= TOL, p


def _run_tunings(probs, tunings, nsteps=3, **kw):
    """Each tuning on a fresh batch from the same inputs: per-step iteration counts and final fields."""
    kw = dict(dict(rtol=1e-8, atol=1e-8, max_iter=50000), **kw)
    out = []
    for tun in tunings:
        b = PseudoTransientBatch([p.mesh for p in probs], [p.bcs for p in probs], precision="fp64")
        for i, pr in enumerate(probs):
            if pr.source is not None:
                b.set_source(i, pr.source.cuda())
        b.set_tuning(*tun)
        assert b.tuning() == dict(zip(("variant", "strip_h", "iter_block"), tun))
        Ts = [p.T0.clone().cuda() for p in probs]
        args = ([p.rho.cuda() for p in probs], [p.cp for p in probs], [p.kappa for p in probs],
                [p.dt for p in probs])
        its = []
        for _ in range(nsteps):
            st, _ = b.step(Ts, *args, **kw)
            its.append([x["niter"] for x in st])
        b.close()
        out.append((its, [t.cpu() for t in Ts]))
    return out


@pytest.mark.parametrize("K", [1, 7, 32])
def test_wavefront_schedule_equals_per_iteration_launches(K):
    """Variant 4 runs the same strips with the same arithmetic as one launch per
    pseudo-iteration; only strips of different problems' iterations overlap in
    time, so fields and iteration counts are identical bit for bit, also for
    problems that converge in the middle of a launch."""
    probs = problems.batch_2d(nprob=10, nmin=20, nmax=400, seed=21)
    (i0, T0), (i1, T1) = _run_tunings(probs, [(0, 32, 8), (4, 32, K)])
    assert len({n for step in i0 for n in step}) > 3  # problems stop at different iterations
    assert i0 == i1
    assert all(torch.equal(a, b) for a, b in zip(T0, T1))


@pytest.mark.parametrize("K", [8, 32])
def test_paced_wavefront_equals_unpaced(K, monkeypatch):
    """From the second step on, the wavefront schedule spreads each problem's
    expected remaining iterations over the launch's rounds (pacing); it only
    reorders iterations of independent problems, so fields and iteration counts
    equal those of the unpaced schedule (CDM_WAVE_PACE=0) bit for bit."""
    probs = problems.batch_2d(nprob=12, nmin=20, nmax=300, seed=5)
    (i1, T1), = _run_tunings(probs, [(5, 16, K)], nsteps=4)
    monkeypatch.setenv("CDM_WAVE_PACE", "0")
    (i0, T0), = _run_tunings(probs, [(5, 16, K)], nsteps=4)
    assert len({n for step in i0[1:] for n in step}) > 3
    assert i0 == i1
    assert all(torch.equal(a, b) for a, b in zip(T0, T1))


def test_wavefront_boundary_conditions_sources_and_one_problem():
    bcs = [[DirichletBC(1.5), NeumannBC(), PeriodicBC(), PeriodicBC()],
           [FixedNegSymmetryBC(), NeumannBC(), NeumannBC(), DirichletBC(2.0)],
           [NeumannBC(), PeriodicBC(), NeumannBC(), NeumannBC()]]
    probs = [small_case_2d(ni=29 + 97 * k, nj=19 + 61 * k, bcs=b, source=True, seed=k) for k, b in enumerate(bcs)]
    (i0, T0), (i1, T1) = _run_tunings(probs, [(0, 16, 4), (4, 16, 16)])
    assert i0 == i1 and all(torch.equal(a, b) for a, b in zip(T0, T1))
    one = [problems.gaussian_2d(300)]
    (i0, T0), (i1, T1) = _run_tunings(one, [(0, 8, 8), (4, 8, 8)], nsteps=2)
    assert i0 == i1 and torch.equal(T0[0], T1[0])


def test_wavefront_matches_the_oracle():
    probs = problems.batch_2d(nprob=3, nmin=30, nmax=140, seed=12)
    ((its, Ts),) = _run_tunings(probs, [(4, 16, 8)], nsteps=1)
    for p, pr in enumerate(probs):
        o = OracleSolver(pr.mesh, pr.bcs)
        T = pr.T0.numpy().copy()
        so, _ = o.step(T, pr.rho.numpy(), pr.cp, pr.kappa.k0, pr.kappa.n, pr.dt, rtol=1e-8, atol=1e-8,
                       max_iter=50000)
        assert so["niter"] == its[0][p] and rel_l2(Ts[p].numpy(), T) <= TOL, p


def test_fast_batch_autotune_includes_the_wavefront():
    probs = problems.batch_2d(nprob=5, nmin=20, nmax=200, seed=3)
    b = PseudoTransientBatch([p.mesh for p in probs], [p.bcs for p in probs], precision="fp64")
    Ts = [p.T0.clone().cuda() for p in probs]
    T0 = [t.clone() for t in Ts]
    args = ([p.rho.cuda() for p in probs], [p.cp for p in probs], [p.kappa for p in probs], [p.dt for p in probs])
    c = b.autotune(Ts, *args, rtol=1e-8, atol=1e-8, max_iter=50000)
    assert 0 <= c < 36 and all(torch.equal(a, t) for a, t in zip(Ts, T0))
    if c >= 18:
        t = c - 18
        assert b.tuning() == {"variant": 4 + t // 9, "strip_h": [16, 32, 64][(t % 9) // 3],
                              "iter_block": [16, 32, 64][t % 3]}
    b.close()


@pytest.mark.parametrize("K", [1, 16])
def test_narrow_wavefront_equals_per_iteration_launches(K):
    """Variant 5: the wavefront schedule with 64-thread blocks (62 owned columns)
    gives the fields and iteration counts of one launch per iteration, bit for bit."""
    probs = problems.batch_2d(nprob=10, nmin=20, nmax=300, seed=22)
    (i0, T0), (i1, T1) = _run_tunings(probs, [(1, 16, 8), (5, 16, K)])
    assert i0 == i1
    assert all(torch.equal(a, b) for a, b in zip(T0, T1))


@pytest.mark.parametrize("tuning", [(0, 8, 8), (4, 8, 8)])
def test_invalid_diffusivity_stops_the_next_step(tuning):
    """validate_scalar (PseudoTransientSolver.jl:238-250) checks the diffusivity the
    previous step's last iteration left, on the domain and the first halo layer.  A
    negative ρ in one ghost cell of a Neumann side gives that ghost a negative α
    without touching the iteration (its face has Δu = 0), so with enforce_positivity
    the first step runs as in the oracle and the second reports CDM_BAD_INPUT."""
    pr = small_case_2d(ni=40, nj=33, seed=5)
    nh = pr.mesh.nhalo
    rho = pr.rho.clone()
    rho[nh + 11, nh - 1] = -2.0 * rho[nh + 11, nh]  # ghost column of the i-low side, row 11
    b = PseudoTransientBatch([pr.mesh], [pr.bcs], precision="fp64")
    b.set_tuning(*tuning)
    T = pr.T0.clone().cuda()
    o = OracleSolver(pr.mesh, pr.bcs)
    To = pr.T0.numpy().copy()
    kw = dict(rtol=1e-8, atol=1e-8, max_iter=50000, enforce_positivity=True)
    for k in range(2):
        st, _ = b.step([T], [rho.cuda()], [pr.cp], [pr.kappa], [pr.dt], raise_on_error=False, **kw)
        so, _ = o.step(To, rho.numpy(), pr.cp, pr.kappa.k0, pr.kappa.n, pr.dt, **kw)
        assert st[0]["status"] == so["status"] == (0 if k == 0 else 3), k
        if k == 0:
            assert st[0]["niter"] == so["niter"] and rel_l2(T.cpu().numpy(), To) <= TOL
    b.close()


def test_bounded_wait_runs_out_and_reports():
    """The wavefront kernel's dependency wait is bounded: waiting on a count that
    nothing raises gives up after the limit, raises the error flag the host turns
    into CDM_TIMEOUT, and leaves the context usable (a step runs afterwards)."""
    import ctypes as C
    import time
    from curvilineardiffusionmanuscript_b200 import _lib as L
    lib = L.load()
    expired = C.c_int(0)
    t0 = time.perf_counter()
    rc = lib.cdm_selftest_bounded_wait(0, 0.05, C.byref(expired))
    dt = time.perf_counter() - t0
    assert rc == L.CDM_OK, L.last_error()
    assert expired.value == 1 and 0.05 <= dt < 5.0
    assert lib.cdm_selftest_bounded_wait(0, 0.0, C.byref(expired)) == L.CDM_BAD_INPUT
    probs = problems.batch_2d(nprob=2, nmin=20, nmax=40, seed=4)
    (its, _), = _run_tunings(probs, [(4, 8, 8)], nsteps=1)
    assert all(n > 0 for n in its[0])


def _gpu_steps(m, bcs, T0, rho, dt, nsteps):
    g = PseudoTransientSolver(m, bcs, precision="fp64")
    T, r = T0.clone().cuda(), rho.cuda()
    for _ in range(nsteps):
        step(g, m, T, r, 1.0, PowerLawConductivity(1.0, 0.0), dt, rtol=1e-10, atol=0.0, max_iter=200000)
    g.close()
    return T.cpu().numpy()[m.domain()]


def _oracle_steps(m, bcs, T0, rho, dt, nsteps):
    o = OracleSolver(m, bcs)
    T = T0.numpy().copy()
    for _ in range(nsteps):
        o.step(T, rho.numpy(), 1.0, 1.0, 0.0, dt, rtol=1e-10, atol=0.0, max_iter=200000)
    return T[m.domain()]


def test_decaying_mode_second_order_on_the_gpu():
    """The reference's analytic case (sin(3πx)e^{−9π²t}, negative-symmetry and
    periodic sides) through the fast FP64 path: second order in h, and the same
    errors as the oracle's."""
    e = [decaying_mode_error(n, _gpu_steps) for n in (16, 32)]
    order = math.log2(e[0] / e[1])
    assert 1.8 < order < 2.2, (e, order)
    eo = decaying_mode_error(16, _oracle_steps)
    assert abs(e[0] - eo) <= 1e-6 * eo, (e[0], eo)
    # 3D, through the plane-marching kernel
    e = [decaying_mode_error(n, _gpu_steps, ndim=3) for n in (12, 24)]
    order = math.log2(e[0] / e[1])
    assert 1.8 < order < 2.2, (e, order)
    eo = decaying_mode_error(12, _oracle_steps, ndim=3)
    assert abs(e[0] - eo) <= 1e-6 * eo, (e[0], eo)


def _gpu_k25_steps(m, bcs, T0, rho, dt, nsteps):
    g = PseudoTransientSolver(m, bcs, precision="fp64")
    T, r = T0.clone().cuda(), rho.cuda()
    for _ in range(nsteps):
        step(g, m, T, r, 1.0, PowerLawConductivity(2.5, 0.0), dt, rtol=1e-10, atol=0.0, max_iter=500000)
    g.close()
    return T.cpu().numpy()[m.domain()]


def test_richardson_order_on_the_gpu():
    """The reference's Richardson study through the fast FP64 path (9², 27², 81²)."""
    order = richardson_order(_gpu_k25_steps)
    assert 1.8 < order < 2.4, order


def test_set_tuning_rejects_invalid_choices():
    probs = problems.batch_2d(nprob=2, nmin=20, nmax=30, seed=1)
    b = PseudoTransientBatch([p.mesh for p in probs], [p.bcs for p in probs])
    for bad in ((7, 0, 8), (0, -1, 8), (0, 0, 0), (0, 0, 65)):
        with pytest.raises(APTError):
            b.set_tuning(*bad)
    # the wavefront schedule runs the reciprocal-form kernel only
    for prec in ("fp64_exact", "mixed"):
        bx = PseudoTransientBatch([probs[0].mesh], [probs[0].bcs], precision=prec)
        with pytest.raises(APTError):
            bx.set_tuning(4, 32, 8)
        bx.close()


# --------------------------------------------------------------- fast FP64 form
# The fast form is compared at the workload's stopping rule (rel <= 1e-8 or
# abs <= 1e-8), where the residual is far above round-off: an absolute 1e-8
# alone stops within a few ulps of the FP64 floor of these problems, where the
# iteration at which the noise dips below the threshold is not reproducible.
FAST = dict(precision="fp64", rtol=1e-8, atol=1e-8)


@pytest.mark.parametrize("mean", ["harmonic", "arithmetic"])
def test_fast_gaussian_128_ten_steps(mean):
    _, _, out = run_pair(problems.gaussian_2d(128), mean=mean, **FAST)
    assert_parity(out, exact=False)


@pytest.mark.parametrize("bcs", [
    [DirichletBC(1.5), NeumannBC(), PeriodicBC(), PeriodicBC()],
    [FixedNegSymmetryBC(), NeumannBC(), NeumannBC(), DirichletBC(2.0)],
    [NeumannBC(), PeriodicBC(), NeumannBC(), NeumannBC()],
])
def test_fast_boundary_conditions(bcs):
    _, _, out = run_pair(small_case_2d(ni=29, nj=19, bcs=bcs, source=True), apply_cutoff=True, **FAST)
    assert_parity(out, exact=False)


def test_fast_no_subcycle_multi_halo():
    # (a 300 x 70 mesh diverges in the reference algorithm itself: Vpdτ = CFL·sqrt(min J)
    # exceeds the stable pseudo-step across the thin cells; both paths report NONFINITE)
    pr = small_case_2d(ni=300, nj=260, nhalo=2, kn=2.5, bcs=[DirichletBC(1.2), DirichletBC(0.8), NeumannBC(),
                                                            NeumannBC()])
    _, _, out = run_pair(pr, subcycle_conductivity=False, **FAST)
    assert_parity(out, exact=False)


def test_fast_and_exact_agree_on_large_grid():
    """Exact and fast kernels on a 700x530 grid (many column blocks and strips)."""
    pr = problems.gaussian_2d(700)
    pr.mesh  # square 700
    ge = PseudoTransientSolver(pr.mesh, pr.bcs, precision="fp64_exact")
    gf = PseudoTransientSolver(pr.mesh, pr.bcs, precision="fp64")
    Te, Tf = pr.T0.clone().cuda(), pr.T0.clone().cuda()
    rho = pr.rho.cuda()
    for _ in range(2):
        se, _ = step(ge, pr.mesh, Te, rho, pr.cp, pr.kappa, pr.dt, rtol=1e-8, atol=1e-8)
        sf, _ = step(gf, pr.mesh, Tf, rho, pr.cp, pr.kappa, pr.dt, rtol=1e-8, atol=1e-8)
        assert se["niter"] == sf["niter"]
        assert rel_l2(Tf.cpu().numpy(), Te.cpu().numpy()) <= TOL


def test_device_inputs_written_just_before_the_call():
    """Solvers exist before their inputs: S, T and rho are produced by torch
    kernels queued immediately before set_source / step on a 3000 x 3000 MMS
    grid (long strips, many column blocks).  The library must read them only
    after those kernels finish; fast and exact then agree to round-off."""
    prd = problems.mms_2d(3000, device="cuda")
    solvers = {p: PseudoTransientSolver(prd.mesh, prd.bcs, precision=p) for p in ("fp64", "fp64_exact")}
    out = {}
    for p, g in solvers.items():
        S = problems.mms_source(prd, prd.dt)
        g.set_source(S)
        T = prd.T0.clone() * 1.0
        rho = prd.rho * 1.0
        st, _ = step(g, prd.mesh, T, rho, 1.0, prd.kappa, prd.dt, rtol=1e-8, atol=1e-8, max_iter=100000)
        out[p] = (st["niter"], T.cpu().numpy())
    assert out["fp64"][0] == out["fp64_exact"][0]
    assert rel_l2(out["fp64"][1], out["fp64_exact"][1]) <= TOL


def test_caller_stream_other_than_the_default():
    """Inputs produced on a non-default torch stream are complete before the
    library reads them."""
    pr = problems.gaussian_2d(512)
    side = torch.cuda.Stream()
    g = PseudoTransientSolver(pr.mesh, pr.bcs, precision="fp64_exact")
    ref = PseudoTransientSolver(pr.mesh, pr.bcs, precision="fp64_exact")
    T0 = pr.T0.cuda()
    rho0 = pr.rho.cuda()
    torch.cuda.synchronize()
    Tr = T0.clone()
    sr, _ = step(ref, pr.mesh, Tr, rho0, pr.cp, pr.kappa, pr.dt, rtol=1e-8, atol=1e-8)
    with torch.cuda.stream(side):
        T = T0 * 1.0
        for _ in range(20):
            T = T * 1.0
        rho = rho0 * 1.0
        sg, _ = step(g, pr.mesh, T, rho, pr.cp, pr.kappa, pr.dt, rtol=1e-8, atol=1e-8)
    torch.cuda.synchronize()
    assert sg["niter"] == sr["niter"]
    assert rel_l2(T.cpu().numpy(), Tr.cpu().numpy()) == 0.0


def test_fast_3d_small():
    """3D plane-marching kernel (reciprocal form) against the oracle."""
    _, _, out = run_pair(small_case_3d(), **FAST)
    assert_parity(out, exact=False)


@pytest.mark.parametrize("mean", ["harmonic", "arithmetic"])
def test_fast_3d_mixed_bcs(mean):
    pr = small_case_3d(n=(12, 7, 9), bcs=[DirichletBC(1.0), NeumannBC(), PeriodicBC(), PeriodicBC(),
                                          NeumannBC(), DirichletBC(3.0)])
    _, _, out = run_pair(pr, mean=mean, **FAST)
    assert_parity(out, exact=False)


def test_fast_3d_no_subcycle_negsym():
    pr = small_case_3d(n=(10, 9, 11), bcs=[FixedNegSymmetryBC(), NeumannBC(), NeumannBC(), DirichletBC(2.0),
                                           PeriodicBC(), PeriodicBC()])
    _, _, out = run_pair(pr, subcycle_conductivity=False, **FAST)
    assert_parity(out, exact=False)


def test_fast_and_exact_agree_on_large_3d_grid():
    """Several column tiles and k-strips (70 x 45 x 37 cells)."""
    pr = small_case_3d(n=(70, 45, 37))
    ge = PseudoTransientSolver(pr.mesh, pr.bcs, precision="fp64_exact")
    gf = PseudoTransientSolver(pr.mesh, pr.bcs, precision="fp64")
    Te, Tf = pr.T0.clone().cuda(), pr.T0.clone().cuda()
    rho = pr.rho.cuda()
    for _ in range(2):
        se, _ = step(ge, pr.mesh, Te, rho, pr.cp, pr.kappa, pr.dt, rtol=1e-8, atol=1e-8)
        sf, _ = step(gf, pr.mesh, Tf, rho, pr.cp, pr.kappa, pr.dt, rtol=1e-8, atol=1e-8)
        assert se["niter"] == sf["niter"]
        assert rel_l2(Tf.cpu().numpy(), Te.cpu().numpy()) <= TOL


def test_divergent_case_reports_nonfinite_like_the_reference():
    """A 300 x 70 mesh makes the reference iteration diverge; the library reports
    the same NONFINITE error at the same pseudo-iteration (exact form)."""
    pr = small_case_2d(ni=300, nj=70, kn=2.5)
    o = OracleSolver(pr.mesh, pr.bcs)
    so, _ = o.step(pr.T0.numpy().copy(), pr.rho.numpy(), pr.cp, 1.0, 2.5, pr.dt, rtol=0.0, atol=1e-8,
                   subcycle_conductivity=False)
    g = PseudoTransientSolver(pr.mesh, pr.bcs, precision="fp64_exact")
    with pytest.raises(APTError) as ei:
        step(g, pr.mesh, pr.T0.numpy().copy(), pr.rho.numpy(), pr.cp, pr.kappa, pr.dt, rtol=0.0, atol=1e-8,
             subcycle_conductivity=False)
    assert so["status"] == 2 and ei.value.status == 2
    assert ei.value.stats["niter"] == so["niter"]


def drivers_loop(g, pr, T, rho, dt, t_end, max_cycles, dt_max, **kw):
    """test/integrated/2d/gaussian/run.jl:192-231 with step() calls."""
    t, it, n = 0.0, 0, 0
    while True:
        st, ndt = step(g, pr.mesh, T, rho, pr.cp, pr.kappa, dt, **kw)
        n += 1
        if t >= t_end:
            break
        it += 1
        t += dt
        if it >= max_cycles - 1:
            break
        dt = min(ndt, dt_max)
    return t, dt, n, st


@pytest.mark.parametrize("host", [True, False])
def test_advance_matches_the_drivers_loop(host):
    """cdm_apt_advance runs the drivers' loop with adaptive Δt in one call:
    the same steps, times, next Δt and fields as step() called in that loop."""
    from curvilineardiffusionmanuscript_b200.solver import advance
    pr = problems.gaussian_2d(64)
    kw = dict(rtol=1e-8, atol=1e-8)
    for t_end, max_cycles in ((4e-5, 100), (1.0, 4)):
        g1 = PseudoTransientSolver(pr.mesh, pr.bcs, precision="fp64_exact")
        g2 = PseudoTransientSolver(pr.mesh, pr.bcs, precision="fp64_exact")
        T1 = pr.T0.numpy().copy() if host else pr.T0.clone().cuda()
        T2 = pr.T0.numpy().copy() if host else pr.T0.clone().cuda()
        rho = pr.rho.numpy() if host else pr.rho.cuda()
        r1 = drivers_loop(g1, pr, T1, rho, 1e-5, t_end, max_cycles, 2e-5, **kw)
        t, dt, n, st = advance(g2, pr.mesh, T2, rho, pr.cp, pr.kappa, 1e-5, t_end=t_end, max_cycles=max_cycles,
                               dt_max=2e-5, **kw)
        assert (t, dt, n) == r1[:3]
        assert st["niter"] == r1[3]["niter"]
        a = T1 if host else T1.cpu().numpy()
        b = T2 if host else T2.cpu().numpy()
        assert np.array_equal(a, b)


def test_save_vtk_from_device_state(tmp_path, monkeypatch):
    """save_vtk writes the state of a step taken on device arrays, in the background."""
    from test_vtk_cpu import read_vts
    from curvilineardiffusionmanuscript_b200.vtk import save_vtk
    monkeypatch.chdir(tmp_path)
    pr = problems.gaussian_2d(32)
    g = PseudoTransientSolver(pr.mesh, pr.bcs)
    T, rho = pr.T0.clone().cuda(), pr.rho.cuda()
    step(g, pr.mesh, T, rho, pr.cp, pr.kappa, pr.dt, rtol=1e-8, atol=1e-8)
    fut = save_vtk(g, T, rho, pr.mesh, iteration=3, t=pr.dt, name="gauss", cp=pr.cp, kappa=pr.kappa, dt=pr.dt,
                   background=True)
    tv, ext, arr = read_vts(fut.result(timeout=60))
    dom = pr.mesh.domain()
    assert tv == pr.dt and ext == [0, 32, 0, 32, 0, 0]
    assert np.array_equal(arr["u"], T.cpu().numpy()[dom].astype(np.float32).reshape(-1))
    q, _ = g.get_state()
    assert np.array_equal(arr["q1"], q[0][dom].astype(np.float32).reshape(-1))
    assert {"rho", "diffusivity", "dτ_ρ", "θr_dτ", "q2"} <= set(arr)


# ------------------------------------------------------ energy balance (n1)
@pytest.mark.parametrize("case", ["2d", "3d"])
@pytest.mark.parametrize("precision", ["fp64_exact", "fp64", "mixed"])
def test_energy_balance_matches_the_oracle(case, precision):
    """Σρcₚ T J before and after the step and Δt·ΣS J (the energy balance the
    mixed path keeps in FP64) against the oracle's StepStats: relative 1e-12 for
    the FP64 forms (summation order differs).  Mixed precision: the same bound for
    the first step's Tⁿ and for the source term, and the stated 1e-6 solution
    bound for every Tⁿ⁺¹ (and for the Tⁿ of later steps, the previous result)."""
    if case == "2d":
        pr = small_case_2d(ni=60, nj=47, source=True)
    else:
        pr = small_case_3d(n=(20, 18, 16))
        x, y, z = pr.mesh.centroids
        pr.source = (3.0 * torch.exp(-((x - 0.4) ** 2 + (y - 0.5) ** 2 + (z - 0.6) ** 2) / 0.05)).contiguous()
    kw = dict(rtol=1e-8, atol=1e-8, max_iter=50000)
    _, _, out = run_pair(pr, nsteps=2, precision=precision, device_arrays=True, **kw)
    bound = 1e-6 if precision == "mixed" else 1e-12
    for k, (so, sg, *_) in enumerate(out):
        assert so["status"] == 0 and sg["status"] == 0
        assert abs(sg["source_work"] - so["source_work"]) <= 1e-12 * abs(so["source_work"])
        b0 = 1e-12 if k == 0 else bound
        assert abs(sg["energy_before"] - so["energy_before"]) <= b0 * abs(so["energy_before"]), k
        assert abs(sg["energy_after"] - so["energy_after"]) <= bound * abs(so["energy_after"]), k
        assert so["source_work"] > 0


def test_nonlinear_thermal_conduction_step_wrapper(capsys):
    """nonlinear_thermal_conduction_step! (nonlinear_thermal_conduction.jl:51-72):
    forwards to step! with its keywords, prints the convergence line with
    show_convergence, returns step!'s (stats, next_Δt)."""
    from curvilineardiffusionmanuscript_b200.solver import nonlinear_thermal_conduction_step
    pr = small_case_2d()
    g1 = PseudoTransientSolver(pr.mesh, pr.bcs, precision="fp64_exact")
    g2 = PseudoTransientSolver(pr.mesh, pr.bcs, precision="fp64_exact")
    T1, T2 = pr.T0.numpy().copy(), pr.T0.numpy().copy()
    kw = dict(rtol=0.0, atol=1e-8, t=0.0, tz=False, tz_dim=1, no_t=True)
    s1, n1 = nonlinear_thermal_conduction_step(g1, pr.mesh, T1, pr.rho.numpy(), pr.cp, pr.kappa, pr.dt, **kw)
    out = capsys.readouterr().out
    s2, n2 = step(g2, pr.mesh, T2, pr.rho.numpy(), pr.cp, pr.kappa, pr.dt, **kw)
    assert np.array_equal(T1, T2) and n1 == n2 and s1["niter"] == s2["niter"]
    assert out == "\trel error: %.3e, abs err: %.3e, %i\n" % (s1["rel_err"], s1["abs_err"], s1["niter"])
    nonlinear_thermal_conduction_step(g1, pr.mesh, T1, pr.rho.numpy(), pr.cp, pr.kappa, pr.dt,
                                      show_convergence=False, **kw)
    assert capsys.readouterr().out == ""


@pytest.mark.parametrize("kbcs", [[DirichletBC(3.0), FixedNegSymmetryBC()], [PeriodicBC(), PeriodicBC()],
                                  [NeumannBC(), DirichletBC(0.5)]])
def test_fast_3d_interior_tiles_with_every_k_rule(kbcs):
    """80 x 30 x 12 cells: interior column tiles (the branch-free body, whose
    stage loads run a plane ahead) beside boundary tiles, two k-strips, and every
    ghost rule on the k sides, which the interior body applies per plane."""
    pr = small_case_3d(n=(80, 30, 12), bcs=[NeumannBC(), DirichletBC(1.0), PeriodicBC(), PeriodicBC()] + kbcs)
    _, _, out = run_pair(pr, nsteps=2, **FAST)
    assert_parity(out, exact=False)


@pytest.mark.parametrize("bcs", [[NeumannBC() for _ in range(6)],
                                 [DirichletBC(1.0), NeumannBC(), PeriodicBC(), PeriodicBC(), DirichletBC(3.0),
                                  FixedNegSymmetryBC()]])
def test_fast_3d_square_column_tiles_match_the_oracle(bcs):
    """The plane march on 16 x 16 column tiles (variant 3, 68 ring cells per
    plane instead of 84): 80 x 50 x 12 cells give interior and boundary tiles
    and two k-strips.  Same
    iteration counts as the oracle and the 32 x 8 tiles, the fields within the
    fast form's bar of the oracle and within 1e-13 of the 32 x 8 tiles (the same
    arithmetic per face and cell; only the compiler's contraction choices may
    differ between the instantiations)."""
    pr = small_case_3d(n=(80, 50, 12), bcs=bcs)
    runs = _run_tunings([pr], [(0, 6, 8), (3, 6, 8)], nsteps=2)
    o = OracleSolver(pr.mesh, pr.bcs)
    T = pr.T0.numpy().copy()
    for s in range(2):
        so, _ = o.step(T, pr.rho.numpy(), pr.cp, pr.kappa.k0, pr.kappa.n, pr.dt, rtol=1e-8, atol=1e-8,
                       max_iter=50000)
        assert all(its[s][0] == so["niter"] for its, _ in runs), (s, so["niter"], [its[s] for its, _ in runs])
    for _, Tv in runs:
        assert rel_l2(Tv[0].numpy(), T) <= TOL, rel_l2(Tv[0].numpy(), T)
        assert rel_l2(Tv[0].numpy(), runs[0][1][0].numpy()) <= 1e-13
    # these tiles serve the FP64 reciprocal form only
    for prec in ("fp64_exact", "mixed"):
        bx = PseudoTransientBatch([pr.mesh], [pr.bcs], precision=prec)
        with pytest.raises(APTError):
            bx.set_tuning(3, 0, 8)
        bx.close()

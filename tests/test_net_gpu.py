"""GPU checks of the learned initial guess (include/cdm_net.h).

* forward and backward of the CUDA network against the CPU oracle
  (oracle/net_oracle.py) on the same bf16 inputs and parameters: relative L2
  ≤ 5e-3 for the output and ≤ 2e-2 per layer for the gradient with the
  oracle's bf16 rounding; ≤ 5e-2 against the exact-arithmetic oracle;
* training on APT trajectories lowers the loss;
* a guessed start stops where the plain start stops.
"""
import numpy as np
import pytest
import torch

from helpers import rel_l2
from oracle.net_oracle import CINS, COUTS, NetOracle, bf16, layout
from curvilineardiffusionmanuscript_b200 import _lib as L
from curvilineardiffusionmanuscript_b200 import learned, problems
from curvilineardiffusionmanuscript_b200.solver import PseudoTransientSolver, step

pytestmark = pytest.mark.gpu


def random_params(seed):
    rng = np.random.default_rng(seed)
    offs, n = layout()
    p = np.zeros(n, dtype=np.float32)
    for (wo, bo), ci, co in zip(offs, CINS, COUTS):
        p[wo:bo] = rng.normal(0.0, np.sqrt(2.0 / (9 * ci)), bo - wo)
        p[bo:bo + co] = rng.normal(0.0, 0.05, co)
    return p


def run_gpu(p, x, t):
    net = learned.GuessNet(seed=0)
    net.set_params(p)
    xb = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).cuda().contiguous()
    y = net.forward(xb).cpu().numpy()
    loss = net.backward(torch.tensor(t, dtype=torch.float32).cuda())
    return y, loss, net.get_grads()


def layer_errors(g_gpu, g_ref):
    offs, _ = layout()
    return [(rel_l2(g_gpu[wo:bo], g_ref[wo:bo]), rel_l2(g_gpu[bo:bo + co], g_ref[bo:bo + co]))
            for (wo, bo), co in zip(offs, COUTS)]


@pytest.fixture(scope="module")
def case():
    rng = np.random.default_rng(11)
    x = bf16(rng.normal(size=(2, 32, 48, 16)))
    t = rng.normal(size=(2, 32, 48))
    p = random_params(5)
    y, loss, g = run_gpu(p, x, t)
    return p, x, t, y, loss, g


def test_forward_matches_oracle(case):
    p, x, t, y, loss, g = case
    ref = NetOracle(p, rounding=True)
    yr = ref.forward(x)
    assert rel_l2(y, yr) <= 5e-3
    assert abs(loss - ref.loss(t)) <= 1e-2 * ref.loss(t)


def test_gradients_match_oracle(case):
    p, x, t, y, loss, g = case
    ref = NetOracle(p, rounding=True)
    ref.forward(x)
    gr = ref.backward(t)
    for l, (ew, eb) in enumerate(layer_errors(g, gr)):
        assert ew <= 2e-2, (l, ew)
        assert eb <= 2e-2, (l, eb)


def test_gradients_match_exact_oracle(case):
    p, x, t, y, loss, g = case
    ref = NetOracle(p, rounding=False)
    ref.forward(x)
    gr = ref.backward(t)
    assert rel_l2(g, gr) <= 5e-2


def test_sizes_must_be_multiples_of_8():
    net = learned.GuessNet(seed=0)
    xb = torch.zeros((1, 12, 16, 16), dtype=torch.bfloat16, device="cuda")
    with pytest.raises(Exception):
        net.forward(xb)


def small_problem(n):
    return lambda seed: problems.multi_gaussian_2d(n, seed=seed, device="cuda")


def test_training_lowers_the_loss():
    pr = small_problem(64)(0)
    trajs = learned.generate_trajectories(small_problem(64), seeds=[1, 2, 3, 4], nsteps=6)
    net = learned.GuessNet(seed=3)
    losses = learned.train(net, trajs, pr.mesh, pr.kappa.k0, pr.kappa.n, steps=150, batch=8, crop=32, lr=2e-3)
    assert np.all(np.isfinite(losses))
    assert np.mean(losses[-20:]) < 0.5 * np.mean(losses[:5])


def test_guessed_start_stops_where_the_plain_start_stops():
    """A user guess equal to Tⁿ repeats the plain run; the exact next state
    converges at the first check; both end at the plain solution."""
    pr = small_problem(128)(900)
    kw = dict(rtol=1e-8, atol=1e-8, max_iter=100000)
    g = PseudoTransientSolver(pr.mesh, pr.bcs)
    T = pr.T0.clone()
    frames, its = [T.clone()], []
    for _ in range(3):
        st, _ = step(g, pr.mesh, T, pr.rho, pr.cp, pr.kappa, pr.dt, **kw)
        frames.append(T.clone())
        its.append(st["niter"])
    for which in ("prev", "exact"):
        g2 = PseudoTransientSolver(pr.mesh, pr.bcs)
        T2 = pr.T0.clone()
        for k in range(3):
            if k >= 1:
                g2.set_guess(frames[k].clone() if which == "prev" else frames[k + 1].clone())
                st, _ = step(g2, pr.mesh, T2, pr.rho, pr.cp, pr.kappa, pr.dt, guess=L.CDM_GUESS_USER, **kw)
                assert st["niter"] == (its[k] if which == "prev" else 1)
            else:
                step(g2, pr.mesh, T2, pr.rho, pr.cp, pr.kappa, pr.dt, **kw)
            assert rel_l2(T2.cpu().numpy(), frames[k + 1].cpu().numpy()) <= 1e-8


def run_steps(pr, nsteps, net=None, check_every=4):
    g = PseudoTransientSolver(pr.mesh, pr.bcs)
    guess = L.CDM_GUESS_PREV
    if net is not None:
        learned.attach(g, net)
        guess = L.CDM_GUESS_LEARNED
    T = pr.T0.clone()
    iters = []
    for _ in range(nsteps):
        st, _ = step(g, pr.mesh, T, pr.rho, pr.cp, pr.kappa, pr.dt, rtol=1e-8, atol=1e-8, max_iter=100000,
                     guess=guess, check_every=check_every)
        iters.append(st["niter"])
    g.close()
    return T, iters


def test_trained_guess_gain_over_the_plain_start():
    """What training buys, on held-out seeds of the 256² multi-Gaussian problem:
    the trained guess is at least 2x closer to the next step than the untrained
    network's (linear extrapolation), and steps 2..6 started from it need fewer
    pseudo-iterations than the plain start while ending at the same solution."""
    n = 256
    make = small_problem(n)
    pr0 = make(0)
    trajs = learned.generate_trajectories(make, seeds=list(range(100, 124)), nsteps=8)
    net = learned.GuessNet(seed=1)
    untrained = learned.GuessNet(seed=1)
    losses = learned.train(net, trajs, pr0.mesh, pr0.kappa.k0, pr0.kappa.n, steps=2500, batch=16, crop=128,
                           lr=2e-3)
    assert np.mean(losses[-50:]) < 0.1 * np.mean(losses[:10])
    ljm = learned.log_jmean(pr0.mesh)
    total_plain = total_learned = 0
    for seed in (901, 902):
        pr = make(seed)
        Tp, ip = run_steps(pr, 6)
        Tl, il = run_steps(pr, 6, net)
        assert il[0] == ip[0]  # step 1 has no previous step: both start from Tⁿ
        total_plain += sum(ip[1:])
        total_learned += sum(il[1:])
        assert rel_l2(Tl.cpu().numpy(), Tp.cpu().numpy()) <= 1e-7
        # guess accuracy on this seed's own trajectory
        fr = learned.generate_trajectories(make, seeds=[seed], nsteps=3)[0]
        h = pr.mesh.nhalo
        dom = (slice(h, -h), slice(h, -h))
        e_tr = e_un = 0.0
        for k in (1, 2):
            nxt = fr[k + 1][dom]
            e_tr += float((net.predict(fr[k - 1], fr[k], pr.mesh, 1.0, 3.0, ljm)[dom] - nxt).norm())
            e_un += float((untrained.predict(fr[k - 1], fr[k], pr.mesh, 1.0, 3.0, ljm)[dom] - nxt).norm())
        assert e_tr <= 0.5 * e_un, (e_tr, e_un)
    print(f"pseudo-iterations of steps 2..6: plain {total_plain}, learned {total_learned}")
    assert total_learned < total_plain, (total_learned, total_plain)


def test_extrapolated_start_matches_the_user_guess_and_the_plain_solution():
    """CDM_GUESS_EXTRAPOLATE starts step n+1 from 2Tⁿ − Tⁿ⁻¹ (the first step
    from Tⁿ): bit for bit the run of a user guess computed the same way, and
    within the stopping tolerance of the plain start's solution."""
    pr = small_problem(128)(901)
    kw = dict(rtol=1e-8, atol=1e-8, max_iter=100000, check_every=4)

    def run(mode):
        g = PseudoTransientSolver(pr.mesh, pr.bcs)
        T, prev, its = pr.T0.clone(), None, []
        for k in range(4):
            guess = L.CDM_GUESS_PREV
            if mode == "extrap":
                guess = L.CDM_GUESS_EXTRAPOLATE
            elif mode == "user" and prev is not None:
                g.set_guess((2.0 * T - prev).contiguous())
                guess = L.CDM_GUESS_USER
            cur = T.clone()
            st, _ = step(g, pr.mesh, T, pr.rho, pr.cp, pr.kappa, pr.dt, guess=guess, **kw)
            prev = cur
            its.append(st["niter"])
        g.close()
        return T, its

    Te, ie = run("extrap")
    Tu, iu = run("user")
    Tp, ip = run("plain")
    assert ie == iu and torch.equal(Te, Tu)
    assert ie[0] == ip[0]
    assert rel_l2(Te.cpu().numpy(), Tp.cpu().numpy()) <= 1e-6

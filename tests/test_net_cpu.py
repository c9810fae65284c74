"""CPU checks of the network oracle (no GPU): its analytic gradient against
central finite differences, and its bfloat16 rounding against torch's."""
import numpy as np
import torch

from oracle.net_oracle import CINS, COUTS, NetOracle, bf16, layout


def random_params(rng, scale=1.0):
    offs, n = layout()
    p = np.zeros(n)
    for (wo, bo), ci, co in zip(offs, CINS, COUTS):
        p[wo:bo] = rng.normal(0.0, scale * np.sqrt(2.0 / (9 * ci)), bo - wo)
        p[bo:bo + co] = rng.normal(0.0, 0.05, co)
    return p


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(7)
    p = random_params(rng)
    x = rng.normal(size=(2, 8, 16, 16))
    t = rng.normal(size=(2, 8, 16))
    net = NetOracle(p, rounding=False)
    net.forward(x)
    g = net.backward(t)
    offs, n = layout()
    # entries of every layer's weights and biases
    idx = []
    for wo, bo in offs:
        idx += list(rng.integers(wo, bo, size=3)) + [bo]
    eps = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        a = NetOracle(pp, rounding=False)
        a.forward(x)
        b = NetOracle(pm, rounding=False)
        b.forward(x)
        fd = (a.loss(t) - b.loss(t)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(3)
    a = np.concatenate([rng.normal(size=1000) * 10 ** rng.uniform(-8, 8, size=1000),
                        [0.0, -0.0, 1.0, 1.00390625, 1.005859375, -3.0e38]])
    ref = torch.tensor(a, dtype=torch.float32).to(torch.bfloat16).double().numpy()
    assert np.array_equal(bf16(a), ref)

"""CPU oracle of the learned initial-guess network (test infrastructure only).

A numpy restatement of the network of include/cdm_net.h — layer list, tap
convention, U-Net schedule, loss and backward pass — used by the tests to
check the CUDA forward and backward kernels.  Nothing in the product imports
it.  The network has no counterpart in the reference (which starts every
step from u = Tⁿ, src/pseudo_transient/PseudoTransientSolver.jl:229), so this
oracle is pinned by its own finite-difference check (tests/test_net_cpu.py).

``rounding=True`` rounds to bfloat16 (round to nearest even) exactly where
the CUDA path stores bf16: weights, every activation, the loss gradient and
every backward tensor between layers; accumulation is float64 here and FP32
on the GPU.  ``rounding=False`` is the exact-arithmetic reference used by the
finite-difference check.
"""
from __future__ import annotations

import numpy as np

CINS = [16, 32, 32, 32, 32, 32, 32, 32, 32]
COUTS = [32, 32, 32, 32, 32, 32, 32, 32, 16]


def layout():
    """(w_offset, b_offset) of each layer in the flat parameter vector."""
    offs, o = [], 0
    for ci, co in zip(CINS, COUTS):
        offs.append((o, o + 9 * ci * co))
        o += 9 * ci * co + co
    return offs, o


def bf16(a):
    """Round to bfloat16 (nearest even), returned as float64."""
    a32 = np.ascontiguousarray(a, dtype=np.float32)
    b = a32.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def conv3x3(x, w, b=None):
    """out[n, y, x, :] = Σ_tap x[n, y + dy − 1, x + dx − 1, :] @ w[3dy + dx] (+ b), zero padding."""
    n, h, wd, _ = x.shape
    xp = np.zeros((n, h + 2, wd + 2, x.shape[3]))
    xp[:, 1:-1, 1:-1] = x
    out = np.zeros((n, h, wd, w.shape[2]))
    for t in range(9):
        dy, dx = divmod(t, 3)
        out += np.einsum("nhwc,cd->nhwd", xp[:, dy:dy + h, dx:dx + wd], w[t])
    if b is not None:
        out += b
    return out


def conv3x3_bwd(x, g, w):
    """(dW, db, dX) of conv3x3 for the output gradient g."""
    n, h, wd, _ = x.shape
    xp = np.zeros((n, h + 2, wd + 2, x.shape[3]))
    xp[:, 1:-1, 1:-1] = x
    dw = np.zeros_like(w)
    dxp = np.zeros_like(xp)
    for t in range(9):
        dy, dx = divmod(t, 3)
        dw[t] = np.einsum("nhwc,nhwd->cd", xp[:, dy:dy + h, dx:dx + wd], g)
        dxp[:, dy:dy + h, dx:dx + wd] += np.einsum("nhwd,cd->nhwc", g, w[t])
    return dw, g.sum(axis=(0, 1, 2)), dxp[:, 1:-1, 1:-1]


def pool2(x):
    n, h, w, c = x.shape
    return x.reshape(n, h // 2, 2, w // 2, 2, c).mean(axis=(2, 4))


def up2(x):
    return x.repeat(2, axis=1).repeat(2, axis=2)


def down_sum(g):
    n, h, w, c = g.shape
    return g.reshape(n, h // 2, 2, w // 2, 2, c).sum(axis=(2, 4))


class NetOracle:
    """Forward / backward of the guess network for a flat FP32 parameter vector."""

    def __init__(self, params, rounding=True):
        self.r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
        offs, n = layout()
        p = np.asarray(params, dtype=np.float64)
        assert p.size == n
        self.W, self.b = [], []
        for (wo, bo), ci, co in zip(offs, CINS, COUTS):
            self.W.append(self.r(p[wo:wo + 9 * ci * co]).reshape(9, ci, co))
            self.b.append(p[bo:bo + co].copy())

    def forward(self, x):
        r, W, b = self.r, self.W, self.b
        relu = lambda a: np.maximum(a, 0.0)
        c = {"X": x}
        c["A0"] = r(relu(conv3x3(x, W[0], b[0])))
        c["S0"] = r(relu(conv3x3(c["A0"], W[1], b[1])))
        c["P1"] = r(pool2(c["S0"]))
        c["S1"] = r(relu(conv3x3(c["P1"], W[2], b[2])))
        c["P2"] = r(pool2(c["S1"]))
        c["S2"] = r(relu(conv3x3(c["P2"], W[3], b[3])))
        c["P3"] = r(pool2(c["S2"]))
        c["B3"] = r(relu(conv3x3(c["P3"], W[4], b[4])))
        c["U2"] = r(up2(c["B3"]) + c["S2"])
        c["D2"] = r(relu(conv3x3(c["U2"], W[5], b[5])))
        c["U1"] = r(up2(c["D2"]) + c["S1"])
        c["D1"] = r(relu(conv3x3(c["U1"], W[6], b[6])))
        c["U0"] = r(up2(c["D1"]) + c["S0"])
        c["D0"] = r(relu(conv3x3(c["U0"], W[7], b[7])))
        c["Y"] = conv3x3(c["D0"], W[8], b[8])
        self.c = c
        return c["Y"]

    def loss(self, target):
        d = self.c["Y"][..., 0] - target
        return float(np.mean(d * d))

    def backward(self, target):
        """Flat gradient of the mean squared error of output channel 0."""
        r, W, c = self.r, self.W, self.c
        npix = target.size
        gy = np.zeros_like(c["Y"])
        gy[..., 0] = 2.0 * (c["Y"][..., 0] - target) / npix
        gy = r(gy)
        mask = lambda g, a: np.where(a > 0, g, 0.0)
        gW = [None] * 9
        gB = [None] * 9

        def layer(l, x, g):
            dw, db, dx = conv3x3_bwd(x, g, W[l])
            gW[l], gB[l] = dw, db
            return dx

        gD0 = r(mask(layer(8, c["D0"], gy), c["D0"]))
        gU0 = r(layer(7, c["U0"], gD0))
        gD1 = r(mask(down_sum(gU0), c["D1"]))
        gU1 = r(layer(6, c["U1"], gD1))
        gD2 = r(mask(down_sum(gU1), c["D2"]))
        gU2 = r(layer(5, c["U2"], gD2))
        gB3 = r(mask(down_sum(gU2), c["B3"]))
        gP3 = r(layer(4, c["P3"], gB3))
        gS2 = r(mask(gU2 + up2(gP3) / 4.0, c["S2"]))
        gP2 = r(layer(3, c["P2"], gS2))
        gS1 = r(mask(gU1 + up2(gP2) / 4.0, c["S1"]))
        gP1 = r(layer(2, c["P1"], gS1))
        gS0 = r(mask(gU0 + up2(gP1) / 4.0, c["S0"]))
        gA0 = r(mask(layer(1, c["A0"], gS0), c["A0"]))
        layer(0, c["X"], gA0)
        offs, n = layout()
        out = np.zeros(n)
        for (wo, bo), dw, db in zip(offs, gW, gB):
            out[wo:wo + dw.size] = dw.ravel()
            out[bo:bo + db.size] = db
        return out


def features(tprev, tcur, J, k0, kn, log_jmean, nh):
    """Input features [1, nj, ni, 16] of a full-domain prediction (the CUDA
    features kernel's definition) and the scale s."""
    dom = (slice(nh, -nh), slice(nh, -nh))
    tc, tp, jj = tcur[dom], tprev[dom], J[dom]
    s = float(np.sqrt(np.mean((tc - tp) ** 2)))
    s = s if s > 0 and np.isfinite(s) else 1.0
    kap = np.where(np.isfinite(tc), k0 * np.abs(tc) ** kn if kn != 0 else k0, 0.0)
    x = np.zeros((1,) + tc.shape + (16,))
    x[0, ..., 0] = np.log(np.maximum(np.abs(tc), 1e-30))
    x[0, ..., 1] = (tc - tp) / s
    x[0, ..., 2] = 0.25 * np.log(np.maximum(kap, 1e-30))
    x[0, ..., 3] = np.log(np.maximum(jj, 1e-300)) - log_jmean
    return x, s

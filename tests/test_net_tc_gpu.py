"""The guess network's convolutions on the fifth-generation tensor cores
(tcgen05.mma with the accumulator in tensor memory, TMA-staged halos), which
serve images whose width is a multiple of 128; narrower levels keep the
mma.sync kernel.  Checked on a 16 x 256 input, whose two finest levels (256
and 128 wide) run on tcgen05:

* forward output and every layer's gradient against the numpy oracle with the
  same bf16 rounding points (the bars of test_net_gpu.py);
* against the mma.sync kernels on the same input (CDM_NET_CONV=mma): the two
  differ only in the FP32 summation order of the same bf16 products.
"""
import os

import numpy as np
import pytest
import torch

from helpers import rel_l2
from oracle.net_oracle import NetOracle, bf16
from curvilineardiffusionmanuscript_b200 import learned
from test_net_gpu import layer_errors, random_params

pytestmark = pytest.mark.gpu


def _run(p, x, t, path):
    old = os.environ.get("CDM_NET_CONV")
    if path == "mma":
        os.environ["CDM_NET_CONV"] = "mma"
    else:
        os.environ.pop("CDM_NET_CONV", None)
    try:
        net = learned.GuessNet(seed=0)
        net.set_params(p)
        xb = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).cuda().contiguous()
        y = net.forward(xb).cpu().numpy()
        loss = net.backward(torch.tensor(t, dtype=torch.float32).cuda())
        g = net.get_grads()
        net.close()
        return y, loss, g
    finally:
        if old is None:
            os.environ.pop("CDM_NET_CONV", None)
        else:
            os.environ["CDM_NET_CONV"] = old


@pytest.fixture(scope="module")
def wide_case():
    rng = np.random.default_rng(21)
    x = bf16(rng.normal(size=(2, 16, 256, 16)))
    t = rng.normal(size=(2, 16, 256))
    p = random_params(8)
    return p, x, t, _run(p, x, t, "tc"), _run(p, x, t, "mma")


def test_tensor_core_forward_and_gradients_match_the_oracle(wide_case):
    p, x, t, (y, loss, g), _ = wide_case
    ref = NetOracle(p, rounding=True)
    yr = ref.forward(x)
    assert rel_l2(y, yr) <= 5e-3, rel_l2(y, yr)
    assert abs(loss - ref.loss(t)) <= 1e-2 * ref.loss(t)
    gr = ref.backward(t)
    for l, (ew, eb) in enumerate(layer_errors(g, gr)):
        assert ew <= 2e-2, (l, ew)
        assert eb <= 2e-2, (l, eb)


def test_tensor_core_and_mma_sync_paths_agree(wide_case):
    _, _, _, (y1, l1, g1), (y2, l2, g2) = wide_case
    assert rel_l2(y1, y2) <= 2e-3, rel_l2(y1, y2)
    assert abs(l1 - l2) <= 1e-3 * abs(l2)
    assert rel_l2(g1, g2) <= 1e-2, rel_l2(g1, g2)

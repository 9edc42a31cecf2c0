"""CPU checks of the network oracle: the backward pass against finite
differences, and the parameter layout shared with the library wrapper."""

import numpy as np

from bart_b200 import precnet
from oracle import precnet_oracle as po


def test_layout_matches_wrapper():
    assert po.NPARAMS == precnet.nparams() == 38178
    assert po.offsets() == precnet.layer_offsets()


def test_oracle_gradient_finite_differences():
    rng = np.random.default_rng(0)
    p = po.init_params(rng).astype(np.float64)
    p[po.offsets()[5][0]:] = rng.standard_normal(po.NPARAMS - po.offsets()[5][0]) * 0.1
    x = rng.standard_normal((2, 5, 6, 2))
    t = rng.standard_normal((2, 5, 6, 2))
    loss, g = po.loss_and_grad(p, x, t, bf16_mode=False)
    idx = rng.choice(po.NPARAMS, 40, replace=False)
    idx = np.concatenate([idx, [o[1] for o in po.offsets()]])   # first bias of every layer
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (po.loss_and_grad(pp, x, t, False)[0] - po.loss_and_grad(pm, x, t, False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_rounding():
    a = np.array([1.0, 1.00390625, 1.005859375, -3.14159], dtype=np.float32)
    r = po.bf16(a)
    assert r[0] == 1.0 and r[1] == 1.0          # tie to even
    assert r[2] == np.float32(1.0078125)
    assert abs(r[3] + 3.140625) < 1e-7

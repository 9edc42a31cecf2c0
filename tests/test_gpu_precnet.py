"""GPU learned preconditioner: the network's forward pass and gradients
through the C ABI against the CPU oracle, Adam training, and its use inside
flexible CG."""

import os

import numpy as np
import pytest

from bart_b200 import precnet
from bart_b200.pics import Pics, PicsConf
from conftest import golden, rel
from oracle import nufft_oracle as orc
from oracle import precnet_oracle as po

pytestmark = pytest.mark.gpu


def _params(rng, last=0.1):
    p = po.init_params(rng)
    wo = po.offsets()[5][0]
    p[wo:] = (rng.standard_normal(po.NPARAMS - wo) * last).astype(np.float32)
    for (_, bo, e) in po.offsets():
        p[bo:e] = (rng.standard_normal(e - bo) * 0.05).astype(np.float32)
    return p


def _img(rng, X, Y, n):
    return (rng.standard_normal((X, Y, n)) + 1j * rng.standard_normal((X, Y, n))).astype(np.complex64, order="F")


@pytest.mark.parametrize("X,Y,n", [(40, 24, 2), (64, 64, 1), (33, 17, 3)])
def test_forward_vs_oracle(X, Y, n):
    rng = np.random.default_rng(X + Y)
    p = _params(rng)
    x = _img(rng, X, Y, n)
    net = precnet.PrecNet(p)
    out = np.asarray(net.forward(x, X, Y, n)).reshape(X, Y, n, order="F")
    net.free()
    ref, _ = po.forward(p, po.to_channels(x), bf16_mode=True)
    assert rel(out, po.from_channels(ref)) < 3e-3


@pytest.mark.parametrize("X,Y,n", [(256, 256, 1), (200, 131, 2), (128, 9, 1)])
def test_tensor_core_layers_match_mma_sync(X, Y, n, monkeypatch):
    """The tcgen05 layers (default) against the mma.sync ones: both sum the
    same exact bf16 products in float32, in another order, so outputs and
    gradients differ only where an activation rounds to the other bf16
    neighbour. Covers partial 128-pixel tiles, an odd row count and a batch."""
    rng = np.random.default_rng(X * Y + n)
    p = _params(rng)
    x, t = _img(rng, X, Y, n), _img(rng, X, Y, n)
    net = precnet.PrecNet(p)
    res = {}
    for tc in ("0", "1"):
        monkeypatch.setenv("BNUFFT_NET_TC", tc)
        out = np.asarray(net.forward(x, X, Y, n)).reshape(X, Y, n, order="F")
        g = np.zeros(po.NPARAMS, dtype=np.float32)
        net.train_step(x, t, X, Y, n, 0.0, grads=g)
        res[tc] = (out, g)
    status = net.status()
    net.free()
    assert status == 0
    assert rel(res["1"][0], res["0"][0]) < 2e-3
    for li, (wo, bo, e) in enumerate(po.offsets()):
        assert rel(res["1"][1][wo:bo], res["0"][1][wo:bo]) < 1e-2, li


def test_gradients_vs_oracle():
    rng = np.random.default_rng(5)
    X, Y, n = 40, 24, 2
    p = _params(rng)
    x, t = _img(rng, X, Y, n), _img(rng, X, Y, n)
    net = precnet.PrecNet(p)
    g = np.zeros(po.NPARAMS, dtype=np.float32)
    loss = net.train_step(x, t, X, Y, n, 0.0, grads=g)
    assert np.array_equal(net.params(), p)      # lr 0: no update
    net.free()
    lo, go = po.loss_and_grad(p, po.to_channels(x), po.to_channels(t), bf16_mode=True)
    assert abs(loss - lo) <= 1e-4 * lo
    for li, (wo, bo, e) in enumerate(po.offsets()):
        assert rel(g[wo:bo], go[wo:bo]) < 1e-2, li
        assert rel(g[bo:e], go[bo:e]) < 1e-2, li


def test_gradients_bit_reproducible():
    rng = np.random.default_rng(6)
    p = _params(rng)
    x, t = _img(rng, 64, 32, 2), _img(rng, 64, 32, 2)
    net = precnet.PrecNet(p)
    g1 = np.zeros(po.NPARAMS, dtype=np.float32)
    g2 = np.zeros(po.NPARAMS, dtype=np.float32)
    net.train_step(x, t, 64, 32, 2, 0.0, grads=g1)
    net.train_step(x, t, 64, 32, 2, 0.0, grads=g2)
    net.free()
    assert np.array_equal(g1.view(np.uint32), g2.view(np.uint32))


def test_adam_training_reduces_loss():
    """Fit a fixed linear map (a 3x3 smoothing of the input) on one batch."""
    rng = np.random.default_rng(7)
    X, Y, n = 32, 32, 4
    x = _img(rng, X, Y, n)
    k = np.array([[1, 2, 1], [2, 4, 2], [1, 2, 1]], dtype=np.float32) / 16
    xp = np.pad(x, ((1, 1), (1, 1), (0, 0)))
    t = sum(k[i, j] * xp[i:i + X, j:j + Y] for i in range(3) for j in range(3)).astype(np.complex64, order="F")
    net = precnet.PrecNet(precnet.init_params(1))
    l0 = net.train_step(x, t, X, Y, n, 0.0)
    for _ in range(200):
        net.train_step(x, t, X, Y, n, 3e-3, want_loss=False)
    l1 = net.train_step(x, t, X, Y, n, 0.0)
    net.free()
    assert l1 < 0.2 * l0, (l0, l1)


def test_learned_fcg_zero_network_equals_padded():
    """An all-zero last layer adds nothing: precond 2 iterates exactly like
    precond 3, its padded-circulant base (bit-identical in deterministic
    mode)."""
    g = golden("pics2d_n64_c4")
    net = precnet.PrecNet(precnet.init_params(3))
    out = {}
    os.environ["BNUFFT_FCG_M"] = "1"     # the same truncation for both
    os.environ["BNUFFT_FCG_FOLD"] = "0"  # and the same launches (no folded dot products)
    try:
        for pc in (3, 2):   # no iteration budget: no restart when the learned term stops
            p = Pics(g["traj"], g["sens"], ksp_dims=list(g["ksp"].shape),
                     conf=PicsConf(lam=0.01, maxiter=100, tol=1e-5, scaling=1.0, precond=pc, deterministic=True,
                                   net_iters=0))
            if pc == 2:
                p.set_precnet(net)
            out[pc] = (np.asarray(p.run(g["ksp"])), p.stats())
            p.free()
    finally:
        os.environ.pop("BNUFFT_FCG_M", None)
        os.environ.pop("BNUFFT_FCG_FOLD", None)
    net.free()
    assert np.array_equal(out[3][0].view(np.uint32), out[2][0].view(np.uint32))
    assert out[3][1] == out[2][1]


@pytest.mark.parametrize("pc", [1, 3])
def test_learned_budget_leaves_linear_methods_alone(pc):
    """net_iters belongs to the learned method: the linear preconditioners
    iterate bit for bit the same whatever it is set to."""
    g = golden("pics2d_n64_c4")
    out = []
    for k in (0, 1, 3):
        p = Pics(g["traj"], g["sens"], ksp_dims=list(g["ksp"].shape),
                 conf=PicsConf(lam=0.01, maxiter=100, tol=1e-5, scaling=1.0, precond=pc, deterministic=True,
                               net_iters=k))
        out.append((np.asarray(p.run(g["ksp"])), p.stats()))
        p.free()
    for x, st in out[1:]:
        assert np.array_equal(x.view(np.uint32), out[0][0].view(np.uint32))
        assert st == out[0][1]


def test_learned_fcg_random_network_still_converges():
    """A random (untrained) correction can only slow the solve down; the
    stall fallback and the flexible CG still reach the FP64 solution."""
    g = golden("pics2d_n64_c4")
    traj = g["traj"].real.reshape(3, -1, order="F")
    C = g["sens"].shape[3]
    A = orc.SenseOracle(traj, g["sens"])
    b = A.adjoint(g["ksp"].reshape(-1, C, order="F"))
    xo, _ = orc.conjgrad(A.normal, b, 0.01, 500, tol=1e-10)
    net = precnet.PrecNet(_params(np.random.default_rng(9), last=0.02))
    res = {}
    for mode in ("1", "0"):
        os.environ["BNUFFT_CG_GRAPH"] = mode
        try:
            p = Pics(g["traj"], g["sens"], ksp_dims=list(g["ksp"].shape),
                     conf=PicsConf(lam=0.01, maxiter=400, tol=1e-6, scaling=1.0, precond=2, deterministic=True))
            p.set_precnet(net)
            res[mode] = (np.asarray(p.run(g["ksp"])), p.stats())
            p.free()
        finally:
            os.environ.pop("BNUFFT_CG_GRAPH", None)
    net.free()
    assert np.array_equal(res["1"][0].view(np.uint32), res["0"][0].view(np.uint32))
    x = res["1"][0].reshape(xo.shape, order="F")
    assert res["1"][1][1] <= 1e-6
    assert orc.normal_residual(A, x, b, 0.01) < 1e-5
    assert rel(x, xo) < 5e-4


def test_trained_network_gain():
    """The committed network on held-out 256x256 problems (seeds not used in
    training): each learned step removes more of the A-norm error than the
    padded-circulant step alone (the network's gain, 0.41 -> 0.31 in
    training), and learned flexible CG reaches the 1e-4 tolerance (true
    residual) in fewer iterations than plain CG. Against the padded-circulant
    PCG alone it needs more iterations: a greedy one-step gain is not a
    Krylov gain."""
    import torch
    from bart_b200.problems import cgsense_problem
    dev = torch.device("cuda", 0)
    net = precnet.PrecNet.load()
    lc, ll = precnet.heldout_loss(net, 3, 11, dev)
    assert ll < 0.85 * lc, (lc, ll)
    prob = cgsense_problem(np.random.default_rng(12))
    s_cg = precnet.solve_stats(prob, dev, 0, reps=1)
    s_l = precnet.solve_stats(prob, dev, 2, net, reps=1)
    net.free()
    assert s_l["true_res"] <= 1.05e-4
    assert s_l["iters"] < s_cg["iters"], (s_l, s_cg)

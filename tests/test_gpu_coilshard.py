"""Coil-sharded CG-SENSE on the device: the library's normal operator and
right-hand side on coil subsets add up to the whole problem's, and the
sharded solve (one rank) gives the reference's pics output."""

import numpy as np
import pytest

from conftest import golden, rel

pytestmark = pytest.mark.gpu


def _d(a, dev):
    import torch
    return torch.from_numpy(np.asfortranarray(a).ravel(order="F").astype(np.complex64)).to(dev)


def _model(g, c0, c1, dev):
    from bart_b200.pics import Pics, PicsConf
    sens = g["sens"][..., c0:c1]
    kd = list(g["ksp"].shape[:3]) + [c1 - c0]
    return Pics(_d(g["traj"], dev), _d(sens, dev), ksp_dims=kd, conf=PicsConf(lam=0.01, scaling=1.0),
                traj_dims=list(g["traj"].shape), sens_dims=list(sens.shape))


def test_coil_shares_add_up_to_the_whole(cuda):
    """Two models on coils [0, 2) and [2, 4): their A^H A x and A^H y sum to
    the four-coil model's (what the per-iteration all-reduce relies on)."""
    g = golden("pics2d_n64_c4")
    rng = np.random.default_rng(1)
    x = _d(rng.standard_normal((64, 64)) + 1j * rng.standard_normal((64, 64)), cuda)
    full, a, b = _model(g, 0, 4, cuda), _model(g, 0, 2, cuda), _model(g, 2, 4, cuda)
    n_full = full.normal(x).cpu().numpy()
    n_sum = (a.normal(x) + b.normal(x)).cpu().numpy()
    assert rel(n_sum, n_full) < 1e-5
    y = g["ksp"]
    r_full = full.rhs(_d(y, cuda)).cpu().numpy()
    r_sum = (a.rhs(_d(y[..., :2], cuda)) + b.rhs(_d(y[..., 2:], cuda))).cpu().numpy()
    assert rel(r_sum, r_full) < 1e-5
    for m in (full, a, b):
        m.free()


def test_sharded_solve_one_rank_vs_reference(cuda):
    """Without a process group the sharded solve holds every coil: 5 and 30
    iterations at scaling 1 give the reference's pics -i5 -w1 and -i30 -w1;
    with the scaling estimated it uses the scaling of the library's own
    pics."""
    from bart_b200.coilshard import CoilShardedPics
    from bart_b200.pics import Pics, PicsConf
    g = golden("pics2d_n64_c4")
    traj, sens, ksp = _d(g["traj"], cuda), _d(g["sens"], cuda), _d(g["ksp"], cuda)
    dims = dict(traj_dims=list(g["traj"].shape), sens_dims=list(g["sens"].shape))
    cs = CoilShardedPics(traj, sens, list(g["ksp"].shape), lam=0.01, maxiter=5, scaling=1.0, **dims)
    x = cs.run(ksp).cpu().numpy()
    assert cs.iters == 5
    assert rel(x, g["x5_w1"]) < 1e-5
    cs.free()
    # 30 unconverged iterations: the reference's float32 scalars (the
    # default) keep the iterates on the reference's, as for the one-GPU pics
    cs = CoilShardedPics(traj, sens, list(g["ksp"].shape), lam=0.01, maxiter=30, scaling=1.0, **dims)
    x = cs.run(ksp).cpu().numpy()
    assert cs.iters == 30
    assert rel(x, g["x30_w1"]) < 1e-4, rel(x, g["x30_w1"])
    cs.free()
    cs = CoilShardedPics(traj, sens, list(g["ksp"].shape), lam=0.01, maxiter=30, **dims)
    cs.run(ksp)
    p = Pics(traj, sens, ksp_dims=list(g["ksp"].shape), conf=PicsConf(lam=0.01, maxiter=30), **dims)
    p.run(ksp)
    assert cs.scale == pytest.approx(p.stats()[2], rel=1e-6)
    cs.free()
    p.free()


@pytest.mark.parametrize("precond", [0, 3])
def test_sharded_solve_to_tolerance_on_the_fused_passes(cuda, precond):
    """The sharded solve's CG runs on the library's fused passes
    (bnufft_cg_*): solved to ||r|| <= 1e-4 ||A^H y|| (plain CG, or PCG with
    the padded-circulant preconditioner), its image meets the true
    normal-equation residual of the oracle like the library's one-call
    solve, in about the same number of iterations."""
    from bart_b200 import _lib
    from bart_b200.coilshard import CoilShardedPics
    from bart_b200.pics import Pics, PicsConf
    from oracle import nufft_oracle as orc
    g = golden("pics2d_n64_c4")
    traj, sens, ksp = _d(g["traj"], cuda), _d(g["sens"], cuda), _d(g["ksp"], cuda)
    dims = dict(traj_dims=list(g["traj"].shape), sens_dims=list(g["sens"].shape))
    n0 = _lib.load().bnufft_launch_count()
    cs = CoilShardedPics(traj, sens, list(g["ksp"].shape), lam=0.01, maxiter=300, tol=1e-4, precond=precond, **dims)
    x = cs.run(ksp).cpu().numpy()
    assert _lib.load().bnufft_launch_count() > n0
    p = Pics(traj, sens, ksp_dims=list(g["ksp"].shape),
             conf=PicsConf(lam=0.01, maxiter=300, tol=1e-4, precond=precond), **dims)
    y = p.run(ksp).cpu().numpy()
    it_lib = p.stats()[0]
    A = orc.SenseOracle(g["traj"].real.reshape(3, -1, order="F"), g["sens"])
    b = A.adjoint(g["ksp"].reshape(-1, g["sens"].shape[3], order="F"))
    b = b / orc.estimate_scaling_norm(b)
    for img in (x, y):
        assert orc.normal_residual(A, img.reshape(b.shape, order="F"), b, 0.01) < 2e-4
    # the plain CG's ~50 iterations to 1e-4 follow the rounding (the
    # one-call solve keeps the reference's float32 scalars and sums p^H A p
    # in its row pass): within 10 %; PCG's ~10 within one
    assert abs(cs.iters - it_lib) <= max(1, it_lib // 10), (cs.iters, it_lib)
    cs.free()
    p.free()

"""Coil-sharded CG-SENSE: the host algorithm on 2 gloo ranks (CPU), each
rank's share of the normal operator from the oracle on its own coils; the
result is the reference's pics output (golden vectors) and the one-rank
solve."""

import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import golden, rel


def test_coil_range_covers_every_coil_once():
    from bart_b200.coilshard import coil_range
    for C in (1, 3, 4, 7, 32):
        for world in (1, 2, 3, 8):
            rs = [coil_range(C, r, world) for r in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == C
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
            sizes = [c1 - c0 for c0, c1 in rs]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        coil_range(4, 2, 2)


def test_scaling_rule_matches_the_oracle():
    import torch
    from bart_b200.coilshard import scaling_from_adjoint
    from oracle import nufft_oracle as orc
    rng = np.random.default_rng(0)
    for tail in (1.0, 50.0):	# the p90 branch and the maximum branch
        a = (rng.standard_normal((40, 40, 1, 1)) + 1j * rng.standard_normal((40, 40, 1, 1))).astype(np.complex64)
        a.flat[7] *= tail
        want = orc.estimate_scaling_norm(a)
        assert scaling_from_adjoint(torch.from_numpy(a)) == pytest.approx(want, rel=1e-6)
    assert scaling_from_adjoint(torch.zeros(16, dtype=torch.complex64)) == 1.0	# as pics: a zero scale is 1


def _solve(name, rank, world, maxiter, scaling, f32_scalars=False):
    import torch
    from bart_b200.coilshard import allreduce_sum, coil_range, scaling_from_adjoint, sharded_cg
    from oracle import nufft_oracle as orc
    g = golden(name)
    traj = g["traj"].real.reshape(3, -1, order="F")
    C = g["sens"].shape[3]
    y = g["ksp"].reshape(-1, C, order="F").astype(np.complex128)
    c0, c1 = coil_range(C, rank, world)
    A = orc.SenseOracle(traj, g["sens"][..., c0:c1])
    b = torch.from_numpy(A.adjoint(y[:, c0:c1]))
    allreduce_sum(b)
    scale = scaling if scaling else scaling_from_adjoint(b)
    b = b / scale

    def normal_local(p):
        return torch.from_numpy(A.normal(p.numpy()))

    x, it = sharded_cg(normal_local, b, 0.01, maxiter, reduce=allreduce_sum, f32_scalars=f32_scalars)
    return x.numpy(), scale, it


def _solve_pcg(name, rank, world, tol=1e-4):
    """PCG with the padded-circulant preconditioner (the trajectory's PSF and
    lambda only, so the same operator on every rank)."""
    import torch
    from bart_b200.coilshard import allreduce_sum, coil_range, sharded_cg
    from oracle import nufft_oracle as orc
    g = golden(name)
    traj = g["traj"].real.reshape(3, -1, order="F")
    C = g["sens"].shape[3]
    y = g["ksp"].reshape(-1, C, order="F").astype(np.complex128)
    c0, c1 = coil_range(C, rank, world)
    A = orc.SenseOracle(traj, g["sens"][..., c0:c1])
    M = orc.padded_precond(A.nufft, 0.01)
    b = torch.from_numpy(A.adjoint(y[:, c0:c1]))
    allreduce_sum(b)
    x, it = sharded_cg(lambda p: torch.from_numpy(A.normal(p.numpy())), b, 0.01, 100, tol, allreduce_sum,
                       precond=lambda r: torch.from_numpy(M(r.numpy())))
    return x.numpy(), b.numpy(), it


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out = {}
        for name in ("pics2d_n64_c4", "pics2d_n48_c3"):	# 2 + 2 and 2 + 1 coils
            out[name, 5] = _solve(name, rank, world, 5, 1.0)
            out[name, 30] = _solve(name, rank, world, 30, 0.0)
            out[name, "30f32"] = _solve(name, rank, world, 30, 0.0, f32_scalars=True)
            out[name, "pcg"] = _solve_pcg(name, rank, world)
        out["pics3d_n16_c2", 5] = _solve("pics3d_n16_c2", rank, world, 5, 1.0)	# 3D, 1 + 1 coils
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_two_ranks_match_reference_and_one_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, 29517, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = golden("pics3d_n16_c2")
    x3 = res[0]["pics3d_n16_c2", 5][0]
    assert rel(x3, g["x5_w1"].reshape(x3.shape, order="F")) < 1e-5
    for name in ("pics2d_n64_c4", "pics2d_n48_c3"):
        g = golden(name)
        x0, _, it0 = res[0][name, 5]
        x1, _, _ = res[1][name, 5]
        assert it0 == 5
        assert np.array_equal(x0, x1)                       # replicated on every rank
        assert rel(x0, g["x5_w1"].reshape(x0.shape, order="F")) < 1e-5   # the reference's pics -i5 -w1
        xs, scale, _ = res[0][name, 30]
        x_one, scale_one, _ = _solve(name, 0, 1, 30, 0.0)    # no process group: all coils here
        assert scale == pytest.approx(scale_one, rel=1e-6)
        assert rel(xs, x_one) < 1e-9
        from oracle import nufft_oracle as orc
        traj = g["traj"].real.reshape(3, -1, order="F")
        y = g["ksp"].reshape(-1, g["sens"].shape[3], order="F")
        _, sc_orc = orc.pics_l2(traj, y, g["sens"], lam=0.01, maxiter=1)	# the scaling rule on all coils
        assert scale == pytest.approx(sc_orc, rel=1e-6)
        # float64 scalars: the oracle's float64 CG on all coils. They agree
        # to 1.2e-8 up to 10 iterations (the oracle scales y by float32(1 /
        # scale), this solve divides b); 30 unconverged iterations amplify
        # those last bits to 8e-5
        x_orc, _ = orc.pics_l2(traj, y, g["sens"], lam=0.01, maxiter=30)
        assert rel(xs, x_orc) < 1e-3
        # the reference's pics -i30 (scaling estimated): with float32 alpha
        # and beta, as the reference rounds them, 30 unconverged iterations
        # stay within 1.6e-4 of it (float64 scalars drift to 1e-2)
        x32 = res[0][name, "30f32"][0]
        assert rel(x32, g["x30"].reshape(x32.shape, order="F")) < 5e-4
        # PCG to 1e-4: the oracle's PCG on all coils, iteration for iteration
        xp, b, itp = res[0][name, "pcg"]
        A = orc.SenseOracle(traj, g["sens"])
        xo, ito = orc.pcg(A.normal, b, 0.01, orc.padded_precond(A.nufft, 0.01), tol=1e-4, maxiter=100)
        assert itp == ito < 100
        assert rel(xp, xo) < 1e-9
        assert np.array_equal(xp, res[1][name, "pcg"][0])


def test_exact_convergence_keeps_the_solution():
    """A normal operator that CG solves exactly in one step (a multiple of
    the identity): later iterations keep x (the reference stops at
    <p, A p> = 0) instead of dividing by zero."""
    import torch
    from bart_b200.coilshard import sharded_cg
    b = torch.tensor([1.0 + 2.0j, -0.5j, 3.0], dtype=torch.complex128)
    x, it = sharded_cg(lambda p: 3.0 * p, b, 1.0, 5)
    assert it == 5
    assert torch.allclose(x, b / 4.0)
    assert torch.isfinite(torch.view_as_real(x)).all()


def test_sharded_model_rejects_other_preconditioners():
    """The sharded solve runs CG or the padded-circulant PCG (Toeplitz); the
    flexible-CG preconditioners are refused before any device work."""
    from bart_b200.coilshard import CoilShardedPics
    for kw in (dict(precond=1), dict(precond=2), dict(precond=3, toeplitz=False)):
        with pytest.raises(ValueError):
            CoilShardedPics(None, None, [1, 2, 2, 1], **kw)

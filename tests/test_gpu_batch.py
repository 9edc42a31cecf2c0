"""Batches of uneven reconstructions as one graph: the same results as single
solves, and the reference's pics on a non-power-of-two problem."""

import numpy as np
import pytest

from bart_b200.batch import BatchRecon, autotune_bins, uneven_problems
from conftest import golden, rel

pytestmark = pytest.mark.gpu


def test_batch_equals_loop_of_single_solves(cuda):
    """Deterministic gridding: the batch graph and a loop of single solves
    give identical bits for every problem (sizes, spokes and coils differ)."""
    probs = uneven_problems(10, 3, sizes=(40, 130), spokes=(12, 48), coils=(2, 6))
    assert len({p["sens"].shape[0] for p in probs}) > 5
    br = BatchRecon(probs, cuda, maxiter=8, deterministic=True).build()
    assert br.kernels() > 10 * 8 * 4
    br.run()
    a = [x.cpu().numpy().copy() for x in br.img]
    for x in br.img:
        x.zero_()
    br.run_loop()
    b = [x.cpu().numpy() for x in br.img]
    br.free()
    for u, v in zip(a, b):
        assert np.array_equal(u.view(np.uint32), v.view(np.uint32))
        assert np.linalg.norm(u) > 0


def test_batch_member_vs_reference(cuda):
    """A 48x48 problem inside a batch with others matches the reference's
    pics -l2 -r0.01 -i5 -w1."""
    g = golden("pics2d_n48_c3")
    prob = {"traj": g["traj"], "sens": g["sens"], "ksp": g["ksp"]}
    others = uneven_problems(3, 5, sizes=(64, 100), spokes=(16, 32), coils=(2, 4))
    br = BatchRecon([prob] + others, cuda, maxiter=5, scaling=1.0).build()
    br.run()
    x = br.img[0].cpu().numpy()
    br.free()
    assert rel(x, g["x5_w1"]) < 1e-5


def test_autotuner_returns_candidates(cuda):
    table, detail = autotune_bins(cuda, sizes=(64, 96), candidates=(16, 32), coils=2, spokes=16, reps=1)
    assert set(table) == {64, 96} and all(v in (16, 32) for v in table.values())
    assert all(len(d) == 2 for d in detail.values())


@pytest.mark.parametrize("traj_per_slice,extra", [(False, []), (True, []), (False, ["--precond", "3"]),
                                                  (True, ["--precond", "3", "--tol", "1e-4", "-i", "200"])])
def test_cli_loop_over_slices_matches_single_runs(cuda, tmp_path, traj_per_slice, extra):
    """python -m bart_b200 -l 8192 pics (slices along dim 13, the reference's
    bart -l): all slices in one batched launch, joined along dim 13, equal to
    running pics on each slice's own files (up to the atomics' summation
    order of the adjoint). The trajectory is shared (size 1 along dim 13) or
    one per slice. With --precond 3 the batch runs the padded-circulant PCG;
    with a tolerance the slices are solved one after another."""
    from bart_b200 import __main__ as cli
    from bart_b200.cfl import readcfl, writecfl
    from bart_b200.problems import cgsense_problem, simulate_ksp

    S = 3
    base = cgsense_problem(np.random.default_rng(10), N=64, coils=4, spokes=24)
    probs = []
    for sl in range(S):
        p = cgsense_problem(np.random.default_rng(20 + sl), N=64, coils=4, spokes=24)
        t = base["traj"].copy()
        if traj_per_slice:	# each slice's spokes rotated by its own angle
            c, sn = np.cos(0.3 * sl), np.sin(0.3 * sl)
            x, y = t[0].real.copy(), t[1].real.copy()
            t[0], t[1] = c * x - sn * y, sn * x + c * y
        p["traj"] = t.astype(np.complex64)
        p["ksp"] = simulate_ksp(p["traj"], p["truth"], p["sens"], 40.0, np.random.default_rng(30 + sl))
        probs.append(p)

    def stack(key):
        arrs = [np.asarray(p[key]) for p in probs]
        a16 = [a.reshape(list(a.shape) + [1] * (16 - a.ndim), order="F") for a in arrs]
        return np.concatenate(a16, axis=13)

    ksp, sens = stack("ksp"), stack("sens")
    traj = stack("traj") if traj_per_slice else probs[0]["traj"]
    d = str(tmp_path)
    writecfl(d + "/traj", traj)
    writecfl(d + "/ksp", ksp)
    writecfl(d + "/sens", sens)
    opts = ["-r", "0.01", "-i", "15"] + extra
    assert 0 == cli.main(["-l", "8192", "pics"] + opts + ["-t", d + "/traj", d + "/ksp", d + "/sens", d + "/out"])
    out = readcfl(d + "/out")
    assert out.shape[13] == S and out.shape[:3] == (64, 64, 1)
    for s in range(S):
        p = probs[s]
        writecfl(d + f"/t{s}", p["traj"])
        writecfl(d + f"/k{s}", p["ksp"])
        writecfl(d + f"/s{s}", p["sens"])
        assert 0 == cli.main(["pics"] + opts + ["-t", d + f"/t{s}", d + f"/k{s}", d + f"/s{s}", d + f"/o{s}"])
        single = readcfl(d + f"/o{s}").reshape(64, 64, order="F")
        joined = out[..., s, :, :].reshape(64, 64, order="F")
        assert np.linalg.norm(single) > 0
        if "--tol" in extra:	# each slice solved to the tolerance of its own problem
            from oracle import nufft_oracle as orc
            A = orc.SenseOracle(p["traj"].real.reshape(3, -1, order="F"), p["sens"])
            b = A.adjoint(p["ksp"].reshape(-1, p["sens"].shape[3], order="F"))
            b = b / orc.estimate_scaling_norm(b)
            assert orc.normal_residual(A, joined.reshape(b.shape, order="F"), b, 0.01) < 2e-4, s
        else:			# fixed iteration counts: up to the adjoint's atomic summation order
            assert rel(joined, single) < 1e-4, (s, rel(joined, single))


def test_cli_loop_two_ranks_split_by_cost(cuda, tmp_path):
    """torchrun with 2 ranks: the slices are split over the ranks by the cost
    model, each rank solves its share with no exchange, rank 0 gathers and
    writes the joined image; it matches the one-process run (both ranks share
    the one GPU here; device = local rank mod GPU count). Two fresh runs of
    these undersampled slices (24 spokes at 64^2) differ by up to 5e-3: the
    adjoint's atomic adds sum in a different order each run and ten CG
    iterations amplify it; hence 1.5e-2, and every slice must also sit at its
    own index (other slices are different phantoms, ~1 apart)."""
    import os
    import socket
    import subprocess
    import sys
    from bart_b200 import __main__ as cli
    from bart_b200.cfl import readcfl, writecfl
    from bart_b200.problems import cgsense_problem, simulate_ksp

    S = 5	# an odd count: the ranks get 3 and 2 slices
    traj = cgsense_problem(np.random.default_rng(39), N=64, coils=4, spokes=24)["traj"]
    ksp_l, sens_l = [], []
    for sl in range(S):
        p = cgsense_problem(np.random.default_rng(40 + sl), N=64, coils=4, spokes=24)
        k = simulate_ksp(traj, p["truth"], p["sens"], 40.0, np.random.default_rng(60 + sl))
        ksp_l.append(k.reshape(list(k.shape) + [1] * (16 - k.ndim), order="F"))
        sens_l.append(p["sens"].reshape(list(p["sens"].shape) + [1] * 12, order="F"))
    d = str(tmp_path)
    writecfl(d + "/traj", traj)
    writecfl(d + "/ksp", np.concatenate(ksp_l, axis=13))
    writecfl(d + "/sens", np.concatenate(sens_l, axis=13))
    opts = ["-r", "0.01", "-i", "10", "-t", d + "/traj", d + "/ksp", d + "/sens"]
    assert 0 == cli.main(["-l", "8192", "pics"] + opts + [d + "/one"])
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, PYTHONPATH=root + os.pathsep + os.environ.get("PYTHONPATH", ""))
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", str(port), "-m", "bart_b200",
                        "-l", "8192", "pics"] + opts + [d + "/two"],
                       cwd=root, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    one, two = readcfl(d + "/one"), readcfl(d + "/two")
    assert one.shape == two.shape and one.shape[13] == S
    for s in range(S):
        a, b = one[..., s, :, :], two[..., s, :, :]
        assert np.linalg.norm(a) > 0
        assert rel(b, a) < 1.5e-2, (s, rel(b, a))
        others = [rel(b, one[..., t, :, :]) for t in range(S) if t != s]
        assert min(others) > 10 * rel(b, a), (s, others)


def test_cli_pics_from_a_reference_stream(cuda, tmp_path, monkeypatch):
    """python -m bart_b200 -l 8192 pics ... - sens out with the k-space on
    stdin as the reference streams it (copy --stream 8192 | tee -b): every
    slice is reconstructed as it arrives, and the images equal those of the
    same loop over the k-space file (there one batched launch, so equal up
    to the atomics' float32 summation order: 30 iterations, where two runs
    of the same slice agree to 2e-5; at 10 they differ by up to 6e-3)."""
    import io
    import sys
    import bart_b200.__main__ as cli
    from bart_b200.cfl import readcfl, writecfl
    g = golden("pics2d_n64_c4")
    s = golden("stream_ksp_c4_s3")
    d = str(tmp_path)
    writecfl(d + "/traj", g["traj"])
    writecfl(d + "/sens", g["sens"])
    writecfl(d + "/ksp", s["ksp"])
    opts = ["-l2", "-r0.01", "-i30"]
    monkeypatch.setattr(sys, "stdin", type("Stdin", (), {"buffer": io.BytesIO(s["stream"].tobytes())})())
    assert 0 == cli.main(["-l", "8192", "pics"] + opts + ["-t", d + "/traj", "-", d + "/sens", d + "/out_stream"])
    assert 0 == cli.main(["-l", "8192", "pics"] + opts + ["-t", d + "/traj", d + "/ksp", d + "/sens", d + "/out_file"])
    a, b = readcfl(d + "/out_stream"), readcfl(d + "/out_file")
    assert a.shape == b.shape and a.shape[13] == 3
    assert rel(a, b) < 1e-4

"""The bart -l / -p loop front-end (src/bart.c:202-217): slicing, joining and
index order, on the CPU."""

import numpy as np
import pytest

from bart_b200 import __main__ as cli
from bart_b200.loop import loop_dims, loop_indices, loop_sizes, place_at, slice_at


def test_loop_dims_and_sizes():
    assert loop_dims(8192) == [13]
    assert loop_dims((1 << 10) | (1 << 13)) == [10, 13]
    assert loop_sizes([[3, 64, 8] + [1] * 10 + [1], [1, 64, 8, 4] + [1] * 9 + [5]], [13]) == [5]
    with pytest.raises(ValueError):
        loop_sizes([[1] * 13 + [3], [1] * 13 + [5]], [13])
    with pytest.raises(ValueError):
        loop_dims(1 << 16)


def test_loop_indices_first_dim_fastest():
    assert loop_indices([2, 3]) == [(0, 0), (1, 0), (0, 1), (1, 1), (0, 2), (1, 2)]
    assert loop_indices([1]) == [(0,)]


def test_slice_and_place_round_trip():
    rng = np.random.default_rng(0)
    a = (rng.standard_normal((4, 3, 1, 2) + (1,) * 9 + (5, 1, 1)) + 0j).astype(np.complex64)
    out = np.zeros_like(a, order="F")
    for idx in loop_indices([5]):
        s = slice_at(a, [13], idx)
        assert s.shape[13] == 1
        np.testing.assert_array_equal(s[..., 0, :, :], a[..., idx[0]:idx[0] + 1, :, :][..., 0, :, :])
        place_at(out, [13], idx, s)
    np.testing.assert_array_equal(out, a)
    # a file of size 1 along the looped dim is used for every index
    b = a[..., :1, :, :]
    np.testing.assert_array_equal(slice_at(b, [13], (3,)), b)


def test_cli_rejects_loop_for_other_tools(capsys):
    assert 2 == cli.main(["-l", "8192", "nufft", "t", "i", "o"])
    assert 2 == cli.main(["-l"])


def test_pics_cli_options_parse(tmp_path):
    """pics command-line options: the reference's defaults (plain CG, -i
    iterations) and the library's opt-in --precond / --tol."""
    from bart_b200.cfl import writecfl
    d = str(tmp_path)
    for name in ("t", "k", "s"):
        writecfl(d + "/" + name, np.zeros((2, 2), dtype=np.complex64))
    a = cli.parse_pics(["-r", "0.01", "-i", "7", "-t", d + "/t", d + "/k", d + "/s", d + "/o"])
    assert (a.precond, a.tol, a.iters, a.lam, a.toeplitz) == (0, 0.0, 7, 0.01, True)
    a = cli.parse_pics(["--precond", "3", "--tol", "1e-4", "-t", d + "/t", d + "/k", d + "/s", d + "/o"])
    assert (a.precond, a.tol) == (3, 1e-4)
    with pytest.raises(SystemExit):
        cli.parse_pics(["--precond", "3", "--no-toeplitz", "-t", d + "/t", d + "/k", d + "/s", d + "/o"])


def test_pics_cli_single_problem_runs_on_rank_0_only(tmp_path, monkeypatch):
    """Under torchrun without -l/-p there is one problem: ranks other than 0
    return at once, write nothing and touch no GPU."""
    from bart_b200.cfl import writecfl
    d = str(tmp_path)
    for name in ("t", "k", "s"):
        writecfl(d + "/" + name, np.zeros((2, 2), dtype=np.complex64))
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    assert 0 == cli.main(["pics", "-r", "0.01", "-t", d + "/t", d + "/k", d + "/s", d + "/o"])
    import os
    assert not os.path.exists(d + "/o.cfl")


def test_loop_split_follows_the_cost_model():
    """The slices a rank of the -l loop takes: the cost-model split of the
    loop indices, disjoint over ranks, all of them together."""
    from bart_b200.dist import partition, problem_cost
    sizes = [64, 64, 128, 256, 64, 32]
    probs = [{"sens": np.zeros((n, n, 1, 4), np.complex64), "ksp": np.zeros((1, 2 * n, 32, 4), np.complex64)}
             for n in sizes]
    costs = [problem_cost(p, 10) for p in probs]
    shards = partition(costs, 2)
    assert 3 in shards[0] and 2 in shards[1]      # the two largest on different ranks
    assert sorted(shards[0] + shards[1]) == list(range(len(sizes)))


def _oracle_ecalib(ksp, conf=None, emaps=True, **kw):
    """Stand-in for the library call in the host-logic tests: the oracle's
    ecalib with the library's output shapes (16 dims)."""
    from oracle import espirit_oracle as eo
    from bart_b200.espirit import EcalibConf, output_dims
    conf = conf or EcalibConf()
    k = np.asarray(ksp)
    s, e, val, n, cd = eo.ecalib(k.reshape(k.shape[:4], order="F") if k.ndim > 4 else k,
                                 kdims=conf.kdims, calsize=conf.calsize, maps=conf.maps, crop=conf.crop,
                                 softcrop=conf.softcrop, rotphase=conf.rotphase, intensity=conf.intensity)
    sd, ed = output_dims(list(k.shape), conf)
    return (s.astype(np.complex64).reshape(sd, order="F"),
            e.astype(np.complex64).reshape(ed, order="F") if emaps else None,
            {"svals": val, "nkernels": n, "caldims": cd})


def test_ecalib_slice_loop_joins_per_slice_calibrations(tmp_path, monkeypatch):
    """python -m bart_b200 -l 8192 ecalib: each slice (dim 13) calibrated on
    its own, maps and eigenvalue maps joined along dim 13 at their slice
    index, with the options parsed as the reference's ecalib does (here -m 1
    -k 5 -r 20:20:1). The calibration itself is stubbed by the oracle."""
    import bart_b200.espirit as esp
    from bart_b200 import synth
    from bart_b200.cfl import readcfl, writecfl
    monkeypatch.setattr(esp, "ecalib", _oracle_ecalib)
    rng = np.random.default_rng(12)
    slices = []
    for _ in range(2):
        img = synth.ellipse_phantom(32, 6, rng)
        k = synth.cartesian_ksp(img, synth.coil_maps(32, 4, rng), rng, 40.0, 20, 2)
        slices.append(k.reshape(list(k.shape) + [1] * 12, order="F"))
    d = str(tmp_path)
    writecfl(d + "/k", np.concatenate(slices, axis=13))
    assert 0 == cli.main(["-l", "8192", "ecalib", "-m", "1", "-k", "5", "-r", "20:20:1", d + "/k", d + "/s", d + "/e"])
    s, e = readcfl(d + "/s"), readcfl(d + "/e")
    assert s.shape[:5] == (32, 32, 1, 4, 1) and s.shape[13] == 2 and e.shape[:5] == (32, 32, 1, 1, 1)
    from bart_b200.espirit import EcalibConf
    for i, k in enumerate(slices):
        si, ei, _ = _oracle_ecalib(k, EcalibConf(maps=1, kdims=(5, 5, 5), calsize=(20, 20, 1)))
        assert np.array_equal(s[..., i, :, :].reshape(si.shape[:5], order="F"), si.reshape(si.shape[:5], order="F"))
        assert np.array_equal(e[..., i, :, :].reshape(ei.shape[:5], order="F"), ei.reshape(ei.shape[:5], order="F"))


def test_ecalib_loop_rejects_inner_dims():
    """The looped dims must lie outside the k-space's own dims 0-4."""
    from bart_b200.espirit import EcalibConf
    from bart_b200.loop import loop_ecalib
    with pytest.raises(ValueError):
        loop_ecalib(1 << 3, np.zeros((8, 8, 1, 2), dtype=np.complex64), EcalibConf())


def test_ecalib_under_torchrun_runs_on_rank_0_only(tmp_path, monkeypatch):
    """Launched with several ranks, ecalib does not split its work: ranks
    other than 0 exit without reading or writing anything."""
    d = str(tmp_path)
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    assert 0 == cli.main(["ecalib", d + "/missing", d + "/s"])
    import os
    assert not os.path.exists(d + "/s.cfl")

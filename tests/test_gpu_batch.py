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

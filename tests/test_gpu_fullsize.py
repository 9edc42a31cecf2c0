"""The configs' own sizes against the reference's own outputs.

C1: 256^2 image, 402 golden-angle spokes x 512 samples, forward NUFFT and
the adjoint of the forward's output (``bart nufft`` / ``bart nufft -a``).
C2: 256^2 CG-SENSE, 16 coils, 96 spokes x 512, 40 dB noise,
``pics -l2 -r0.01`` at 5 and 30 iterations. The fixtures hold the reference's
outputs and the seeds; the inputs are regenerated here (the k-space by the
oracle's forward model, checked against the stored checksum).
"""

import hashlib
import importlib.util
import os

import numpy as np
import pytest

from bart_b200 import synth
from bart_b200.nufft import NufftConf, nufft_create2
from bart_b200.pics import Pics, PicsConf
from conftest import GOLDEN, golden, rel

pytestmark = pytest.mark.gpu

OPS_TOL = 1e-5      # per operator apply
RECON_TOL = 1e-4    # reconstructions


def _make_golden():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes(order="F")).hexdigest()


def test_c1_forward_adjoint_fullsize():
    g = golden("nufft2d_c1_n256")
    rng = np.random.default_rng(int(g["seed"]))
    traj = synth.radial_traj(256, int(g["spokes"]))
    img = (rng.standard_normal((256, 256)) + 1j * rng.standard_normal((256, 256))).astype(np.complex64)
    assert _sha(img) == str(g["img_sha256"])
    kd = [1, 512, int(g["spokes"]), 1]
    op = nufft_create2(kd, [256, 256, 1, 1], list(traj.shape), traj, conf=NufftConf(toeplitz=False))
    try:
        fwd = np.asarray(op.forward(img.reshape(256, 256, 1, 1)))
        adj = np.asarray(op.adjoint(g["fwd"].reshape(kd, order="F")))
    finally:
        op.free()
    assert rel(fwd, g["fwd"]) < OPS_TOL
    assert rel(adj, g["adj"]) < OPS_TOL


@pytest.fixture(scope="module")
def c2():
    g = golden("pics2d_c2_n256_c16")
    traj, _, sens, ksp = _make_golden().sense_problem(int(g["N"]), int(g["C"]), int(g["spokes"]), int(g["seed"]))
    assert _sha(ksp) == str(g["ksp_sha256"]), "regenerated k-space differs from the fixture's"
    return g, traj, sens, ksp


def _pics(traj, sens, ksp, **kw):
    p = Pics(traj, sens, ksp_dims=list(ksp.shape), conf=PicsConf(lam=0.01, **kw))
    try:
        x = np.asarray(p.run(ksp))
        st = p.stats()
    finally:
        p.free()
    return x, st


def test_c2_pics_5_iterations_fullsize(c2):
    g, traj, sens, ksp = c2
    x, st = _pics(traj, sens, ksp, maxiter=5, scaling=1.0)
    assert st[0] == 5
    assert rel(x, g["x5_w1"]) < OPS_TOL


# 30 iterations leave CG unconverged (residual ~4e-4) at lambda 0.01: the
# iterates then amplify float32 rounding of every operator apply. The
# reference's own outputs move by up to 1.9e-3 between OpenMP thread counts
# (its gridding adds in thread order) and by 1.2e-3 .. 2.6e-3 between its two
# normal operators (Toeplitz and explicit) over 30 iterations, so the bar
# there is 5e-3. Run to convergence (300 iterations, residual ~2e-7) the
# solution is still sensitive to the last bit of A^H y: the reference's
# runs at 1..8 threads differ by ~4e-4, and the bar is twice that measured
# spread (the *_spread values the fixture stores).
UNCONVERGED_BAR = 5e-3


@pytest.mark.parametrize("key,kw", [("x30_w1", dict(scaling=1.0)), ("x30", dict()),
                                    ("x300_w1", dict(scaling=1.0)), ("x300", dict())])
def test_c2_pics_iterations_fullsize(c2, key, kw):
    g, traj, sens, ksp = c2
    it = int(key[1:].split("_")[0])
    x, st = _pics(traj, sens, ksp, maxiter=it, **kw)
    assert st[0] == it
    e = rel(x, g[key])
    x2, _ = _pics(traj, sens, ksp, maxiter=it, **kw)
    spread = float(g[key + "_spread"])
    drift = rel(g[key + "_notoep"], g[key]) if (key + "_notoep") in g else float("nan")
    print(f"{key}: GPU vs reference {e:.2e}, GPU run to run {rel(x2, x):.2e}, reference thread spread "
          f"{spread:.2e}, reference toeplitz vs explicit {drift:.2e}, residual {st[1]:.2e}")
    if it >= 300:
        assert st[1] < 1e-5                     # converged
        assert e < 2 * spread
    else:
        assert e < UNCONVERGED_BAR

"""3D radial kooshball NUFFT on the GPU: the reference's outputs at 32^3, the
oracle at 64^3 with 8 coils, and size-independent properties at the full
128^3 / 8-coil / 20000 x 256 configuration.

Bar: relative L2 <= 1e-5 per operator apply against the reference and the
oracle; at full size, adjointness <A x, y> = <x, A^H y> to 1e-5 and the
default (output-stationary) scatter against the global-atomic scatter to
1e-6 (same sums, other float32 order).
"""

import hashlib

import numpy as np
import pytest

from bart_b200 import synth
from bart_b200.nufft import NufftConf, nufft_create2
from conftest import golden, rel
from oracle import nufft_oracle as orc

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _cplx(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes(order="F")).hexdigest()


def test_kooshball_32_vs_reference():
    g = golden("nufft3d_n32_c2")
    rng = np.random.default_rng(int(g["seed"]))
    traj = synth.kooshball_traj(32, 400)
    img = _cplx(rng, (32, 32, 32, 2))
    ksp = _cplx(rng, (1, 64, 400, 2))
    assert _sha(img) == str(g["img_sha256"]) and _sha(ksp) == str(g["ksp_sha256"])
    cd, kd = [32, 32, 32, 2], [1, 64, 400, 2]
    op = nufft_create2(kd, cd, list(traj.shape), traj, conf=NufftConf(toeplitz=True))
    try:
        assert rel(op.forward(img), g["fwd"]) < TOL
        assert rel(op.adjoint(ksp), g["adj"]) < TOL
        assert rel(op.normal(img), g["normal"]) < TOL
    finally:
        op.free()


def test_kooshball_64_eight_coils_vs_oracle():
    """64^3, 8 coils, 1000 spokes x 128: the multi-coil 3D scatter (the
    output-stationary kernel) and gather against the FP64 oracle."""
    import torch
    rng = np.random.default_rng(64)
    N, C = 64, 8
    traj = synth.kooshball_traj(N, 1000)
    M = traj.shape[1] * traj.shape[2]
    img = _cplx(rng, (N, N, N, C))
    y = _cplx(rng, (1, traj.shape[1], traj.shape[2], C))
    cd, kd = [N, N, N, C], [1, traj.shape[1], traj.shape[2], C]
    dev = torch.device("cuda:0")

    def d(a):
        return torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).to(dev)

    op = nufft_create2(kd, cd, list(traj.shape), d(traj), conf=NufftConf(toeplitz=False))
    try:
        fwd = op.forward(d(img)).cpu().numpy()
        adj = op.adjoint(d(y)).cpu().numpy()
    finally:
        op.free()
    o = orc.NufftOracle(traj.real.reshape(3, -1, order="F"), (N, N, N))
    assert rel(fwd, o.forward(img)) < TOL
    assert rel(adj, o.adjoint(y.reshape(M, C, order="F")).ravel(order="F")) < TOL


def test_kooshball_full_size_properties(monkeypatch):
    """The config's own size: 128^3, 8 coils, 20000 x 256 golden-means
    kooshball (5.12 M samples per coil). <A x, y> = <x, A^H y> in float64
    sums of the GPU's float32 outputs, and the default scatter equals the
    global-atomic one (an explicit bin edge selects it) to float32 order."""
    import torch
    rng = np.random.default_rng(128)
    N, C = 128, 8
    traj = synth.kooshball_traj(N, 20000)
    dev = torch.device("cuda:0")
    t_d = torch.from_numpy(np.asfortranarray(traj).ravel(order="F").copy()).to(dev)
    M = traj.shape[1] * traj.shape[2]
    cd, kd = [N, N, N, C], [1, traj.shape[1], traj.shape[2], C]
    gen = torch.Generator(device=dev).manual_seed(5)
    x = torch.randn(N ** 3 * C, dtype=torch.complex64, device=dev, generator=gen)
    y = torch.randn(M * C, dtype=torch.complex64, device=dev, generator=gen)
    monkeypatch.delenv("BNUFFT_GRIDDING", raising=False)
    op = nufft_create2(kd, cd, list(traj.shape), t_d, conf=NufftConf(toeplitz=False))
    ref = nufft_create2(kd, cd, list(traj.shape), t_d, conf=NufftConf(toeplitz=False, bin=16))
    try:
        ax = op.forward(x)
        ahy = op.adjoint(y)
        ahy_atomic = ref.adjoint(y)
        lhs = torch.vdot(y.to(torch.complex128), ax.to(torch.complex128))
        rhs = torch.vdot(ahy.to(torch.complex128), x.to(torch.complex128))
        assert abs(complex(lhs - rhs)) / abs(complex(lhs)) < TOL
        assert float(torch.linalg.vector_norm(ahy - ahy_atomic) / torch.linalg.vector_norm(ahy_atomic)) < 1e-6
    finally:
        op.free()
        ref.free()

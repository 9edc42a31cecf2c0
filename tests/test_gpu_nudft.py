"""GPU direct NDFT (bart nufft -s) against the reference and the FP64 oracle."""

import numpy as np
import pytest

from bart_b200 import synth
from bart_b200.nufft import Nudft
from conftest import golden, rel
from oracle import nufft_oracle as orc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["nudft2d_n24", "nudft2d_n16_coils2"])
def test_nudft_vs_reference(name):
    """The reference forms its phases in float32; the GPU's are float64-exact,
    so they agree to the reference's phase rounding (the FP64 oracle agrees
    with the reference to the same bar)."""
    g = golden(name)
    img = g["img"]
    cd = list(img.shape) + [1] * (4 - img.ndim)
    td = list(g["traj"].shape)
    kd = [1, td[1], td[2], cd[3]]
    op = Nudft(kd, cd, td, g["traj"])
    assert rel(op.forward(img.reshape(cd, order="F")), g["fwd"]) < 2e-5
    assert rel(op.adjoint(g["ksp"].reshape(kd, order="F")), g["adj"]) < 2e-5
    op.free()


@pytest.mark.parametrize("N,nd,coils", [(32, 2, 3), (10, 3, 2)])
def test_nudft_vs_fp64_oracle(N, nd, coils):
    rng = np.random.default_rng(N + coils)
    t = synth.radial_traj(N, 12) if nd == 2 else synth.kooshball_traj(N, 40)
    Z = 1 if nd == 2 else N
    cd = [N, N, Z, coils]
    img = (rng.standard_normal(cd) + 1j * rng.standard_normal(cd)).astype(np.complex64, order="F")
    kd = [1, t.shape[1], t.shape[2], coils]
    op = Nudft(kd, cd, list(t.shape), t)
    tr = t.real.reshape(3, -1, order="F")
    s = 1.0 / np.sqrt(coils)    # the reference's scale counts the coils
    assert rel(op.forward(img), orc.ndft_forward(tr, img) * s) < 1e-5
    y = (rng.standard_normal((tr.shape[1], coils)) + 1j * rng.standard_normal((tr.shape[1], coils))).astype(np.complex64)
    assert rel(op.adjoint(y.reshape(kd, order="F")), orc.ndft_adjoint(tr, y, (N, N, Z)) * s) < 1e-5
    op.free()

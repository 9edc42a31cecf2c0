"""Host-side logic: .cfl I/O, synthetic inputs, CLI dimension rules."""

import numpy as np

from bart_b200 import synth
from bart_b200.__main__ import estimate_im_dims
from bart_b200.cfl import readcfl, writecfl


def test_cfl_roundtrip(tmp_path):
    a = (np.arange(24) + 1j * np.arange(24)).astype(np.complex64).reshape(2, 3, 4, order="F")
    writecfl(str(tmp_path / "a"), a)
    b = readcfl(str(tmp_path / "a"))
    assert b.shape[:3] == (2, 3, 4) and all(d == 1 for d in b.shape[3:])
    assert np.array_equal(b.reshape(2, 3, 4, order="F"), a)
    hdr = open(str(tmp_path / "a.hdr")).read().split("\n")
    assert hdr[0] == "# Dimensions" and len(hdr[1].split()) == 16


def test_radial_traj_layout():
    t = synth.radial_traj(256, 402)
    assert t.shape == (3, 512, 402)
    assert np.isclose(t.real.max(), 127.75, atol=1e-3) and np.isclose(t.real.min(), -127.75, atol=1e-3)
    assert np.all(t.imag == 0) and np.all(t[2] == 0)


def test_synthetic_problem_is_seeded():
    a = synth.coil_maps(32, 4, np.random.default_rng(1))
    b = synth.coil_maps(32, 4, np.random.default_rng(1))
    assert np.array_equal(a, b)
    rss = np.sqrt(np.sum(np.abs(a) ** 2, axis=-1))
    assert np.allclose(rss, 1.0, atol=1e-5)
    p = synth.ellipse_phantom(64, 20, np.random.default_rng(2))
    assert p.shape == (64, 64, 1) and np.abs(p).max() > 0


def test_kooshball_directions_are_unit():
    t = synth.kooshball_traj(16, 100)
    d = t.real[:, -1, :] / np.abs(t.real[:, -1, :]).max()
    n = np.linalg.norm(t.real[:, -1, :], axis=0)
    assert np.allclose(n, n[0], rtol=1e-5)


def test_estimate_im_dims():
    t = synth.radial_traj(64, 8)
    assert estimate_im_dims(t) == [2 * int(np.ceil(np.abs(t.real[0]).max())), 2 * int(np.ceil(np.abs(t.real[1]).max())), 1]


def test_stream_reader_on_the_reference_stream():
    """bart_b200.stream reads a stream the reference wrote (copy --stream
    8192 | tee -b: header, settings, then index / raw / break per slice):
    every slice arrives once, at its position, with the array's values."""
    import io
    from bart_b200.stream import StreamReader
    from conftest import golden
    g = golden("stream_ksp_c4_s3")
    r = StreamReader(io.BytesIO(g["stream"].tobytes()))
    assert r.binary and r.flags == 8192 and r.dims[13] == 3
    seen = []
    for index, pos, block in r:
        seen.append(index)
        assert np.array_equal(block[..., 0, 0].reshape(block.shape[:4], order="F"),
                              g["ksp"][..., pos[0]].reshape(block.shape[:4], order="F"))
    assert seen == [0, 1, 2]

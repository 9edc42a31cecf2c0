"""Allocation-free forward NUFFT (bnufft_forward2d_noalloc) through the C ABI.

The entry point serves callers that cannot allocate device memory while they
run (fixed device-memory budgets, no mid-stream cudaMalloc); its scratch is a
file-scope device array shared by all calls. It must agree with the regular
plan-based forward NUFFT on two calls in a row (the second call finds the
first call's data in the shared array). This file is named so that pytest
collects it last.
"""

import ctypes

import numpy as np
import pytest

from bart_b200 import _lib, synth
from bart_b200.nufft import NufftConf, nufft_create2
from conftest import rel

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _dev(a, device):
    import torch
    return torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).to(device)


def _traj(X, Y, spokes):
    readout = max(X, Y)
    t = synth.radial_traj(readout, spokes)
    t[0] *= X / readout
    t[1] *= Y / readout
    return t


def _call(lib, X, Y, M, traj_d, img_d, out):
    import torch
    return lib.bnufft_forward2d_noalloc(X, Y, M, ctypes.c_void_p(traj_d.data_ptr()),
                                        ctypes.c_void_p(img_d.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


# every grid length the entry point dispatches (2X, 2Y = 16 .. 512), square,
# wide (X > Y) and tall images, and fewer rows than a row block holds
@pytest.mark.parametrize("X,Y,spokes", [(256, 256, 402), (64, 128, 40), (8, 8, 4), (16, 64, 10), (128, 32, 20),
                                        (32, 16, 12)])
def test_noalloc_forward_matches_plan_forward(cuda, X, Y, spokes):
    import torch
    lib = _lib.load()
    rng = np.random.default_rng(X + Y)
    t = _traj(X, Y, spokes)
    M = t.shape[1] * t.shape[2]
    op = nufft_create2([1, t.shape[1], t.shape[2], 1], [X, Y, 1, 1], list(t.shape), t,
                       conf=NufftConf(toeplitz=False))
    traj_d = _dev(t, cuda)
    out = torch.empty(M, dtype=torch.complex64, device=cuda)
    for call in range(2):
        img = (rng.standard_normal((X, Y)) + 1j * rng.standard_normal((X, Y))).astype(np.complex64)
        img_d = _dev(img, cuda)
        want = op.forward(img_d)
        out.fill_(float("nan"))
        _lib.check(_call(lib, X, Y, M, traj_d, img_d, out))
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got)), f"call {call}"
        assert rel(got, want.cpu().numpy()) < TOL, f"call {call}"
    op.free()


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    import torch
    lib = _lib.load()
    buf = torch.zeros(16, dtype=torch.complex64, device=cuda)
    p = ctypes.c_void_p(buf.data_ptr())
    assert lib.bnufft_forward2d_noalloc(512, 512, 4, p, p, p, None) == 1
    assert "image side" in lib.bnufft_last_error().decode()
    assert lib.bnufft_forward2d_noalloc(64, 64, 262145, p, p, p, None) == 1
    assert "samples" in lib.bnufft_last_error().decode()


def test_noalloc_allocates_no_device_memory(cuda):
    """The property the entry point exists for: once set up, calls take no
    device memory. The device's free memory (cudaMemGetInfo) is the same
    before and after two calls in a row; everything else is synchronised
    first, so that no stream-ordered free of other work lands in between."""
    import torch
    lib = _lib.load()
    X, Y, spokes = 128, 128, 64
    t = _traj(X, Y, spokes)
    M = t.shape[1] * t.shape[2]
    rng = np.random.default_rng(7)
    img = (rng.standard_normal((X, Y)) + 1j * rng.standard_normal((X, Y))).astype(np.complex64)
    traj_d, img_d = _dev(t, cuda), _dev(img, cuda)
    out = torch.empty(M, dtype=torch.complex64, device=cuda)
    _lib.check(_call(lib, X, Y, M, traj_d, img_d, out))     # set-up and the kernels' first use
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    free0, _ = torch.cuda.mem_get_info(cuda)
    stats0 = torch.cuda.memory_stats(cuda).get("allocation.all.allocated", 0)
    for _ in range(2):
        _lib.check(_call(lib, X, Y, M, traj_d, img_d, out))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(cuda)
    assert free1 >= free0, f"free device memory fell by {free0 - free1} bytes"
    assert torch.cuda.memory_stats(cuda).get("allocation.all.allocated", 0) == stats0

"""Batches of independent CG-SENSE reconstructions of uneven size.

Many slices or frames (each its own matrix size, trajectory, coil count and
maps) are reconstructed by one launch of one CUDA graph in which every
problem's whole solve is an independent child graph
(``bnufft_batch_create``); the GPU runs them concurrently instead of one
small solve after another. ``run_loop`` is the baseline: a loop of single
solves on the same GPU.

Gridding bin sizes are picked per matrix size by ``autotune_bins``: for a
few sizes spanning the batch it times the model set-up and one solve with
each candidate bin edge and keeps the fastest, then uses the nearest tuned
size for every problem.
"""

from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _lib
from .pics import Pics, PicsConf
from .problems import cgsense_problem


def uneven_problems(n, seed, sizes=(64, 320), spokes=(16, 256), coils=(4, 32), snr_db=40.0, forward=None):
    """n problems: N ~ U{even sizes}, spokes ~ U, 2N samples per spoke, coils ~ U.
    The first k problems of any n are the same (one random stream, drawn in
    order); ``forward`` as in problems.simulate_ksp."""
    rng = np.random.default_rng(seed)
    evens = np.arange(sizes[0], sizes[1] + 1, 2)
    out = []
    for _ in range(n):
        N = int(rng.choice(evens))
        out.append(cgsense_problem(rng, N=N, coils=coils, spokes=spokes, snr_db=snr_db, forward=forward))
    return out


def _dev(a, dev):
    import torch
    return torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy()).to(dev)


class BatchRecon:
    """Device copies of the problems, one Pics model each, output images, and
    the batch graph over them."""

    def __init__(self, problems, dev, lam=0.01, maxiter=20, bins=None, **conf_kw):
        import torch
        self.dev = dev
        self.models, self.ksp, self.img, self._keep = [], [], [], []
        for prob in problems:
            traj, sens, ksp = prob["traj"], prob["sens"], prob["ksp"]
            N = sens.shape[0]
            npix = int(np.prod(sens.shape[:3]))
            conf = PicsConf(lam=lam, maxiter=maxiter, toeplitz=True, bin=pick_bin(bins, N), **conf_kw)
            td, sd = _dev(traj, dev), _dev(sens, dev)
            p = Pics(td, sd, ksp_dims=list(ksp.shape), conf=conf, traj_dims=list(traj.shape), sens_dims=list(sens.shape))
            self.models.append(p)
            self.ksp.append(_dev(ksp, dev))
            self.img.append(torch.empty(npix, dtype=torch.complex64, device=dev))
        self.batch = None

    def build(self):
        """Capture the batch graph (once)."""
        n = len(self.models)
        hs = (ctypes.c_void_p * n)(*[m._h.value for m in self.models])
        im = (ctypes.c_void_p * n)(*[t.data_ptr() for t in self.img])
        ks = (ctypes.c_void_p * n)(*[t.data_ptr() for t in self.ksp])
        h = ctypes.c_void_p()
        _lib.check(_lib.load().bnufft_batch_create(ctypes.byref(h), hs, n, im, ks, None))
        self.batch = h
        return self

    def kernels(self):
        return _lib.load().bnufft_batch_kernels(self.batch)

    def run(self, stream=None):
        """All reconstructions, one graph launch."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream(self.dev).cuda_stream
        _lib.check(_lib.load().bnufft_batch_run(self.batch, ctypes.c_void_p(s)))

    def run_loop(self):
        """The baseline: one single solve after another."""
        for p, k, x in zip(self.models, self.ksp, self.img):
            p.run(k, out=x)

    def free(self):
        if self.batch is not None:
            _lib.load().bnufft_batch_free(self.batch)
            self.batch = None
        for p in self.models:
            p.free()
        self.models = []


def pick_bin(bins, N):
    """Tuned bin edge of the tuned size nearest to N (0 = library default)."""
    if not bins:
        return 0
    k = min(bins, key=lambda n: abs(int(n) - N))
    return int(bins[k])


def autotune_bins(dev, sizes=(64, 128, 192, 256, 320), candidates=(8, 16, 32, 64), coils=16, spokes=128, reps=3,
                  seed=0):
    """Bin edge per matrix size: the fastest model set-up + one 20-iteration
    solve (the bin size changes only the gridding order, never results)."""
    import torch
    rng = np.random.default_rng(seed)
    table, detail = {}, {}
    for N in sizes:
        prob = cgsense_problem(rng, N=N, coils=coils, spokes=spokes)
        td, sd, kd = _dev(prob["traj"], dev), _dev(prob["sens"], dev), _dev(prob["ksp"], dev)
        times = {}
        for b in candidates:
            conf = PicsConf(lam=0.01, maxiter=20, toeplitz=True, bin=b)
            best = float("inf")
            for _ in range(reps):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                p = Pics(td, sd, ksp_dims=list(prob["ksp"].shape), conf=conf, traj_dims=list(prob["traj"].shape),
                         sens_dims=list(prob["sens"].shape))
                p.run(kd)
                torch.cuda.synchronize()
                best = min(best, time.perf_counter() - t0)
                p.free()
            times[b] = best * 1e3
        table[N] = min(times, key=times.get)
        detail[N] = times
    return table, detail

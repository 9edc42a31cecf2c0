"""NUFFT linop with the reference's interface, backed by libbnufft.

Mirrors ``nufft_create2`` (src/noncart/nufft.h:48-57) and the linop
callbacks forward / adjoint / normal (src/linops/linop.h). Arrays are BART
arrays: numpy arrays in column-major order, or torch tensors whose memory
holds the column-major data (any contiguous complex64 tensor of the right
size). Host arrays are staged by the library; device tensors are used in
place on the current torch stream.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .cfl import dims16


@dataclass
class NufftConf:
    """struct nufft_conf_s subset (src/noncart/nufft.h:7-30)."""
    toeplitz: bool = True
    periodic: bool = False
    deterministic: bool = False
    os: float = 2.0
    width: float = 6.0
    bin: int = 0              # gridding bin edge (0 = default); tuning only
    lowmem: bool = False      # --lowmem: one coil's grid at a time

    def c(self) -> _lib.NufftConfC:
        return _lib.NufftConfC(int(self.toeplitz), int(self.periodic), int(self.deterministic),
                               float(self.os), float(self.width), int(self.bin), int(self.lowmem))


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def _stream_of(*arrays):
    for a in arrays:
        if _is_torch(a) and a.is_cuda:
            import torch
            return ctypes.c_void_p(torch.cuda.current_stream(a.device).cuda_stream)
    return None


def _ptr_in(a, n: int):
    """(pointer, keepalive) of an input array holding n complex64 values."""
    if _is_torch(a):
        import torch
        if a.dtype != torch.complex64 or not a.is_contiguous() or a.numel() != n:
            raise ValueError(f"expected contiguous complex64 tensor with {n} values")
        return ctypes.c_void_p(a.data_ptr()), a
    arr = np.asarray(a)
    if arr.size != n:
        raise ValueError(f"expected {n} values, got {arr.size}")
    arr = np.asfortranarray(arr.astype(np.complex64, copy=False))
    return ctypes.c_void_p(arr.ctypes.data), arr


def _ptr_out(a, n: int):
    if _is_torch(a):
        import torch
        if a.dtype != torch.complex64 or not a.is_contiguous() or a.numel() != n:
            raise ValueError(f"expected contiguous complex64 tensor with {n} values")
        return ctypes.c_void_p(a.data_ptr())
    if not (isinstance(a, np.ndarray) and a.dtype == np.complex64 and a.flags.f_contiguous and a.size == n):
        raise ValueError("output must be an F-contiguous complex64 numpy array")
    return ctypes.c_void_p(a.ctypes.data)


def _alloc_like(src, dims):
    n = int(np.prod(dims))
    if _is_torch(src):
        import torch
        return torch.empty(n, dtype=torch.complex64, device=src.device)
    return np.zeros(dims, dtype=np.complex64, order="F")


class Linop:
    """Forward / adjoint / normal operator pair (struct linop_s)."""

    def __init__(self, handle, domain_dims, codomain_dims, has_normal):
        self._h = handle
        self.domain_dims = list(domain_dims)
        self.codomain_dims = list(codomain_dims)
        self.has_normal = has_normal

    def _call(self, fn, src, dst, in_dims, out_dims):
        if self._h is None:
            raise RuntimeError("linop was freed")
        nin, nout = int(np.prod(in_dims)), int(np.prod(out_dims))
        if dst is None:
            dst = _alloc_like(src, out_dims)
        ps, keep = _ptr_in(src, nin)
        pd = _ptr_out(dst, nout)
        _lib.check(fn(self._h, pd, ps, _stream_of(src, dst)))
        del keep
        return dst

    def forward(self, src, dst=None):
        """linop_forward: domain (coil images) -> codomain (k-space)."""
        return self._call(_lib.load().bnufft_apply_forward, src, dst, self.domain_dims, self.codomain_dims)

    def adjoint(self, src, dst=None):
        """linop_adjoint: codomain -> domain."""
        return self._call(_lib.load().bnufft_apply_adjoint, src, dst, self.codomain_dims, self.domain_dims)

    def normal(self, src, dst=None):
        """linop_normal: domain -> domain (Toeplitz when the plan has a PSF)."""
        return self._call(_lib.load().bnufft_apply_normal, src, dst, self.domain_dims, self.domain_dims)

    def inverse(self, ksp, lam=0.0, maxiter=50, precond=False, dst=None):
        """``bart nufft -i [-c] -l lam -m maxiter``: CG over the coil images
        on (N^H N + lam) x = N^H y, optionally with the reference's circulant
        preconditioner (needs the Toeplitz PSF)."""
        if self._h is None:
            raise RuntimeError("linop was freed")
        nin, nout = int(np.prod(self.codomain_dims)), int(np.prod(self.domain_dims))
        if dst is None:
            dst = _alloc_like(ksp, self.domain_dims)
        pk, keep = _ptr_in(ksp, nin)
        pd = _ptr_out(dst, nout)
        _lib.check(_lib.load().bnufft_nufft_inverse(self._h, pd, pk, float(lam), int(maxiter), int(precond),
                                                    _stream_of(ksp, dst)))
        del keep
        return dst

    def psf(self):
        """nufft_get_psf: the Toeplitz PSF in the reference's decomposed layout."""
        lib = _lib.load()
        nd = len(self.domain_dims) + 1
        d = (ctypes.c_long * nd)()
        _lib.check(lib.bnufft_get_psf_dims(self._h, nd, d))
        dims = list(d)
        out = np.zeros(dims, dtype=np.complex64, order="F")
        _lib.check(lib.bnufft_get_psf(self._h, nd, d, ctypes.c_void_p(out.ctypes.data), None))
        return out

    def update_traj(self, traj):
        """nufft_update_traj with a trajectory of the same dims."""
        lib = _lib.load()
        t = np.asarray(traj) if not _is_torch(traj) else traj
        tdims = dims16(t.shape) if not _is_torch(traj) else self._traj_dims
        pt, keep = _ptr_in(t, int(np.prod(tdims)))
        _lib.check(lib.bnufft_update_traj(self._h, len(tdims), _lib.dims_array(tdims), pt, _stream_of(traj)))
        del keep

    def free(self):
        """linop_free."""
        if self._h is not None:
            _lib.load().bnufft_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def nufft_create2(ksp_dims, cim_dims, traj_dims, traj, wgh_dims=None, weights=None,
                  bas_dims=None, basis=None, conf: NufftConf | None = None) -> Linop:
    """nufft_create2 (src/noncart/nufft.c:1174): NUFFT linop for a trajectory.

    ``traj`` is the reference's [3, Mr, Ms] complex64 trajectory (numpy, or a
    torch tensor on the device). ``weights`` (density compensation / sampling
    pattern, ``bart nufft -p``) is [1, Mr, Ms] or [1, Mr, Ms, C]; with the
    Toeplitz PSF it must be shared by all channels. ``basis`` (``bart nufft
    -B``) is [1, 1, 1, 1, 1, T, K]: then cim_dims has K coefficients in dim 6,
    ksp_dims T frames in dim 5, the trajectory 1 or T frames in dim 5 and the
    weights [1, Mr, Ms, 1, 1, T or 1].
    """
    lib = _lib.load()
    conf = conf or NufftConf()
    kd, cd, td = dims16(ksp_dims), dims16(cim_dims), dims16(traj_dims)
    pt, keep = _ptr_in(traj, int(np.prod(td)))
    wd_arr, pw, keep_w = None, None, None
    if weights is not None:
        wd = dims16(wgh_dims if wgh_dims is not None else np.shape(weights))
        wd_arr = _lib.dims_array(wd)
        pw, keep_w = _ptr_in(weights, int(np.prod(wd)))
    bd_arr, pb, keep_b = None, None, None
    if basis is not None:
        bd = dims16(bas_dims if bas_dims is not None else np.shape(basis))
        bd_arr = _lib.dims_array(bd)
        pb, keep_b = _ptr_in(basis, int(np.prod(bd)))
    h = ctypes.c_void_p()
    cc = conf.c()
    _lib.check(lib.bnufft_create2(ctypes.byref(h), 16, _lib.dims_array(kd), _lib.dims_array(cd),
                                  _lib.dims_array(td), pt, wd_arr, pw, bd_arr, pb, ctypes.byref(cc),
                                  _stream_of(traj)))
    del keep, keep_w, keep_b
    if basis is not None:   # the k-space has the basis' frames and no coefficient dim
        kd = list(kd)
        kd[5], kd[6] = bd[5], 1
    op = Linop(h, cd, kd, has_normal=True)
    op._traj_dims = td
    return op


def nufft_create(ksp_dims, cim_dims, traj_dims, traj, weights=None, conf: NufftConf | None = None) -> Linop:
    """nufft_create (src/noncart/nufft.c:1315): weights share the traj dims."""
    wd = None if weights is None else [1] + list(dims16(traj_dims))[1:]
    return nufft_create2(ksp_dims, cim_dims, traj_dims, traj, wd, weights, None, None, conf)


class Nudft:
    """nudft_create (src/noncart/nudft.c:331): the exact non-uniform DFT as a
    linop (``bart nufft -s``), scaled like the reference (1/sqrt of all image
    dims, coils included)."""

    def __init__(self, ksp_dims, cim_dims, traj_dims, traj):
        lib = _lib.load()
        kd, cd, td = dims16(ksp_dims), dims16(cim_dims), dims16(traj_dims)
        pt, keep = _ptr_in(traj, int(np.prod(td)))
        h = ctypes.c_void_p()
        _lib.check(lib.bnufft_nudft_create(ctypes.byref(h), 16, _lib.dims_array(kd), _lib.dims_array(cd),
                                           _lib.dims_array(td), pt, _stream_of(traj)))
        del keep
        self._h = h
        self.domain_dims, self.codomain_dims = cd, kd

    def _call(self, fn, src, dst, in_dims, out_dims):
        nin, nout = int(np.prod(in_dims)), int(np.prod(out_dims))
        if dst is None:
            dst = _alloc_like(src, out_dims)
        ps, keep = _ptr_in(src, nin)
        _lib.check(fn(self._h, _ptr_out(dst, nout), ps, _stream_of(src, dst)))
        del keep
        return dst

    def forward(self, src, dst=None):
        return self._call(_lib.load().bnufft_nudft_apply_forward, src, dst, self.domain_dims, self.codomain_dims)

    def adjoint(self, src, dst=None):
        return self._call(_lib.load().bnufft_nudft_apply_adjoint, src, dst, self.codomain_dims, self.domain_dims)

    def free(self):
        if getattr(self, "_h", None) is not None:
            _lib.load().bnufft_nudft_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

"""ESPIRiT calibration of coil sensitivities, ``bart ecalib``, through the
library's C ABI (include/bespirit.h).

``ecalib(ksp, conf)`` takes Cartesian k-space ``[X, Y, Z, C]`` (a NumPy array
in BART order, or a contiguous complex64 CUDA tensor with its dims) and
returns the maps ``[X, Y, Z, C, maps]``, their eigenvalues ``[X, Y, Z, 1,
maps]`` and the calibration facts (singular values, kernels kept,
calibration region). The options and defaults are main_ecalib's
(src/ecalib.c:64-97, src/calib/calib.c:693-714).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .nufft import _is_torch


@dataclass
class EcalibConf:
    kdims: tuple = (6, 6, 6)		# -k
    calsize: tuple = (24, 24, 24)	# -r
    maps: int = 2			# -m
    threshold: float = 0.001		# -t
    numsv: int = -1			# -n
    percentsv: float = -1.0		# -p
    crop: float = 0.8			# -c
    softcrop: bool = False		# -S
    rotphase: bool = True		# -P clears
    num_orthiter: int = 30
    intensity: bool = False		# -I
    # not built (the call fails with BNUFFT_ERR_UNSUPPORTED)
    weighting: bool = False		# -W
    phase_normalize: bool = False	# -N
    nystroem: bool = False		# -A
    orthiter: bool = True		# hidden -O clears

    def to_c(self) -> _lib.EcalibConfC:
        c = _lib.EcalibConfC()
        _lib.load().bnufft_ecalib_defaults(ctypes.byref(c))
        for i in range(3):
            c.kdims[i] = int(self.kdims[i])
            c.calsize[i] = int(self.calsize[i])
        c.maps = int(self.maps)
        c.threshold = float(self.threshold)
        c.numsv = int(self.numsv)
        c.percentsv = float(self.percentsv)
        c.crop = float(self.crop)
        c.softcrop = int(bool(self.softcrop))
        c.rotphase = int(bool(self.rotphase))
        c.num_orthiter = int(self.num_orthiter)
        c.weighting = int(bool(self.weighting))
        c.intensity = int(bool(self.intensity))
        c.phase_normalize = int(bool(self.phase_normalize))
        c.nystroem = int(bool(self.nystroem))
        c.orthiter = int(bool(self.orthiter))
        return c


def output_dims(ksp_dims, conf: EcalibConf | None = None):
    """(sens dims, emaps dims), 16 each."""
    conf = conf or EcalibConf()
    kd = _lib.dims_array(list(ksp_dims) + [1] * (16 - len(ksp_dims)))
    sd, ed = _lib.dims_array([1] * 16), _lib.dims_array([1] * 16)
    _lib.check(_lib.load().bnufft_ecalib_dims(ctypes.byref(conf.to_c()), 16, kd, sd, ed))
    return list(sd), list(ed)


def ecalib(ksp, conf: EcalibConf | None = None, dims=None, emaps: bool = True, stream=None, out=None):
    """(sens, emaps or None, info). ``dims`` is required for a torch tensor
    (BART order); outputs are NumPy arrays (F order) for NumPy input and
    flat CUDA tensors for tensor input. ``out`` (NumPy input only): a pair
    (sens, emaps or None) of F-contiguous complex64 arrays of the output
    shapes to write into (e.g. views of pinned host memory). info:
    ``svals`` (descending), ``nkernels``, ``caldims``."""
    conf = conf or EcalibConf()
    lib = _lib.load()
    if _is_torch(ksp):
        import torch
        if dims is None:
            raise ValueError("dims are required for a tensor")
        kdims = list(dims) + [1] * (16 - len(dims))
        if ksp.dtype != torch.complex64 or not ksp.is_contiguous() or ksp.numel() != int(np.prod(kdims)):
            raise ValueError("expected a contiguous complex64 tensor matching dims")
        sd, ed = output_dims(kdims, conf)
        sens = torch.empty(int(np.prod(sd)), dtype=torch.complex64, device=ksp.device)
        ev = torch.empty(int(np.prod(ed)), dtype=torch.complex64, device=ksp.device) if emaps else None
        pk, ps = ctypes.c_void_p(ksp.data_ptr()), ctypes.c_void_p(sens.data_ptr())
        pe = ctypes.c_void_p(ev.data_ptr()) if emaps else None
        st = stream if stream is not None else ctypes.c_void_p(torch.cuda.current_stream(ksp.device).cuda_stream)
        keep = ksp
    else:
        arr = np.asfortranarray(np.asarray(ksp).astype(np.complex64, copy=False))
        kdims = list(arr.shape) + [1] * (16 - arr.ndim)
        sd, ed = output_dims(kdims, conf)
        if out is not None:
            sens, ev = out
            for a_, d_ in ((sens, sd), (ev, ed)):
                if a_ is not None and not (a_.dtype == np.complex64 and a_.flags.f_contiguous
                                           and a_.size == int(np.prod(d_))):
                    raise ValueError("ecalib: out arrays must be F-contiguous complex64 of the output sizes")
            emaps = ev is not None
        else:
            sens = np.zeros(sd, dtype=np.complex64, order="F")
            ev = np.zeros(ed, dtype=np.complex64, order="F") if emaps else None
        pk, ps = ctypes.c_void_p(arr.ctypes.data), ctypes.c_void_p(sens.ctypes.data)
        pe = ctypes.c_void_p(ev.ctypes.data) if emaps else None
        st = stream
        keep = arr
    ncol = int(np.prod([1 if kdims[i] == 1 else conf.kdims[i] for i in range(3)])) * int(kdims[3])
    sv = (ctypes.c_float * max(ncol, 1))()
    nk = ctypes.c_long(0)
    cd = (ctypes.c_long * 3)()
    _lib.check(lib.bnufft_ecalib(ctypes.byref(conf.to_c()), 16, _lib.dims_array(kdims), pk, ps, pe, sv,
                                 ctypes.byref(nk), cd, st))
    del keep
    info = {"svals": np.array(sv[:ncol], dtype=np.float32), "nkernels": int(nk.value), "caldims": tuple(cd)}
    return sens, ev, info


def calone(ksp, conf: EcalibConf | None = None):
    """``ecalib -1``: (the kernels' low-resolution covariance [xh, yh, zh,
    C(C+1)/2] as a NumPy array, info) for NumPy k-space in BART order."""
    conf = conf or EcalibConf()
    lib = _lib.load()
    arr = np.asfortranarray(np.asarray(ksp).astype(np.complex64, copy=False))
    kdims = list(arr.shape) + [1] * (16 - arr.ndim)
    kd = [1 if kdims[i] == 1 else int(conf.kdims[i]) for i in range(3)]
    C = int(kdims[3])
    cov = np.zeros([1 if k == 1 else 2 * k for k in kd] + [C * (C + 1) // 2], dtype=np.complex64, order="F")
    ncol = int(np.prod(kd)) * C
    sv = (ctypes.c_float * max(ncol, 1))()
    nk = ctypes.c_long(0)
    cd = (ctypes.c_long * 3)()
    _lib.check(lib.bnufft_calone(ctypes.byref(conf.to_c()), 16, _lib.dims_array(kdims), ctypes.c_void_p(arr.ctypes.data),
                                 ctypes.c_void_p(cov.ctypes.data), sv, ctypes.byref(nk), cd, None))
    return cov, {"svals": np.array(sv[:ncol], dtype=np.float32), "nkernels": int(nk.value), "caldims": tuple(cd)}

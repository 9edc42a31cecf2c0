"""CG-SENSE reconstruction: ``bart pics -l2 -r lambda -i iter -t traj``.

Mirrors the CG branch of main_pics (src/pics.c:499-760): data scaling from
the adjoint (estimate_scaling_norm, src/sense/optcom.c:74-109) unless a
scaling is given, then CG (src/iter/italgos.c:497-572) on
(A^H A + lambda I) x = A^H y with A = NUFFT o maps, run entirely on the GPU by
libbnufft.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .cfl import dims16
from .nufft import _alloc_like, _ptr_in, _ptr_out, _stream_of


@dataclass
class PicsConf:
    lam: float = 0.0          # -r
    maxiter: int = 30         # -i
    tol: float = 0.0
    scaling: float = 0.0      # -w (0 = estimate)
    rescale: bool = False     # -S
    toeplitz: bool = True     # --no-toeplitz clears it
    periodic: bool = False
    deterministic: bool = False
    bin: int = 0              # gridding bin edge (0 = default); tuning only
    precond: int = 0          # 0 plain CG, 1 FCG + circulant, 2 FCG + padded circulant + learned, 3 FCG + padded circulant
    ref_scalars: bool = True  # plain CG keeps its scalars in float32 as the reference's conjgrad does
    net_iters: int = 1        # precond 2: iterations that use the learned term (0 = until it stalls)

    def c(self) -> _lib.PicsConfC:
        return _lib.PicsConfC(float(self.lam), int(self.maxiter), float(self.tol), float(self.scaling),
                              int(self.rescale), int(self.toeplitz), int(self.periodic), int(self.deterministic),
                              int(self.bin), int(self.precond), int(self.ref_scalars), int(self.net_iters))


class Pics:
    """A SENSE model for one trajectory and one set of maps, solvable repeatedly."""

    def __init__(self, traj, sens, ksp_dims=None, conf: PicsConf | None = None, traj_dims=None, sens_dims=None):
        lib = _lib.load()
        self.conf = conf or PicsConf()
        td = dims16(traj_dims if traj_dims is not None else np.shape(traj))
        sd = dims16(sens_dims if sens_dims is not None else np.shape(sens))
        if ksp_dims is None:
            ksp_dims = [1, td[1], td[2], sd[3]]
        kd = dims16(ksp_dims)
        self.img_dims = sd[:3] + [1] * 13
        self.ksp_dims = kd
        pt, k1 = _ptr_in(traj, int(np.prod(td)))
        ps, k2 = _ptr_in(sens, int(np.prod(sd)))
        h = ctypes.c_void_p()
        cc = self.conf.c()
        _lib.check(lib.bnufft_pics_create(ctypes.byref(h), 16, _lib.dims_array(kd), _lib.dims_array(sd),
                                          _lib.dims_array(td), pt, ps, ctypes.byref(cc), _stream_of(traj, sens)))
        self._h = h

    def run(self, ksp, out=None):
        """One reconstruction of ``ksp`` -> image [X, Y, Z]."""
        n_in = int(np.prod(self.ksp_dims))
        n_out = int(np.prod(self.img_dims))
        if out is None:
            out = _alloc_like(ksp, self.img_dims)
        pk, keep = _ptr_in(ksp, n_in)
        po = _ptr_out(out, n_out)
        _lib.check(_lib.load().bnufft_pics_run(self._h, po, pk, _stream_of(ksp, out)))
        del keep
        return out

    def normal(self, x, out=None):
        """A^H A x."""
        n = int(np.prod(self.img_dims))
        if out is None:
            out = _alloc_like(x, self.img_dims)
        px, keep = _ptr_in(x, n)
        _lib.check(_lib.load().bnufft_pics_normal(self._h, _ptr_out(out, n), px, _stream_of(x, out)))
        del keep
        return out

    def stats(self, stream=None):
        """(iterations, recursive relative residual, scaling) of the last run."""
        it, res, sc = ctypes.c_int(), ctypes.c_double(), ctypes.c_float()
        _lib.check(_lib.load().bnufft_pics_stats(self._h, ctypes.byref(it), ctypes.byref(res),
                                                 ctypes.byref(sc), stream))
        return it.value, res.value, sc.value

    def set_iter(self, maxiter, tol=0.0):
        """Iteration limit and tolerance of later runs."""
        _lib.check(_lib.load().bnufft_pics_set_iter(self._h, int(maxiter), float(tol)))
        self.conf.maxiter, self.conf.tol = int(maxiter), float(tol)

    def rhs(self, ksp, out=None):
        """b = A^H y / scale, the right-hand side of the solve."""
        n_in = int(np.prod(self.ksp_dims))
        n_out = int(np.prod(self.img_dims))
        if out is None:
            out = _alloc_like(ksp, self.img_dims)
        pk, keep = _ptr_in(ksp, n_in)
        _lib.check(_lib.load().bnufft_pics_rhs(self._h, _ptr_out(out, n_out), pk, _stream_of(ksp, out)))
        del keep
        return out

    def precond(self, r, out=None):
        """z = M(r) with the model's preconditioner (precond 1, 2 or 3)."""
        n = int(np.prod(self.img_dims))
        if out is None:
            out = _alloc_like(r, self.img_dims)
        pr, keep = _ptr_in(r, n)
        _lib.check(_lib.load().bnufft_pics_precond(self._h, _ptr_out(out, n), pr, _stream_of(r, out)))
        del keep
        return out

    def set_precnet(self, net):
        """Attach a learned preconditioner (a PrecNet) to a precond=2 model."""
        _lib.check(_lib.load().bnufft_pics_set_precnet(self._h, net.handle, None))
        self._net = net     # keep it alive while attached

    def kernels(self, stream=None):
        """Kernels the last run executed on the device (host launches plus the
        CG loop graph's body once per iteration it ran)."""
        n = ctypes.c_long()
        _lib.check(_lib.load().bnufft_pics_kernels(self._h, ctypes.byref(n), stream))
        return n.value

    def free(self):
        if getattr(self, "_h", None) is not None:
            _lib.load().bnufft_pics_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def pics_l2(traj, ksp, sens, lam=0.0, maxiter=30, toeplitz=True, scaling=0.0, rescale=False, tol=0.0):
    """``bart pics -l2 -r lam -i maxiter -t traj ksp sens out`` on the GPU."""
    p = Pics(traj, sens, ksp_dims=np.shape(ksp) if not hasattr(ksp, "is_cuda") else None,
             conf=PicsConf(lam=lam, maxiter=maxiter, tol=tol, scaling=scaling, rescale=rescale, toeplitz=toeplitz))
    try:
        return p.run(ksp)
    finally:
        p.free()

"""CG-SENSE on one problem with its coils split over ranks (one per GPU).

The SENSE normal operator is a sum over coils, A^H A = sum_c S_c^H F^H F S_c,
so rank r holding coils [c0, c1) (their maps and k-space) computes its share
of A^H A p with the library's own normal operator (a ``Pics`` model built on
those coils) and one all-reduce (sum) of that image-sized vector per
iteration completes it. The CG vectors x, r, p are image-sized and
replicated: after the reduction every rank holds the same A^H A p, so the
dot products need no further exchange. This is the reference's
``--md-split-mpi-dims`` on the coil dim with ``mpi_reduce_zsum`` after each
normal application (src/pics.c:245-251, src/num/mpi_ops.c:680-735), with
the CG of src/iter/italgos.c:497-572.

The right-hand side is reduced the same way (one all-reduce of A_r^H y_r)
before the data scaling is estimated on it, so the scaling is the one the
whole problem would get (src/sense/optcom.c:74-109).
"""

from __future__ import annotations


def coil_range(coils: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous coils [c0, c1) of ``rank``; shares differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("coil_range: need 0 <= rank < world")
    base, extra = divmod(int(coils), int(world))
    c0 = rank * base + min(rank, extra)
    return c0, c0 + base + (1 if rank < extra else 0)


def scaling_from_adjoint(adj) -> float:
    """Data scaling of ``pics`` from the adjoint image A^H y
    (estimate_scaling_norm, src/sense/optcom.c:74-109): the 90th percentile
    of the magnitudes, or their maximum when the tail above it is longer
    than twice the median-to-p90 gap; 1 when it comes out zero."""
    import torch
    mag = torch.sort(adj.reshape(-1).abs().to(torch.float32)).values
    n = mag.numel()
    median, p90, mx = (float(mag[i]) for i in (n // 2, int(n * 0.9), n - 1))
    s = p90 if (mx - p90) < 2 * (p90 - median) else mx
    return s if s != 0.0 else 1.0


def sharded_cg(normal_local, b, lam: float, maxiter: int, tol: float = 0.0, reduce=None, precond=None,
               f32_scalars: bool = False):
    """CG from zero on (sum over ranks of normal_local + lam I) x = b.

    ``normal_local(p)`` returns this rank's share of A^H A p; ``reduce(t)``
    sums a tensor over the ranks in place (None: one rank). ``b`` is the
    already-reduced right-hand side, the same on every rank. One reduction
    per iteration; the dots sum in float64 and are local (the vectors are
    replicated). Stops after ``maxiter`` iterations or when
    ||r|| <= tol ||b|| (tol > 0 reads the residual on the host each
    iteration). Returns (x, iterations run).

    Without ``precond`` this is the reference's CG; ``f32_scalars`` keeps
    alpha, beta and the residual norms in float32 as the reference stores
    them (the library's one-GPU pics default, which reproduces its
    unconverged iterates closely), else they stay in float64. With
    ``precond(r)`` (the same operator on every rank, e.g. the
    padded-circulant one, which depends
    only on the trajectory's PSF and lambda) it is preconditioned CG with
    float64 scalars, the library's precond-3 solve.

    CUDA tensors run the library's fused CG passes with device scalars
    (bnufft_cg_*: two or three launches per iteration besides A p and the
    all-reduce); CPU tensors (the multi-process tests on gloo ranks) run the
    same recurrence in torch operations."""
    import torch
    if b.is_cuda:
        return _sharded_cg_device(normal_local, b, lam, maxiter, tol, reduce, precond, f32_scalars)
    x = torch.zeros_like(b)
    r = b.clone()
    z = precond(r) if precond is not None else r
    p = z.clone()
    f32 = f32_scalars and precond is None

    def dot(u, v):
        return torch.sum((u.conj() * v).real.to(torch.float64))

    def ratio(num, den):
        # where the reference stops (a zero denominator: r reached exactly
        # zero) the ratio is 0, so x and r stay as they are without a host
        # read of the scalars
        q = torch.where(den != 0, num / den, torch.zeros_like(den))
        return q.to(torch.float32) if f32 else q

    rr = dot(r, r)
    rz = rr if precond is None else dot(r, z)
    eps2 = (tol ** 2) * float(rr) if tol > 0 else 0.0
    if float(rr) == 0.0:
        return x, 0
    it = 0
    for it in range(1, maxiter + 1):
        q = normal_local(p)
        if reduce is not None:
            reduce(q)
        q = q + lam * p
        alpha = ratio(rz, dot(p, q))
        x = x + alpha * p
        r = r - alpha * q
        if precond is None:
            rz_new = dot(r, r)
            rr = rz_new
        else:
            if tol > 0:
                rr = dot(r, r)
            z = precond(r)
            rz_new = dot(r, z)
        beta = ratio(rz_new, rz)
        rz = rz_new
        if tol > 0 and float(rr) <= eps2:
            break
        p = beta * p + (r if precond is None else z)
    return x, it


def _sharded_cg_device(normal_local, b, lam, maxiter, tol, reduce, precond, f32_scalars):
    """sharded_cg on the library's fused CG passes (include/bnufft.h,
    bnufft_cg_*)."""
    import ctypes
    import torch
    from . import _lib
    lib = _lib.load()
    st = ctypes.c_void_p(torch.cuda.current_stream(b.device).cuda_stream)
    b = b.contiguous()
    ptr = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None	# noqa: E731
    h = ctypes.c_void_p()
    f32 = bool(f32_scalars) and precond is None
    _lib.check(lib.bnufft_cg_create(ctypes.byref(h), b.numel(), float(lam), float(tol), int(f32), st))
    try:
        x, r, p = torch.empty_like(b), torch.empty_like(b), torch.empty_like(b)
        z = precond(b).contiguous() if precond is not None else None
        _lib.check(lib.bnufft_cg_start(h, ptr(x), ptr(r), ptr(p), ptr(b), ptr(z), st))
        done, iters = ctypes.c_int(0), ctypes.c_int(0)
        _lib.check(lib.bnufft_cg_status(h, ctypes.byref(done), ctypes.byref(iters), None, st))
        if done.value:
            return x, 0
        for _ in range(maxiter):
            q = normal_local(p).contiguous()
            if reduce is not None:
                reduce(q)
            _lib.check(lib.bnufft_cg_update(h, ptr(x), ptr(r), ptr(p), ptr(q), st))
            z = precond(r).contiguous() if precond is not None else None
            _lib.check(lib.bnufft_cg_direction(h, ptr(p), ptr(r), ptr(z), st))
            if tol > 0:		# the stopping test needs the device flag each iteration
                _lib.check(lib.bnufft_cg_status(h, ctypes.byref(done), ctypes.byref(iters), None, st))
                if done.value:
                    break
        _lib.check(lib.bnufft_cg_status(h, ctypes.byref(done), ctypes.byref(iters), None, st))
        return x, int(iters.value)
    finally:
        lib.bnufft_cg_free(h)


def allreduce_sum(t) -> None:
    """In-place sum over the process group of a complex or real tensor."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return
    dist.all_reduce(torch.view_as_real(t) if t.is_complex() else t, op=dist.ReduceOp.SUM)


class CoilShardedPics:
    """``pics -l2 -r lam -i iters -t`` on one problem whose coils are split
    over the ranks of the process group: this rank's ``traj``, its coils'
    ``sens`` (X, Y, Z, C_r) and ``ksp`` (1, R, S, C_r), the k-space as a
    CUDA tensor on this rank's device. ``run`` returns the image (a flat
    complex64 CUDA tensor) on every rank."""

    def __init__(self, traj, sens_local, ksp_dims, lam=0.01, maxiter=30, tol=0.0, scaling=0.0,
                 rescale=False, toeplitz=True, traj_dims=None, sens_dims=None, precond=0, ref_scalars=True):
        from .pics import Pics, PicsConf
        if precond not in (0, 3) or (precond == 3 and not toeplitz):
            raise ValueError("CoilShardedPics: precond 0 (CG) or 3 (padded-circulant PCG, Toeplitz only)")
        self.lam, self.maxiter, self.tol = float(lam), int(maxiter), float(tol)
        self.scaling, self.rescale, self.precond = float(scaling), bool(rescale), int(precond)
        self.ref_scalars = bool(ref_scalars)	# plain CG: float32 scalars as the reference (PicsConf default)
        # scaling 1: rhs() returns this rank's A_r^H y unscaled; the scale is
        # estimated on the reduced sum. The padded-circulant preconditioner
        # depends only on the trajectory and lambda, so every rank's model
        # applies the same one.
        conf = PicsConf(lam=lam, maxiter=maxiter, scaling=1.0, toeplitz=toeplitz, precond=precond)
        self.model = Pics(traj, sens_local, ksp_dims=list(ksp_dims), conf=conf, traj_dims=traj_dims,
                          sens_dims=sens_dims)
        self.iters = 0
        self.scale = None

    def run(self, ksp_local):
        import torch
        b = self.model.rhs(ksp_local)
        if not torch.is_tensor(b):
            raise TypeError("CoilShardedPics.run: give CUDA tensors (k-space on this rank's device)")
        allreduce_sum(b)
        scale = self.scaling if self.scaling != 0.0 else scaling_from_adjoint(b)
        b = b / scale
        x, self.iters = sharded_cg(self.model.normal, b, self.lam, self.maxiter, self.tol, allreduce_sum,
                                   precond=self.model.precond if self.precond else None,
                                   f32_scalars=self.ref_scalars)
        self.scale = scale
        return x * scale if self.rescale else x

    def free(self):
        self.model.free()

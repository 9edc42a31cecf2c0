"""ctypes binding of the C ABI in include/bnufft.h and include/bespirit.h
(``bart_b200/lib/libbnufft.so``).

The library is the product; this module only declares its signatures. There
is no fallback: if the shared library or a CUDA device is missing, loading or
the first call fails loudly.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libbnufft.so")

c_long_p = ctypes.POINTER(ctypes.c_long)


class NufftConfC(ctypes.Structure):
    _fields_ = [("toeplitz", ctypes.c_int), ("periodic", ctypes.c_int), ("deterministic", ctypes.c_int),
                ("os", ctypes.c_float), ("width", ctypes.c_float), ("bin", ctypes.c_int), ("lowmem", ctypes.c_int)]


class PicsConfC(ctypes.Structure):
    _fields_ = [("lambda_", ctypes.c_float), ("maxiter", ctypes.c_int), ("tol", ctypes.c_float),
                ("scaling", ctypes.c_float), ("rescale", ctypes.c_int), ("toeplitz", ctypes.c_int),
                ("periodic", ctypes.c_int), ("deterministic", ctypes.c_int), ("bin", ctypes.c_int),
                ("precond", ctypes.c_int), ("ref_scalars", ctypes.c_int),
                ("net_iters", ctypes.c_int)]


class EcalibConfC(ctypes.Structure):
    _fields_ = [("kdims", ctypes.c_long * 3), ("calsize", ctypes.c_long * 3), ("maps", ctypes.c_int),
                ("threshold", ctypes.c_float), ("numsv", ctypes.c_int), ("percentsv", ctypes.c_float),
                ("crop", ctypes.c_float), ("softcrop", ctypes.c_int), ("rotphase", ctypes.c_int),
                ("orthiter", ctypes.c_int), ("num_orthiter", ctypes.c_int), ("weighting", ctypes.c_int),
                ("intensity", ctypes.c_int), ("phase_normalize", ctypes.c_int), ("nystroem", ctypes.c_int)]


_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libbnufft.so once and declare the prototypes."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"bnufft shared library not found at {path}; run `python -m bart_b200.build`")
    lib = ctypes.CDLL(path)
    vp, i, cl = ctypes.c_void_p, ctypes.c_int, c_long_p

    def sig(name, res, *args):
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = list(args)

    sig("bnufft_conf_defaults", None, ctypes.POINTER(NufftConfC))
    sig("bnufft_create2", i, ctypes.POINTER(vp), i, cl, cl, cl, vp, cl, vp, cl, vp, ctypes.POINTER(NufftConfC), vp)
    sig("bnufft_apply_forward", i, vp, vp, vp, vp)
    sig("bnufft_apply_adjoint", i, vp, vp, vp, vp)
    sig("bnufft_apply_normal", i, vp, vp, vp, vp)
    sig("bnufft_get_psf_dims", i, vp, i, cl)
    sig("bnufft_get_psf", i, vp, i, cl, vp, vp)
    sig("bnufft_update_traj", i, vp, i, cl, vp, vp)
    sig("bnufft_free", None, vp)
    sig("bnufft_nufft_inverse", i, vp, vp, vp, ctypes.c_float, i, i, vp)
    sig("bnufft_forward2d_noalloc", i, ctypes.c_long, ctypes.c_long, ctypes.c_long, vp, vp, vp, vp)
    sig("bnufft_pics_conf_defaults", None, ctypes.POINTER(PicsConfC))
    sig("bnufft_pics_create", i, ctypes.POINTER(vp), i, cl, cl, cl, vp, vp, ctypes.POINTER(PicsConfC), vp)
    sig("bnufft_pics_run", i, vp, vp, vp, vp)
    sig("bnufft_pics_normal", i, vp, vp, vp, vp)
    sig("bnufft_pics_stats", i, vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
        ctypes.POINTER(ctypes.c_float), vp)
    sig("bnufft_pics_kernels", i, vp, ctypes.POINTER(ctypes.c_long), vp)
    sig("bnufft_pics_free", None, vp)
    sig("bnufft_pics_rhs", i, vp, vp, vp, vp)
    sig("bnufft_nudft_create", i, ctypes.POINTER(vp), i, cl, cl, cl, vp, vp)
    sig("bnufft_nudft_apply_forward", i, vp, vp, vp, vp)
    sig("bnufft_nudft_apply_adjoint", i, vp, vp, vp, vp)
    sig("bnufft_nudft_free", None, vp)
    sig("bnufft_batch_create", i, ctypes.POINTER(vp), ctypes.POINTER(vp), i, ctypes.POINTER(vp),
        ctypes.POINTER(vp), vp)
    sig("bnufft_batch_run", i, vp, vp)
    sig("bnufft_batch_kernels", ctypes.c_long, vp)
    sig("bnufft_batch_free", None, vp)
    sig("bnufft_pics_set_iter", i, vp, i, ctypes.c_float)
    sig("bnufft_pics_precond", i, vp, vp, vp, vp)
    sig("bnufft_pics_set_precnet", i, vp, vp, vp)
    fp = ctypes.POINTER(ctypes.c_float)
    sig("bnufft_precnet_nparams", i)
    sig("bnufft_precnet_create", i, ctypes.POINTER(vp), vp, vp)
    sig("bnufft_precnet_set_params", i, vp, vp, vp)
    sig("bnufft_precnet_get_params", i, vp, fp, vp)
    sig("bnufft_precnet_forward", i, vp, vp, vp, ctypes.c_long, ctypes.c_long, ctypes.c_long, vp)
    sig("bnufft_precnet_train_step", i, vp, vp, vp, ctypes.c_long, ctypes.c_long, ctypes.c_long, ctypes.c_float,
        ctypes.POINTER(ctypes.c_double), vp, vp)
    sig("bnufft_precnet_backward", i, vp, vp, vp, ctypes.c_long, ctypes.c_long, ctypes.c_long, ctypes.c_float, vp, vp)
    sig("bnufft_precnet_status", i, vp, ctypes.POINTER(i), vp)
    sig("bnufft_precnet_free", None, vp)
    sig("bnufft_calc_beta", ctypes.c_double, ctypes.c_float, ctypes.c_float)
    sig("bnufft_kb_precompute", i, ctypes.c_double, i, fp)
    sig("bnufft_rolloff_axis", i, ctypes.c_float, ctypes.c_float, ctypes.c_long, ctypes.POINTER(ctypes.c_double))
    sig("bnufft_ecalib_defaults", None, ctypes.POINTER(EcalibConfC))
    sig("bnufft_ecalib_dims", i, ctypes.POINTER(EcalibConfC), i, cl, cl, cl)
    sig("bnufft_ecalib", i, ctypes.POINTER(EcalibConfC), i, cl, vp, vp, vp, fp, cl, cl, vp)
    sig("bnufft_calib", i, ctypes.POINTER(EcalibConfC), i, cl, vp, vp, i, fp, cl, vp, vp)
    sig("bnufft_calone", i, ctypes.POINTER(EcalibConfC), i, cl, vp, vp, fp, cl, cl, vp)
    sig("bnufft_cg_create", i, ctypes.POINTER(vp), ctypes.c_long, ctypes.c_float, ctypes.c_float, i, vp)
    sig("bnufft_cg_start", i, vp, vp, vp, vp, vp, vp, vp)
    sig("bnufft_cg_update", i, vp, vp, vp, vp, vp, vp)
    sig("bnufft_cg_direction", i, vp, vp, vp, vp, vp)
    sig("bnufft_cg_status", i, vp, ctypes.POINTER(i), ctypes.POINTER(i), fp, vp)
    sig("bnufft_cg_free", None, vp)
    sig("bnufft_last_error", ctypes.c_char_p)
    sig("bnufft_launch_count", ctypes.c_long)
    sig("bnufft_prof_start", i, ctypes.c_char_p)
    sig("bnufft_prof_stop", i, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_long))
    _lib = lib
    return lib


class BnufftError(RuntimeError):
    """A bnufft call returned a non-zero status."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"bnufft error {status}: {msg}")
        self.status = status


def check(status: int) -> None:
    if status != 0:
        msg = load().bnufft_last_error().decode(errors="replace")
        raise BnufftError(status, msg)


def dims_array(dims) -> ctypes.Array:
    return (ctypes.c_long * len(dims))(*[int(d) for d in dims])

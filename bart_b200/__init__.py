"""bart_b200: B200-native NUFFT and CG-SENSE behind BART's linop / pics surface.

The compute runs in ``lib/libbnufft.so`` (hand-written sm_100a kernels, C ABI
in include/bnufft.h); this package is the host-side mirror of the
reference's interfaces (nufft_create2 / linop callbacks, pics, .cfl I/O).
"""

from .cfl import readcfl, writecfl  # noqa: F401
from .nufft import Linop, NufftConf, nufft_create, nufft_create2  # noqa: F401
from .pics import Pics, PicsConf, pics_l2  # noqa: F401

__all__ = ["readcfl", "writecfl", "Linop", "NufftConf", "nufft_create", "nufft_create2",
           "Pics", "PicsConf", "pics_l2"]

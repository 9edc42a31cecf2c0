"""The ESPIRiT oracle against the reference's own ecalib outputs (fixtures
from tests/golden/make_golden.py --ecalib)."""

import numpy as np
import pytest

from conftest import golden, rel
from oracle import espirit_oracle as eo

CASES = ["ecalib2d_n64_c8", "ecalib2d_n64_c8_m3_soft", "ecalib2d_n64_c8_k5_r20_n30_P", "ecalib2d_40x48_c20",
         "ecalib3d_n24_c4", "ecalib2d_n64_c8_I", "ecalib2d_50x45_c8_m6"]


def ecalib_kwargs(args):
    """main_ecalib's options (src/ecalib.c:64-97) as oracle keywords."""
    kw, i = {}, 0
    args = [str(a) for a in args]
    while i < len(args):
        a = args[i]
        if a in ("-m", "-c", "-t", "-n", "-k", "-r"):
            v = args[i + 1]
            i += 2
            if a == "-m":
                kw["maps"] = int(v)
            elif a == "-c":
                kw["crop"] = float(v)
            elif a == "-t":
                kw["threshold"] = float(v)
            elif a == "-n":
                kw["numsv"] = int(v)
            else:
                vals = [int(x) for x in v.split(":")] if ":" in v else [int(v)] * 3
                kw["kdims" if a == "-k" else "calsize"] = tuple(vals)
            continue
        if a == "-S":
            kw["softcrop"] = True
        elif a == "-I":
            kw["intensity"] = True
        elif a == "-P":
            kw["rotphase"] = False
        i += 1
    return kw


def map_error(a, b):
    """Relative L2 difference of one map, up to the global sign that the
    reference takes from its LAPACK; 0 when both are all zero (cropped)."""
    if np.linalg.norm(b) == 0:
        return float(np.linalg.norm(a))
    return min(rel(a, b), rel(-a, b))


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_ecalib(name):
    g = golden(name)
    kw = ecalib_kwargs(g["args"])
    sens, ev, val, n, cd = eo.ecalib(g["ksp"], **kw)
    assert n == int(g["nkernels"])
    assert list(cd) == list(g["caldims"])
    # the kept singular values to the reference's float eigen-decomposition;
    # the small tail (printed with "%f", from float eigenvalues near zero)
    # within that decomposition's absolute error
    sv = g["svals"]
    assert rel(val[:n], sv[:n]) < 1e-5
    assert np.max(np.abs(val - sv)) < 1e-3 * sv[0]
    M = sens.shape[-1]
    rs = g["sens"].reshape(sens.shape, order="F")
    re = g["emaps"].reshape(ev.shape, order="F")
    for m in range(M):
        # from the third map on, 30 orthogonal iterations leave the
        # eigenvalues far from converged and the float32 rounding shows
        assert rel(ev[..., m], re[..., m]) < (2e-5 if m < 2 else 1e-3), (m, rel(ev[..., m], re[..., m]))
        # lower maps converge less in 30 orthogonal iterations and follow
        # the float rounding more closely
        assert map_error(sens[..., m], rs[..., m]) < (1e-5 if m == 0 else 1e-4), (m, map_error(sens[..., m], rs[..., m]))


def test_oracle_sinc_matrix_is_the_resize():
    """The per-axis linear map the GPU path uses equals the reference's
    sinc_resize chain applied to the data."""
    rng = np.random.default_rng(3)
    x = rng.standard_normal((12, 5)) + 1j * rng.standard_normal((12, 5))
    for m in (12, 40, 64, 65):
        R = eo.sinc_matrix(12, m)
        assert np.allclose(R @ x, eo.sinc_resize_axis(x, 0, m)) if m != 12 else np.allclose(R, np.eye(12))


def test_oracle_calibration_region_search():
    """A fully sampled 10 x 6 centre inside a 24 x 24 limit: the region stops
    at the first unsampled line in each phase dimension and takes the
    readout window of largest energy."""
    rng = np.random.default_rng(5)
    k = np.zeros((32, 32, 1, 2), dtype=np.complex64)
    k[:, 13:19] = (rng.standard_normal((32, 6, 1, 2)) + 1j * rng.standard_normal((32, 6, 1, 2)))
    k[:, ::5] = 1.0		# lines 10 and 20 sampled, 12 and 19 not
    cal, cd, pos = eo.calib_region(k, (10, 24, 24))
    assert cd == (10, 6, 1)
    assert pos[1] == 13


def test_oracle_calone_matches_reference():
    """ecalib -1: the kernels' low-resolution covariance [12, 12, 1, 36]."""
    g = golden("calone2d_n64_c8")
    k = g["ksp"]
    kd = eo.kernel_dims(k.shape[:3], (6, 6, 6))
    cal, _, _ = eo.calib_region(k, (24, 24, 24))
    kern, _ = eo.compute_kernels(cal, kd)
    cov = eo.compute_imgcov(kern, kd, k.shape[3])
    assert cov.shape == g["cov"].shape[:4]
    assert rel(cov, g["cov"]) < 1e-5

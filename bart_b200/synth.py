"""Seeded synthetic MRI problems in BART's array layout.

Stands in for the measured data and the ``bart traj`` / ``bart phantom`` /
``bart noise`` fixture tools of the reference (src/traj.c, src/phantom.c,
src/noise.c): golden-angle radial and 3D golden-means kooshball trajectories,
ellipse / ellipsoid phantoms, smooth polynomial coil maps normalised to unit
root-sum-of-squares, and complex Gaussian noise at a chosen SNR.

All arrays use BART's column-major layout (numpy index order = BART dim
order): trajectories ``[3, Mr, Ms]``, images ``[X, Y, Z]``, maps
``[X, Y, Z, C]``, k-space ``[1, Mr, Ms, C]``; complex64.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

GOLDEN_RATIO = (1.0 + math.sqrt(5.0)) / 2.0


def radial_traj(readout: int, spokes: int, os: int = 2, golden: bool = True) -> np.ndarray:
    """2D radial trajectory ``[3, readout*os, spokes]`` in cycles per FOV.

    Samples sit at (i + 0.5 - D/2) / os along each spoke (D = readout * os
    samples), as ``bart traj -r -x<readout> -o<os>`` places them, so the
    coordinates span [-readout/2 + 1/(2 os), readout/2 - 1/(2 os)]. Spoke s
    has angle s * pi / phi (golden angle) or s * pi / spokes (uniform).
    """
    D = readout * os
    read = (np.arange(D) + 0.5 - D / 2.0) / os
    s = np.arange(spokes)
    ang = s * (math.pi / GOLDEN_RATIO) if golden else s * (math.pi / spokes)
    t = np.zeros((3, D, spokes), dtype=np.float64)
    t[0] = read[:, None] * np.cos(ang)[None, :]
    t[1] = read[:, None] * np.sin(ang)[None, :]
    return t.astype(np.complex64)


def kooshball_traj(readout: int, spokes: int, os: int = 2) -> np.ndarray:
    """3D radial kooshball ``[3, readout*os, spokes]`` on golden means.

    Spoke directions follow the 2D golden-means scheme (Chan et al., MRM
    2009): with phi1 = 0.4656, phi2 = 0.6823 (the golden means of the
    3x3 Fibonacci recurrence), spoke s has z = 2*frac(s*phi1) - 1 and
    azimuth 2*pi*frac(s*phi2); samples lie at (i + 0.5 - D/2)/os.
    """
    phi1, phi2 = 0.465571231876768, 0.682327803828019
    D = readout * os
    read = (np.arange(D) + 0.5 - D / 2.0) / os
    s = np.arange(spokes)
    z = 2.0 * np.mod(s * phi1, 1.0) - 1.0
    az = 2.0 * math.pi * np.mod(s * phi2, 1.0)
    rxy = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    d = np.stack([rxy * np.cos(az), rxy * np.sin(az), z])
    t = read[None, :, None] * d[:, None, :]
    return t.astype(np.complex64)


def ellipse_phantom(n: int, count: int, rng: np.random.Generator, ndim: int = 2) -> np.ndarray:
    """Sum of ``count`` random ellipses (2D) or ellipsoids (3D) on an n^d grid.

    Centres uniform in the central 60% of the FOV, semi-axes 5-60 pixels
    (scaled to the matrix for n != 256), angles uniform, magnitude U(0.1, 1)
    and a random constant phase per ellipse; rasterised at pixel centres.
    """
    shape = (n,) * ndim + (1,) * (3 - ndim)
    img = np.zeros(shape, dtype=np.complex128)
    coords = np.meshgrid(*[np.arange(n) - n / 2 + 0.5] * ndim, indexing="ij")
    scale = n / 256.0
    for _ in range(count):
        c = rng.uniform(-0.3 * n, 0.3 * n, size=ndim)
        ax = rng.uniform(5.0, 60.0, size=ndim) * scale
        mag = rng.uniform(0.1, 1.0)
        ph = rng.uniform(0.0, 2.0 * math.pi)
        if ndim == 2:
            a = rng.uniform(0.0, math.pi)
            dx, dy = coords[0] - c[0], coords[1] - c[1]
            u = dx * math.cos(a) + dy * math.sin(a)
            v = -dx * math.sin(a) + dy * math.cos(a)
            inside = (u / ax[0]) ** 2 + (v / ax[1]) ** 2 <= 1.0
        else:
            q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
            d = np.stack([coords[i] - c[i] for i in range(3)])
            rot = np.einsum("ij,j...->i...", q.T, d)
            inside = sum((rot[i] / ax[i]) ** 2 for i in range(3)) <= 1.0
        img[inside.reshape(shape)] += mag * np.exp(1j * ph)
    return img.astype(np.complex64)


def coil_maps(n: int, coils: int, rng: np.random.Generator, ndim: int = 2) -> np.ndarray:
    """Smooth maps exp(p_c(r)) with random complex 2nd-order polynomials p_c
    on [-1, 1]^d, normalised so that sum_c |S_c|^2 = 1 at every pixel.
    Returns ``[X, Y, Z, C]``."""
    shape = (n,) * ndim + (1,) * (3 - ndim)
    r = np.meshgrid(*[np.linspace(-1.0, 1.0, n)] * ndim, indexing="ij")
    terms = [np.ones(r[0].shape)] + list(r)
    for i in range(ndim):
        for j in range(i, ndim):
            terms.append(r[i] * r[j])
    out = np.zeros(shape + (coils,), dtype=np.complex128)
    for c in range(coils):
        coef = (rng.standard_normal(len(terms)) + 1j * rng.standard_normal(len(terms))) * 0.5
        p = sum(coef[k] * terms[k] for k in range(len(terms)))
        out[..., c] = np.exp(p).reshape(shape)
    out /= np.sqrt(np.sum(np.abs(out) ** 2, axis=-1, keepdims=True))
    return out.astype(np.complex64)


def add_noise(ksp: np.ndarray, snr_db: float, rng: np.random.Generator) -> np.ndarray:
    """Complex Gaussian noise with power = signal power / 10^(snr/10)."""
    p = float(np.mean(np.abs(ksp) ** 2))
    sigma = math.sqrt(p / (10.0 ** (snr_db / 10.0)) / 2.0)
    noise = rng.standard_normal(ksp.shape) + 1j * rng.standard_normal(ksp.shape)
    return (ksp + sigma * noise).astype(np.complex64)


@dataclass
class SenseProblem:
    traj: np.ndarray      # [3, Mr, Ms] complex64
    sens: np.ndarray      # [X, Y, Z, C] complex64
    truth: np.ndarray     # [X, Y, Z] complex64
    lam: float
    iters: int


def random_image(n: int, rng: np.random.Generator, ndim: int = 2) -> np.ndarray:
    """i.i.d. standard complex Gaussian image (the NUFFT benchmark input)."""
    shape = (n,) * ndim + (1,) * (3 - ndim)
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def cartesian_ksp(img: np.ndarray, sens: np.ndarray, rng: np.random.Generator, snr_db: float = 40.0,
                  calib: int = 24, accel: int = 2) -> np.ndarray:
    """Cartesian multi-coil k-space ``[X, Y, Z, C]`` of ``img * sens``: the
    centred DFT (DC at n/2) of every coil image, complex Gaussian noise, a
    fully sampled centre of ``calib`` lines along every phase-encoding
    dimension (1 and 2) and every ``accel``-th line outside it; the readout
    (dimension 0) is fully sampled. The input of ``bart ecalib``."""
    X, Y, Z, C = sens.shape
    cim = img.reshape(X, Y, Z, 1) * sens
    axes = tuple(a for a, n in enumerate((X, Y, Z)) if n > 1)
    k = np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(cim, axes=axes), axes=axes, norm="ortho"), axes=axes)
    k = add_noise(k, snr_db, rng)
    mask = np.ones((X, Y, Z), dtype=bool)
    for a, n in ((1, Y), (2, Z)):
        if n == 1:
            continue
        idx = np.arange(n)
        keep = (np.abs(idx - n // 2) < calib // 2 + (idx >= n // 2) * (calib % 2)) | (idx % accel == 0)
        shape = [1, 1, 1]
        shape[a] = n
        mask &= keep.reshape(shape)
    return (k * mask[..., None]).astype(np.complex64)

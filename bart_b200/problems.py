"""Seeded synthetic CG-SENSE problems (2D radial), generated on the GPU.

A problem is a golden-angle radial trajectory, smooth polynomial coil maps
normalised to unit root-sum-of-squares, k-space of an ellipse phantom
simulated with the library's own NUFFT, and complex Gaussian noise at a
given SNR: the inputs of ``bart pics -l2 -t traj ksp sens out``.
"""

from __future__ import annotations

import numpy as np

from . import synth


def simulate_ksp(traj, img, sens, snr_db, rng, forward=None):
    """k-space of the SENSE model (NUFFT of img * maps, no Toeplitz) + noise.
    ``forward(traj, cim, kd)``, if given, computes the noiseless k-space
    instead of the library (a host that must not touch the GPU)."""
    N = img.shape[0]
    C = sens.shape[3]
    cim = (img.reshape(N, N, 1, 1) * sens).astype(np.complex64)
    kd = [1, traj.shape[1], traj.shape[2], C]
    if forward is not None:
        y = np.asarray(forward(traj, cim, kd)).reshape(kd, order="F")
        return synth.add_noise(y, snr_db, rng)
    from .nufft import NufftConf, nufft_create2
    op = nufft_create2(kd, list(cim.shape), list(traj.shape), traj, conf=NufftConf(toeplitz=False))
    try:
        y = np.asarray(op.forward(cim)).reshape(kd, order="F")
    finally:
        op.free()
    return synth.add_noise(y, snr_db, rng)


def cgsense_problem(rng, N=256, coils=(8, 32), spokes=(48, 128), ellipses=20, snr_db=40.0, forward=None):
    """One problem with coil count and spoke count drawn uniformly from the
    inclusive ranges (or fixed ints); ``forward`` as in simulate_ksp."""
    C = int(coils) if np.isscalar(coils) else int(rng.integers(coils[0], coils[1] + 1))
    S = int(spokes) if np.isscalar(spokes) else int(rng.integers(spokes[0], spokes[1] + 1))
    traj = synth.radial_traj(N, S)
    truth = synth.ellipse_phantom(N, ellipses, rng)
    sens = synth.coil_maps(N, C, rng)
    ksp = simulate_ksp(traj, truth, sens, snr_db, rng, forward)
    return {"traj": traj, "sens": sens, "ksp": ksp, "truth": truth, "coils": C, "spokes": S}

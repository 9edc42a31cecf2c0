"""CPU oracle for ESPIRiT calibration (``bart ecalib``) of mrirecon/bart v1.0.00.

TEST INFRASTRUCTURE ONLY. This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it. The product (``bart_b200``) never calls it.

It restates the reference's default ecalib path in float64 NumPy:

1. The calibration region: the largest fully sampled centred block up to
   ``calsize``, grown one line at a time in the three spatial dimensions, then
   moved along the readout to the position of largest energy
   (src/misc/mri2.c:100-218).
2. The calibration Gram matrix over all kernel-sized patches of the region
   (src/calib/calmat.c:180-186, src/linops/casorati.c:275-307), its Hermitian
   eigen-decomposition as LAPACK sees it (the conjugate matrix), and the
   kernels whose singular value ratio exceeds sqrt(threshold)
   (src/calib/calib.c:906-1001, 848-887).
3. The kernels zero-padded to twice their size, inverse-FFT'd and reduced to
   a packed C x C Gram matrix per low-resolution pixel
   (src/calib/calib.c:1004-1094).
4. The low-resolution covariance interpolated to the image size by sinc
   (Fourier zero-padding) one axis at a time (src/misc/resize.c:234-292).
5. Per pixel, ``num_orthiter`` steps of orthogonal iteration from the
   identity with a recursive Gram-Schmidt (src/calib/calib.c:73-86,
   src/num/linalg.c:1235-1313), the maps in order of decreasing eigenvalue
   (src/calib/calib.c:418-487).
6. Optionally (-I) each map divided by its l1 norm over the coils times
   sqrt(C) (src/calib/calib.c:754-769, src/misc/utils.c:83-109); crop where
   the eigenvalue is below ``crop`` (hard or soft), and the phase
   of every map aligned to the first principal coil component of the
   calibration data (src/calib/calib.c:136-164, 770-795, src/calib/cc.c:45-75,
   src/misc/utils.c:148-174).

Conventions: arrays are indexed like BART arrays, ``a[x, y, z, c, ...]``
(NumPy index order = BART dimension order). Eigenvectors from LAPACK are
defined up to a phase; the reference's (UPLO 'U') have a real last component
and a sign chosen by the tridiagonal solver. Everything that reaches the
output is invariant to that phase except the principal coil component used
in step 6, whose sign therefore flips the sign of all maps; this module takes
the sign that makes the last component positive.
"""

from __future__ import annotations

import math

import numpy as np

from .nufft_oracle import _fftmod_axis


DEFAULTS = dict(kdims=(6, 6, 6), calsize=(24, 24, 24), maps=2, threshold=0.001, numsv=-1, percentsv=-1.0,
                crop=0.8, softcrop=False, rotphase=True, num_orthiter=30)


def _as4(ksp):
    k = np.asarray(ksp)
    k = k.reshape(k.shape + (1,) * (4 - k.ndim)) if k.ndim < 4 else k
    return k.reshape(k.shape[:4])


# ---------------------------------------------------------------------------
# 1. Calibration region (src/misc/mri2.c:100-218)
# ---------------------------------------------------------------------------

def calib_region(ksp, calsize=(24, 24, 24)):
    """(cal [cx, cy, cz, C], caldims, position in ksp)."""
    k = _as4(ksp).astype(np.complex128)
    dims = k.shape[:3]
    tdims = [dims[0]] + [min(calsize[i], dims[i]) for i in (1, 2)]		# extract_calib2: full readout
    tpos = [(dims[i] - tdims[i]) // 2 for i in range(3)]
    tmp = k[tpos[0]:tpos[0] + tdims[0], tpos[1]:tpos[1] + tdims[1], tpos[2]:tpos[2] + tdims[2]]
    pattern = np.sqrt(np.sum(np.abs(tmp) ** 2, axis=3)) != 0.0			# estimate_pattern
    cal = [1, 1, 1]
    pos = [(tdims[i] - 1) // 2 for i in range(3)]
    stop = [False] * 3
    while not all(stop):							# calib_geom
        for i in range(3):
            if cal[i] == tdims[i] or cal[i] >= calsize[i]:
                stop[i] = True
            if stop[i]:
                continue
            cal[i] += 1
            pos[i] = (tdims[i] - cal[i]) // 2
            blk = pattern[pos[0]:pos[0] + cal[0], pos[1]:pos[1] + cal[1], pos[2]:pos[2] + cal[2]]
            if not blk.all():
                cal[i] -= 1
                pos[i] = (tdims[i] - cal[i]) // 2
                stop[i] = True
    best, beng = 0, 0.0								# calib_readout_pos
    for r in range(tdims[0] - cal[0] + 1):
        blk = tmp[r:r + cal[0], pos[1]:pos[1] + cal[1], pos[2]:pos[2] + cal[2]]
        e = float(np.sqrt(np.sum(np.abs(blk) ** 2)))
        if e > beng:
            best, beng = r, e
    pos[0] = best
    c = tmp[pos[0]:pos[0] + cal[0], pos[1]:pos[1] + cal[1], pos[2]:pos[2] + cal[2]]
    return c, tuple(cal), tuple(tpos[i] + pos[i] for i in range(3))


# ---------------------------------------------------------------------------
# 2. Calibration matrix, Gram matrix, kernels (src/calib/calmat.c, calib.c)
# ---------------------------------------------------------------------------

def calibration_matrix(cal, kdims):
    """Rows = patch positions, columns j = kx_i + kx (ky_i + ky (kz_i + kz c)):
    A[p, j] = cal[p + k_j, c_j] (src/num/casorati.c:34-65)."""
    cx, cy, cz, C = cal.shape
    kx, ky, kz = kdims
    px, py, pz = cx - kx + 1, cy - ky + 1, cz - kz + 1
    cols = []
    for c in range(C):
        for z in range(kz):
            for y in range(ky):
                for x in range(kx):
                    cols.append(cal[x:x + px, y:y + py, z:z + pz, c].reshape(-1, order="F"))
    return np.stack(cols, axis=1)


def kernel_dims(ksp_dims3, kdims):
    return tuple(1 if ksp_dims3[i] == 1 else int(kdims[i]) for i in range(3))


def compute_kernels(cal, kdims, threshold=0.001, numsv=-1, percentsv=-1.0):
    """(kernels [n, N] in descending order, singular values [N]).

    The reference's Gram matrix G = A^H A is handed to LAPACK in row-major
    order, so LAPACK decomposes conj(G); its eigenvectors (the kernels) are
    the conjugates of G's (src/linops/casorati.c:300-306, src/calib/calib.c
    :935-975)."""
    A = calibration_matrix(cal, kdims)
    G = A.conj().T @ A
    w, V = np.linalg.eigh(np.conj(G))
    N = G.shape[0]
    val = np.sqrt(np.maximum(w[::-1], 0.0))
    if numsv != -1:
        n = int(numsv)
    elif percentsv != -1.0:
        n = int(np.float32(N) * np.float32(percentsv) / np.float32(100.0))
    else:
        n = int(np.sum(val / val[0] > math.sqrt(np.float32(threshold))))
    if val[0] <= 0.0:
        raise ValueError("No signal.")
    kern = V[:, ::-1][:, :n].T
    return kern, val


def resize_center(x, out_shape):
    """md_resize_center (src/num/multind.c:1412-1431): centre positions as in
    the FFT (n / 2), zero-padding or truncation at both ends."""
    out = np.zeros(out_shape, dtype=x.dtype)
    so, si = [], []
    for o, i in zip(out_shape, x.shape):
        p = abs(o // 2 - i // 2)
        if o >= i:
            so.append(slice(p, p + i))
            si.append(slice(0, i))
        else:
            so.append(slice(0, o))
            si.append(slice(p, p + o))
    out[tuple(so)] = x[tuple(si)]
    return out


def _mod(x, axis, inverse=False):
    n = x.shape[axis]
    ph = _fftmod_axis(n)
    if inverse:
        ph = np.conj(ph)
    shape = [1] * x.ndim
    shape[axis] = n
    return x * ph.reshape(shape)


def compute_imgcov(kern, kdims, C):
    """Packed lower-triangular C x C Gram matrices of the kernels' images on
    the (2k)^d grid, divided by kx ky kz * xh yh zh: [xh, yh, zh, C(C+1)/2]
    (src/calib/calib.c:1004-1094, src/num/linalg.c:642-664, 1211-1232)."""
    kx, ky, kz = kdims
    n = kern.shape[0]
    hd = tuple(1 if k == 1 else 2 * k for k in kdims)
    K = kern.reshape(n, C, kz, ky, kx).transpose(4, 3, 2, 1, 0)	# [kx, ky, kz, C, n]
    img = resize_center(K, hd + (C, n))
    for a in range(3):
        img = _mod(img, a, inverse=True)
    img = np.fft.ifftn(img, axes=(0, 1, 2)) * float(np.prod(hd))	# unnormalised
    scalesq = float(kx * ky * kz) * float(np.prod(hd))
    out = np.zeros(hd + (C * (C + 1) // 2,), dtype=np.complex128)
    l = 0
    for i in range(C):
        for j in range(i + 1):
            out[..., l] = np.sum(np.conj(img[..., i, :]) * img[..., j, :], axis=-1) / scalesq
            l += 1
    return out


# ---------------------------------------------------------------------------
# 4. sinc interpolation (src/misc/resize.c:234-292)
# ---------------------------------------------------------------------------

def sinc_resize_axis(x, axis, n_out):
    t = _mod(x, axis)
    t = np.fft.fft(t, axis=axis)
    t = _mod(t, axis)
    shape = list(x.shape)
    shape[axis] = n_out
    t = resize_center(t, tuple(shape))
    t = _mod(t, axis, inverse=True)
    t = np.fft.ifft(t, axis=axis) * n_out				# unnormalised inverse
    return _mod(t, axis, inverse=True)


def sinc_zeropad(x, out_shape):
    """Last differing axis first, as the reference recurses."""
    for a in reversed(range(len(out_shape))):
        if out_shape[a] != x.shape[a]:
            assert out_shape[a] > x.shape[a]
            x = sinc_resize_axis(x, a, out_shape[a])
    return x


def sinc_matrix(n_in, n_out):
    """The linear map of sinc_resize_axis along one axis: [n_out, n_in]."""
    if n_in == n_out:
        return np.eye(n_in, dtype=np.complex128)
    return sinc_resize_axis(np.eye(n_in, dtype=np.complex128), 0, n_out)


# ---------------------------------------------------------------------------
# 5. Point-wise orthogonal iteration (src/calib/calib.c:73-86, 418-487)
# ---------------------------------------------------------------------------

def unpack_hermitian(cov, C):
    """[..., C(C+1)/2] packed (i, j <= i) -> [..., C, C], the upper triangle
    the conjugate of the lower (src/calib/calib.c:75-77)."""
    H = np.zeros(cov.shape[:-1] + (C, C), dtype=np.complex128)
    l = 0
    for i in range(C):
        for j in range(i + 1):
            H[..., i, j] = cov[..., l]
            if j != i:
                H[..., j, i] = np.conj(cov[..., l])
            l += 1
    return H


def orthiter(H, M, iters):
    """Rows x (M of them) start as the identity; each step x <- x H and a
    Gram-Schmidt that normalises the last row first (src/num/linalg.c
    :1235-1253, 1296-1313). Returns (rows [..., M, C], norms [..., M])."""
    C = H.shape[-1]
    x = np.zeros(H.shape[:-2] + (M, C), dtype=np.complex128)
    for m in range(M):
        x[..., m, m] = 1.0
    val = np.zeros(H.shape[:-2] + (M,))
    for _ in range(iters):
        x = x @ H
        for m in reversed(range(M)):
            v = x[..., m, :]
            for j in range(m + 1, M):
                s = np.sum(v * np.conj(x[..., j, :]), axis=-1)
                v = v - s[..., None] * x[..., j, :]
            nv = np.sqrt(np.sum(np.abs(v) ** 2, axis=-1))
            val[..., m] = nv
            x[..., m, :] = v / nv[..., None]
    return x, val


def scc_rotation(cal):
    """First principal coil component as the reference's scc leaves it:
    LAPACK's eigenvector of conj(D^H D) (D = calibration data, coils as
    columns) for the largest eigenvalue (src/calib/cc.c:45-62)."""
    C = cal.shape[3]
    D = cal.reshape(-1, C, order="F")
    G = D.conj().T @ D
    w, V = np.linalg.eigh(np.conj(G))
    r = V[:, -1]
    r = r * (np.conj(r[-1]) / abs(r[-1])) if abs(r[-1]) > 0 else r
    return r


def _scurve(t):
    return (t >= 1.0).astype(np.float64) + (t >= -1.0) * (t / (t * t + 1.0) + 0.5)


def ecalib(ksp, kdims=(6, 6, 6), calsize=(24, 24, 24), maps=2, threshold=0.001, numsv=-1, percentsv=-1.0,
           crop=0.8, softcrop=False, rotphase=True, num_orthiter=30, intensity=False):
    """The reference's ``ecalib`` (src/ecalib.c:46-262): (maps [X, Y, Z, C,
    maps] with X etc. 1 where the kernel is 1, eigenvalue maps [X, Y, Z, 1,
    maps], singular values, number of kernels, caldims)."""
    k = _as4(ksp)
    dims = k.shape[:3]
    C = k.shape[3]
    kd = kernel_dims(dims, kdims)
    cal, caldims, _ = calib_region(k, calsize)
    if any(caldims[i] == 1 and dims[i] != 1 for i in range(3)):
        raise ValueError("Calibration region not found!")
    kern, val = compute_kernels(cal, kd, threshold, numsv, percentsv)
    imgcov = compute_imgcov(kern, kd, C)
    od = tuple(dims[i] if kd[i] > 1 else 1 for i in range(3))
    cov = sinc_zeropad(imgcov, od + (imgcov.shape[3],))
    H = unpack_hermitian(cov, C)
    x, v = orthiter(H, maps, num_orthiter)
    sens = np.zeros(od + (C, maps), dtype=np.complex128)
    ev = np.zeros(od + (1, maps), dtype=np.complex128)
    for u in range(maps):
        sens[..., u] = x[..., maps - 1 - u, :]
        ev[..., 0, u] = v[..., maps - 1 - u]
    if intensity:							# normalizel1 * sqrt(C), src/calib/calib.c:754-769
        l1 = np.sum(np.abs(sens), axis=3, keepdims=True)
        sens = np.where(l1 == 0.0, 0.0, sens / np.where(l1 == 0.0, 1.0, l1)) * math.sqrt(C)
    a = np.abs(ev)							# crop_sens
    if softcrop:
        w = _scurve((np.sqrt(a) - crop) / (1.0 - crop))
    else:
        w = (a >= crop).astype(np.float64)
    sens = sens * w
    rot = scc_rotation(cal) if rotphase else np.eye(C)[0]
    s = np.sum(sens * np.conj(rot).reshape(1, 1, 1, C, 1), axis=3, keepdims=True)	# fixphase2
    ph = np.where(np.abs(s) == 0.0, 1.0, s / np.where(np.abs(s) == 0.0, 1.0, np.abs(s)))
    sens = sens * np.conj(ph)
    return sens, ev, val, kern.shape[0], caldims

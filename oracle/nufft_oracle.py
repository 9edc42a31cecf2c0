"""CPU oracle for the NUFFT / Toeplitz / CG-SENSE path of mrirecon/bart v1.0.00.

TEST INFRASTRUCTURE ONLY. This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it. The product (``bart_b200``) never calls it.

It restates the reference algorithm in NumPy:

* The Kaiser-Bessel table, its lookup and the tap windows are evaluated with
  exactly the reference's single-precision arithmetic, so every interpolation
  weight is bit-identical to the reference's
  (src/noncart/grid.c:38-149, 403-512).
* The oversampled spectrum is computed in float64 with a 2N-point centred FFT.
  The reference obtains the same values as 2^d N-point FFTs of linearly phased
  copies (src/noncart/nufft.c:196-248, 1388-1458); both equal the continuous
  Fourier transform of the apodised image at half-integer frequencies.
* All accumulation runs in float64, so the oracle is the reference's
  discretisation without its float32 rounding.

Conventions (the reference's, src/misc/mri.h): arrays are column-major BART
arrays; images are ``[X, Y, Z, C]``, k-space ``[1, Mr, Ms, C]`` flattened here
to ``[M, C]`` with the sample index fastest, trajectories ``[3, M]`` real.
In this module arrays are NumPy arrays indexed ``a[x, y, z, c]`` (numpy
order = BART order, with ``order='F'`` used at the file boundary).
"""

from __future__ import annotations

import math

import numpy as np

KB_SIZE = 1000           # kb_size_max, src/noncart/grid.c:38
F32 = np.float32


# ---------------------------------------------------------------------------
# Kaiser-Bessel window (src/noncart/grid.c:38-149, src/num/specfun.c:120-129)
# ---------------------------------------------------------------------------

def bessel_i0(x: float) -> float:
    """Modified Bessel function I0 in float64 from its power series.

    The reference evaluates I0 with a published minimax approximation
    (src/num/specfun.c:120-129); both are accurate to float64 rounding for the
    arguments used here (|x| <= 14), which is far below the float32 table.
    """
    x = abs(float(x))
    q = 0.25 * x * x
    term = 1.0
    total = 1.0
    k = 1
    while True:
        term *= q / (k * k)
        total += term
        if term < 1e-18 * total:
            break
        k += 1
    return total


def calc_beta(os: float = 2.0, width: float = 6.0) -> float:
    """beta = pi * sqrt(((w/os)*(os-0.5))^2 - 0.8) (src/noncart/grid.c:516-519).

    ``width / os`` is a float32 division in the reference (both are float).
    """
    wos = float(F32(width) / F32(os))
    return math.pi * math.sqrt((wos * (float(F32(os)) - 0.5)) ** 2 - 0.8)


def kernel_beta(os: float = 2.0, width: float = 6.0) -> float:
    """The beta the reference's KB table is built with.

    The first caller of kb_init is rolloff_correction(), whose beta parameter
    is a float (src/noncart/grid.c:559, called from src/noncart/nufft.c:903),
    so the table and I0(beta) use beta rounded to float32.
    """
    return float(F32(calc_beta(os, width)))


def kb_table(beta: float, n: int = KB_SIZE) -> np.ndarray:
    """kb_precompute: table[i] = I0(beta*sqrt(1-(2x)^2))/I0(beta), x=i/(n-1)/2.

    src/noncart/grid.c:73-97. Values rounded to float32.
    """
    i0b = bessel_i0(beta)
    out = np.zeros(n + 1, dtype=F32)
    for i in range(n + 1):
        x = float(i) / float(n - 1) / 2.0
        if abs(x) >= 0.5:
            out[i] = 0.0
        else:
            out[i] = F32(bessel_i0(beta * math.sqrt(1.0 - (2.0 * x) ** 2)) / i0b)
    return out


def intlookup(table: np.ndarray, x: np.ndarray) -> np.ndarray:
    """Table lookup with linear interpolation (src/noncart/grid.c:120-149).

    ``x`` is float32; ``x *= 2`` and the index product are float32; the lerp
    ``(1. - c) * a + c * b`` runs in float64 and is rounded to float32.
    """
    n = table.shape[0] - 1
    x = (x.astype(F32) * F32(2.0)).astype(F32)
    xs = (x * F32(n - 1)).astype(F32)
    idx = xs.astype(np.int64)                      # C truncation, x >= 0
    fpart = (xs - idx.astype(F32)).astype(F32)
    a = table[idx].astype(np.float64)
    b = table[idx + 1].astype(np.float64)
    c = fpart.astype(np.float64)
    return ((1.0 - c) * a + c * b).astype(F32)


def ftkb(beta: float, x, i0b: float):
    """Fourier transform of the KB window (src/noncart/grid.c:100-112)."""
    x = np.asarray(x, dtype=np.float64)
    a = beta * beta - (math.pi * x) ** 2
    out = np.empty_like(a)
    pos = a > 0
    neg = a < 0
    zer = a == 0
    sa = np.sqrt(np.abs(a))
    out[pos] = np.sinh(sa[pos]) / sa[pos] / i0b
    out[neg] = np.sin(sa[neg]) / sa[neg] / i0b
    out[zer] = 1.0 / i0b
    return out


def rolloff_axis(n: int, os: float, width: float, beta: float) -> np.ndarray:
    """Per-axis apodisation 1/(width*ftkb(beta, pos*width)) in float64.

    pos(d, i, os) (src/noncart/grid.c:522-533): oi = i + (os*d/2 - d/2),
    pos = (oi - os*d/2) / (os*d); singleton axes give 1.
    """
    if n == 1:
        return np.ones(1)
    od = int(F32(os) * n)
    i = np.arange(n)
    oi = i + (od // 2 - n // 2)
    p = (oi.astype(np.float64) - float(od // 2)) / float(od)
    p = p.astype(F32).astype(np.float64)           # pos() returns float
    i0b = bessel_i0(beta)
    return 1.0 / ftkb(beta, p * float(F32(width)), i0b) / float(F32(width))


def rolloff_table(dims3, os: float = 2.0, width: float = 6.0) -> np.ndarray:
    """Separable roll-off table [X, Y, Z], float32 like the reference's
    precomputed ``roll`` (src/noncart/grid.c:537-556, nufft.c:898-906)."""
    beta = kernel_beta(os, width)
    rx, ry, rz = (rolloff_axis(int(d), os, width, beta) for d in dims3)
    tab = rx[:, None, None] * ry[None, :, None] * rz[None, None, :]
    return tab.astype(F32)


# ---------------------------------------------------------------------------
# Interpolation weights: the decomposed gridding of the reference
# ---------------------------------------------------------------------------

def _subgrid_shifts(dims3):
    """Sub-grid shifts -s/2 in the reference's order (compute_shift,
    src/noncart/nufft.c:133-147): bit i of the index selects axis i."""
    fac = [2 if d > 1 else 1 for d in dims3]
    out = []
    for idx in range(fac[0] * fac[1] * fac[2]):
        s = []
        r = idx
        for i in range(3):
            s.append(r % fac[i])
            r //= fac[i]
        out.append(tuple(s))
    return out


def interp_taps(traj: np.ndarray, dims3, periodic: bool = False,
                width: float = 6.0, os: float = 2.0):
    """All (sample, oversampled-grid cell, weight) taps of the gridding.

    Restates grid2_decomp/grid2H_decomp (src/noncart/nufft.c:158-188) over
    the 2^d sub-grids, gridH/grid (src/noncart/grid.c:153-253) and
    grid_point_gen (src/noncart/grid.c:403-465):

    * sub-grid s has width w/2 on the N-grid, os = 1, shift -s/2;
    * pos = float(1 * (k + shift)) + float(N/2) (float32);
    * taps from ceil(pos - w/4) to floor(pos + w/4) (float64 bounds);
    * weight = ((1 * wz) * wy) * wx, each w* = intlookup(|tap - pos| / (w/2)).

    Returns (sample index, flat cell index of the 2N grid in x-fastest order,
    float32 weight). The 2N-grid cell of sub-grid s tap t is 2 t + s per axis.
    """
    beta = kernel_beta(os, width)
    table = kb_table(beta)
    traj = np.asarray(traj, dtype=F32).reshape(3, -1)
    M = traj.shape[1]
    dims3 = [int(d) for d in dims3]
    g2 = [2 * d if d > 1 else 1 for d in dims3]
    hw = F32(F32(width) / F32(2.0))                 # conf.width /= 2 (float)

    samples, cells, weights = [], [], []
    for s in _subgrid_shifts(dims3):
        per_axis = []
        for ax in range(3):
            n = dims3[ax]
            shift = F32(-float(s[ax]) / 2.0)
            if n > 1:
                # odd-size correction (src/noncart/nufft.c:164-166) is 0 here
                shift = F32(shift + F32((n / 2.0 - n // 2) / 1.0))
            pos = (F32(1.0) * (traj[ax] + shift)).astype(F32)
            if n > 1:
                pos = (pos + F32(n // 2)).astype(F32)
            if n == 1:
                taps = [np.zeros(M, dtype=np.int64)]
                wts = [np.full(M, intlookup(table, np.zeros(1, dtype=F32))[0], dtype=F32)]
                valid = [np.ones(M, dtype=bool)]
                idxs = [np.zeros(M, dtype=np.int64)]
            else:
                sti = np.ceil(pos.astype(np.float64) - 0.5 * float(hw)).astype(np.int64)
                eni = np.floor(pos.astype(np.float64) + 0.5 * float(hw)).astype(np.int64)
                taps, wts, valid, idxs = [], [], [], []
                span = int((eni - sti).max()) + 1 if M else 0
                for o in range(span):
                    t = sti + o
                    ok = t <= eni
                    if not periodic:
                        ok &= (t >= 0) & (t <= n - 1)
                        ti = t
                    else:
                        ti = np.mod(t, n)
                    frac = np.abs(t.astype(F32) - pos).astype(F32)
                    frac = np.where(t <= eni, frac, F32(0.0)).astype(F32)   # masked taps
                    wv = intlookup(table, (frac / hw).astype(F32))
                    taps.append(t)
                    wts.append(wv)
                    valid.append(ok)
                    idxs.append(2 * ti + s[ax])
            per_axis.append((idxs, wts, valid))

        (ix, wx, vx), (iy, wy, vy), (iz, wz, vz) = per_axis
        for a in range(len(iz)):
            for b in range(len(iy)):
                d_zy = (F32(1.0) * wz[a]).astype(F32)
                d_zy = (d_zy * wy[b]).astype(F32)
                for c in range(len(ix)):
                    ok = vz[a] & vy[b] & vx[c]
                    d = (d_zy * wx[c]).astype(F32)
                    cell = ix[c] + g2[0] * (iy[b] + g2[1] * iz[a])
                    sel = np.nonzero(ok)[0]
                    samples.append(sel)
                    cells.append(cell[sel])
                    weights.append(d[sel])
    return (np.concatenate(samples), np.concatenate(cells),
            np.concatenate(weights).astype(np.float64))


# ---------------------------------------------------------------------------
# Oversampled spectrum (centred 2N FFT) and its adjoint
# ---------------------------------------------------------------------------

def _axes(dims3):
    return tuple(i for i in range(3) if dims3[i] > 1)


def spectrum(x: np.ndarray) -> np.ndarray:
    """E x: centred 2N-point spectrum of an [X,Y,Z,...] array, 1/sqrt(N) scaled.

    E x [j] = N^-1/2 sum_n x_n exp(-2 pi i (j - N)(n - N/2) / (2N)) per axis,
    i.e. the image's Fourier transform at frequency (j - N)/2 (cycles/FOV).
    This is what the reference's linphase/FFT/fftmod chain produces on its
    2^d sub-grids (src/noncart/nufft.c:1410-1423) with sub-grid s, index w
    holding cell j = 2w + s.
    """
    dims3 = x.shape[:3]
    axes = _axes(dims3)
    pad = [(0, 0)] * x.ndim
    for a in axes:
        n = dims3[a]
        pad[a] = (n // 2, n - n // 2)
    xp = np.pad(x.astype(np.complex128), pad)
    scale = 1.0 / math.sqrt(float(np.prod([dims3[a] for a in axes])))
    return np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(xp, axes=axes), axes=axes), axes=axes) * scale


def spectrum_adjoint(g: np.ndarray, dims3) -> np.ndarray:
    """E^H: adjoint of :func:`spectrum` (crop of the centred inverse DFT)."""
    axes = _axes(dims3)
    tot = float(np.prod([g.shape[a] for a in axes]))
    scale = 1.0 / math.sqrt(float(np.prod([dims3[a] for a in axes])))
    full = np.fft.fftshift(np.fft.ifftn(np.fft.ifftshift(g, axes=axes), axes=axes), axes=axes) * tot
    sl = [slice(None)] * g.ndim
    for a in axes:
        n = dims3[a]
        sl[a] = slice(n // 2, n // 2 + n)
    return full[tuple(sl)] * scale


# ---------------------------------------------------------------------------
# NUFFT operators (src/noncart/nufft.c:1388-1540)
# ---------------------------------------------------------------------------

class NufftOracle:
    """Forward / adjoint / Toeplitz-normal NUFFT of the reference, in float64.

    ``dims`` is the coil-image size (X, Y, Z); ``traj`` is [3, M] in cycles per
    FOV (the real parts of the reference's trajectory array).
    """

    def __init__(self, traj, dims, periodic=False, width=6.0, os=2.0, weights=None):
        self.weights = None if weights is None else np.asarray(weights).reshape(-1, order="F").astype(np.complex64)
        self.dims3 = tuple(int(d) for d in dims)
        self.traj = np.asarray(traj, dtype=F32).reshape(3, -1)
        self.M = self.traj.shape[1]
        self.periodic = periodic
        self.g2 = tuple(2 * d if d > 1 else 1 for d in self.dims3)
        self.roll = rolloff_table(self.dims3, os, width).astype(np.float64)
        self.samp, self.cell, self.wgt = interp_taps(self.traj, self.dims3, periodic, width, os)
        self._psf = None

    # gridding on the 2N grid (x-fastest flat cells)
    def degrid(self, g):
        """Interpolate k-space samples from an oversampled grid [2X,2Y,2Z,C]."""
        C = g.shape[3]
        gf = g.reshape(-1, C, order="F")
        out = np.zeros((self.M, C), dtype=np.complex128)
        for c in range(C):
            contrib = gf[self.cell, c] * self.wgt
            out[:, c] = (np.bincount(self.samp, weights=contrib.real, minlength=self.M)
                         + 1j * np.bincount(self.samp, weights=contrib.imag, minlength=self.M))
        return out

    def grid(self, y):
        """Spread k-space samples [M, C] onto the oversampled grid."""
        C = y.shape[1]
        ncell = int(np.prod(self.g2))
        out = np.zeros((ncell, C), dtype=np.complex128)
        for c in range(C):
            contrib = y[self.samp, c] * self.wgt
            out[:, c] = (np.bincount(self.cell, weights=contrib.real, minlength=ncell)
                         + 1j * np.bincount(self.cell, weights=contrib.imag, minlength=ncell))
        return out.reshape(self.g2 + (C,), order="F")

    def forward(self, img):
        """img [X,Y,Z,C] -> ksp [M,C] (nufft_apply_forward, :1388-1458)."""
        img = _as4(img)
        x = img * self.roll[..., None]
        y = self.degrid(spectrum(x))
        if self.weights is not None:     # md_zmul2 by the weights (:1456)
            y = y * self.weights.astype(np.complex128)[:, None]
        return y

    def adjoint(self, ksp):
        """ksp [M,C] -> img [X,Y,Z,C] (nufft_apply_adjoint, :1462-1540)."""
        ksp = np.asarray(ksp).reshape(self.M, -1).astype(np.complex128)
        if self.weights is not None:     # md_zmulc2 by the weights (:1474)
            ksp = ksp * np.conj(self.weights.astype(np.complex128))[:, None]
        g = self.grid(ksp)
        x = spectrum_adjoint(g, self.dims3)
        return x * self.roll[..., None]

    def psf(self):
        """Toeplitz kernel on the centred 2N spectrum grid.

        compute_psf2 (src/noncart/nufft.c:727-776): adjoint NUFFT of ones with
        trajectory 2*traj onto a 2N image with periodic gridding (the caller
        passes periodic=true, :1146), then the centred unitary FFT (fftuc).
        The reference then splits it into the 2^d sub-grids (md_decompose);
        here it stays on the 2N grid, cell j = 2w + s.
        """
        if self._psf is None:
            dims2 = self.g2
            inner = NufftOracle((self.traj.astype(F32) * F32(2.0)), dims2, periodic=True)
            ones = np.ones((self.M, 1), dtype=np.complex128)
            if self.weights is not None:  # squared weights (compute_square_weights, :509-518)
                w = self.weights
                ones = (w * np.conj(w)).astype(np.complex64).astype(np.complex128)[:, None]
            psft = inner.adjoint(ones)[..., 0]
            axes = _axes(dims2)
            tot = float(np.prod([dims2[a] for a in axes]))
            self._psf = np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(psft, axes=axes), axes=axes),
                                        axes=axes) / math.sqrt(tot)
        return self._psf

    def normal_toeplitz(self, img):
        """E^H (P . E x) (toeplitz_mult, src/noncart/nufft.c:1546-1625)."""
        img = _as4(img)
        P = self.psf()
        return spectrum_adjoint(spectrum(img) * P[..., None], self.dims3)

    def normal_explicit(self, img):
        """adjoint(forward(img)), the normal without Toeplitz embedding."""
        return self.adjoint(self.forward(img))


def _fftmod_axis(n):
    """fftmod phases of one axis (src/num/fft.c:62-67 with phase 0)."""
    c = n // 2
    j = np.arange(n)
    return np.exp(2j * np.pi * (j - c / 2.0) * (c / n)) if n > 1 else np.ones(1)


def _fftuc(x, axes):
    tot = float(np.prod([x.shape[a] for a in axes]))
    return np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(x, axes=axes), axes=axes), axes=axes) / math.sqrt(tot)


def _ifftuc(x, axes):
    tot = float(np.prod([x.shape[a] for a in axes]))
    return np.fft.fftshift(np.fft.ifftn(np.fft.ifftshift(x, axes=axes), axes=axes), axes=axes) * math.sqrt(tot)


def circulant_precond(op: "NufftOracle") -> np.ndarray:
    """Strang circulant preconditioner of the Toeplitz normal operator,
    restating compute_precond (src/noncart/precond.c:36-64) literally on the
    reference's decomposed PSF: pre = sum_s conj(linphase_s) ifftuc(psf_s),
    then |fftuc(pre)| + 1e-3, kept in the array order fftuc returns (it is
    applied element-wise after an uncentred FFT, precond.c:82-91)."""
    dims3 = op.dims3
    axes = _axes(dims3)
    Pc = op.psf()
    fm = np.ones(dims3, dtype=np.complex128)
    for a in axes:
        sh = [1, 1, 1]
        sh[a] = dims3[a]
        fm = fm * _fftmod_axis(dims3[a]).reshape(sh)
    E1 = spectrum(np.ones(dims3 + (1,)))[..., 0]
    pre = np.zeros(dims3, dtype=np.complex128)
    for s in _subgrid_shifts(dims3):
        sl = tuple(slice(s[a], None, 2) if dims3[a] > 1 else slice(None) for a in range(3))
        Ls = np.fft.ifftn(np.conj(fm) * E1[sl], axes=axes)     # linphase_s as a multiplier
        pre += np.conj(Ls) * _ifftuc(Pc[sl], axes)
    return np.abs(_fftuc(pre, axes)) + 1e-3


def padded_precond(op: "NufftOracle", lam: float, beta: float = 2.5):
    """The library's padded-circulant preconditioner (precond 3; no
    counterpart in the reference): the Toeplitz product's own circulant
    inverted on the zero-padded image, M^-1 v = S^H (|P| + mu)^-1 S v with
    S = spectrum (S^H S = 2^d here), mu = beta lam 2^d, floored at
    1e-3 |P| at DC. The device kernel uses the same operator with its
    unnormalised FFTs and P / npix: its z is npix^2 times this one."""
    dims3 = op.dims3
    d = len(_axes(dims3))
    P = np.abs(op.psf())
    dc = P[tuple(n // 2 for n in P.shape)]
    mu = max(beta * lam * 2.0 ** d, 1e-3 * float(dc))
    Pm = (P + mu)[..., None]

    def apply(v):
        return spectrum_adjoint(spectrum(_as4(v)) / Pm, dims3)

    return apply


def pcg(normal, b, lam, M, tol=1e-4, maxiter=300):
    """Preconditioned CG on (normal + lam I) x = b with the preconditioner
    M (float64); stops when ||r|| <= tol ||b||. Returns (x, iterations)."""
    x = np.zeros_like(b)
    r = b.copy()
    z = M(r)
    p = z.copy()
    rz = float(np.vdot(r, z).real)
    nb = math.sqrt(float(np.vdot(b, b).real))
    for it in range(1, maxiter + 1):
        Ap = normal(p) + lam * p
        a = rz / float(np.vdot(p, Ap).real)
        x = x + a * p
        r = r - a * Ap
        if math.sqrt(float(np.vdot(r, r).real)) <= tol * nb:
            return x, it
        z = M(r)
        rz2 = float(np.vdot(r, z).real)
        p = z + (rz2 / rz) * p
        rz = rz2
    return x, maxiter


def nufft_inverse(op: "NufftOracle", ksp, lam=0.0, maxiter=50, precond=False):
    """``bart nufft -i [-c] -l lam -m maxiter`` (src/nufft.c:250-263): CG
    (l2lambda 0) on P^-1 (N^H N + lam) x = P^-1 N^H y over all coil images
    jointly (lsqr2_create, src/iter/lsqr.c:78-167); P^-1 v = ifft(fft(v)/pre)
    with the uncentred, unnormalised FFT (precond.c:82-91)."""
    dims3 = op.dims3
    axes = _axes(dims3)
    y = np.asarray(ksp).reshape(op.M, -1)
    pre = circulant_precond(op)[..., None] if precond else None

    def pinv(v):
        if pre is None:
            return v
        tot = float(np.prod([dims3[a] for a in axes]))
        return np.fft.ifftn(np.fft.fftn(v, axes=axes) / pre, axes=axes) * tot

    def normal(v):
        return pinv(op.normal_toeplitz(v) + lam * v)

    b = pinv(op.adjoint(y))
    x, _ = conjgrad(normal, b, 0.0, maxiter)
    return x


def _as4(a):
    a = np.asarray(a)
    while a.ndim < 4:
        a = a[..., None]
    return a.astype(np.complex128)


# ---------------------------------------------------------------------------
# Chained NUFFT for os != 2 (nufft_create2 -> nufft_create_chain,
# src/noncart/nufft.c:1185-1198, src/noncart/nufft_chain.c:190-244)
# ---------------------------------------------------------------------------

class ChainNufftOracle:
    """roll-off (os) -> centred in the G = lround(os N) grid -> unitary
    centred FFT -> KB gridding on that grid (width w, beta(os, w)) -> times
    os^(d/2) (and the weights); the adjoint in reverse. float64 except the
    taps, which follow gridH / grid_point_gen in float32 (src/noncart/grid.c:
    150-199, 403-465): pos = float(os k) + float(G/2), taps ceil(pos - w/2) ..
    floor(pos + w/2) in float64, weight ((1 wz) wy) wx with
    w* = intlookup(|t - pos| / w)."""

    def __init__(self, traj, dims, os, width=6.0, periodic=False, weights=None):
        self.dims3 = tuple(int(d) for d in dims)
        self.os, self.width = float(os), float(width)
        # lround: halves away from zero (Python's round() would round them to even)
        self.G = tuple(int(math.floor(float(os) * d + 0.5)) if d > 1 else 1 for d in self.dims3)
        self.nd = sum(1 for d in self.dims3 if d > 1)
        beta = kernel_beta(os, width)
        self.roll = rolloff_table(self.dims3, os, width).astype(np.float64)
        self.scale = self.os ** (0.5 * self.nd) / math.sqrt(float(np.prod(self.G)))
        self.weights = None if weights is None else np.asarray(weights).reshape(-1, order="F").astype(np.complex128)
        table = kb_table(beta)
        traj = np.asarray(traj, dtype=F32).reshape(3, -1)
        self.M = M = traj.shape[1]
        w = F32(width)
        per_axis = []
        for ax in range(3):
            G = self.G[ax]
            if G == 1:
                per_axis.append(([np.zeros(M, dtype=np.int64)],
                                 [np.full(M, intlookup(table, np.zeros(1, dtype=F32))[0], dtype=F32)],
                                 [np.ones(M, dtype=bool)]))
                continue
            pos = (F32(os) * traj[ax]).astype(F32)
            pos = (pos + F32(G // 2)).astype(F32)
            sti = np.ceil(pos.astype(np.float64) - 0.5 * float(w)).astype(np.int64)
            eni = np.floor(pos.astype(np.float64) + 0.5 * float(w)).astype(np.int64)
            idxs, wts, valid = [], [], []
            for o in range(int((eni - sti).max()) + 1 if M else 0):
                t = sti + o
                ok = t <= eni
                if periodic:
                    ti = np.mod(t, G)
                else:
                    ok &= (t >= 0) & (t <= G - 1)
                    ti = t
                frac = np.where(ok, np.abs(t.astype(F32) - pos), F32(0.0)).astype(F32)
                wts.append(intlookup(table, (frac / w).astype(F32)))
                idxs.append(np.clip(ti, 0, G - 1))
                valid.append(ok)
            per_axis.append((idxs, wts, valid))
        (ix, wx, vx), (iy, wy, vy), (iz, wz, vz) = per_axis
        samp, cell, wgt = [], [], []
        for a in range(len(iz)):
            for b in range(len(iy)):
                dzy = ((F32(1.0) * wz[a]).astype(F32) * wy[b]).astype(F32)
                for c in range(len(ix)):
                    ok = vz[a] & vy[b] & vx[c]
                    d = (dzy * wx[c]).astype(F32)
                    sel = np.nonzero(ok)[0]
                    samp.append(sel)
                    cell.append((ix[c] + self.G[0] * (iy[b] + self.G[1] * iz[a]))[sel])
                    wgt.append(d[sel])
        self.samp, self.cell = np.concatenate(samp), np.concatenate(cell)
        self.wgt = np.concatenate(wgt).astype(np.float64)

    def _axes(self):
        return tuple(i for i in range(3) if self.G[i] > 1)

    def forward(self, img):
        img = _as4(img)
        C = img.shape[3]
        x = img * self.roll[..., None]
        xg = np.zeros(self.G + (C,), dtype=np.complex128)
        sl = tuple(slice(g // 2 - n // 2, g // 2 - n // 2 + n) for g, n in zip(self.G, self.dims3))
        xg[sl] = x
        ax = self._axes()
        spec = np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(xg, axes=ax), axes=ax), axes=ax) * self.scale
        gf = spec.reshape(-1, C, order="F")
        out = np.zeros((self.M, C), dtype=np.complex128)
        for c in range(C):
            v = gf[self.cell, c] * self.wgt
            out[:, c] = (np.bincount(self.samp, weights=v.real, minlength=self.M)
                         + 1j * np.bincount(self.samp, weights=v.imag, minlength=self.M))
        if self.weights is not None:
            out = out * self.weights[:, None]
        return out

    def adjoint(self, ksp):
        ksp = np.asarray(ksp).reshape(self.M, -1).astype(np.complex128)
        if self.weights is not None:
            ksp = ksp * np.conj(self.weights)[:, None]
        C = ksp.shape[1]
        n = int(np.prod(self.G))
        g = np.zeros((n, C), dtype=np.complex128)
        for c in range(C):
            v = ksp[self.samp, c] * self.wgt
            g[:, c] = (np.bincount(self.cell, weights=v.real, minlength=n)
                       + 1j * np.bincount(self.cell, weights=v.imag, minlength=n))
        g = g.reshape(self.G + (C,), order="F")
        ax = self._axes()
        xg = np.fft.fftshift(np.fft.ifftn(np.fft.ifftshift(g, axes=ax), axes=ax), axes=ax) * (self.scale * n)
        sl = tuple(slice(gg // 2 - nn // 2, gg // 2 - nn // 2 + nn) for gg, nn in zip(self.G, self.dims3))
        return xg[sl] * self.roll[..., None]


# ---------------------------------------------------------------------------
# Subspace basis (nufft_create2 with a basis, src/noncart/nufft.c:1018-1042,
# 1427-1491, 1546-1625, 470-505)
# ---------------------------------------------------------------------------

class BasisNufftOracle:
    """NUFFT with a temporal basis B [T, K]: frame t has its own trajectory
    (or the shared one) and optional sampling weights w_t;
    y_t = w_t * sum_k B[t, k] NUFFT_t(x_k), adjoint x_k = sum_t conj(B[t, k])
    NUFFT_t^H(conj(w_t) y_t). Images [X, Y, Z, C, K] (coils C), k-space
    [M, C, T] (M samples of one frame)."""

    def __init__(self, trajs, dims, basis, weights=None):
        self.B = np.asarray(basis, dtype=np.complex128).reshape(-1, np.shape(basis)[-1], order="F")  # [T, K]
        self.T, self.K = self.B.shape
        self.ops = [NufftOracle(trajs[t if len(trajs) > 1 else 0], dims) for t in range(self.T)]
        self.w = None if weights is None else [np.asarray(weights[t]).reshape(-1).astype(np.complex128)
                                               for t in range(self.T)]

    def forward(self, x):
        x = np.asarray(x, dtype=np.complex128)      # [X, Y, Z, C, K]
        out = []
        for t, op in enumerate(self.ops):
            y = sum(self.B[t, k] * op.forward(x[..., k]) for k in range(self.K))
            out.append(y if self.w is None else y * self.w[t][:, None])
        return np.stack(out, axis=-1)               # [M, C, T]

    def adjoint(self, y):
        y = np.asarray(y, dtype=np.complex128)      # [M, C, T]
        acc = None
        for t, op in enumerate(self.ops):
            yt = y[..., t] if self.w is None else y[..., t] * np.conj(self.w[t])[:, None]
            a = op.adjoint(yt)                      # [X, Y, Z, C]
            v = np.stack([np.conj(self.B[t, k]) * a for k in range(self.K)], axis=-1)
            acc = v if acc is None else acc + v
        return acc

    def normal_toeplitz(self, x):
        """sum_t conj(B[t, k]) B[t, k'] applied to each frame's Toeplitz
        normal (with |w_t|^2 weights): the block-Toeplitz product."""
        x = np.asarray(x, dtype=np.complex128)
        out = np.zeros_like(x)
        for t, op in enumerate(self.ops):
            if self.w is not None and op.weights is None:
                op.weights = self.w[t].astype(np.complex64)
                op._psf = None
            for kp in range(self.K):
                n = op.normal_toeplitz(x[..., kp])
                for k in range(self.K):
                    out[..., k] += np.conj(self.B[t, k]) * self.B[t, kp] * n
        return out


# ---------------------------------------------------------------------------
# SENSE model, data scaling and CG (pics -l2 -r lambda -t ...)
# ---------------------------------------------------------------------------

def estimate_scaling_norm(adj: np.ndarray, rescale: float = 1.0) -> float:
    """src/sense/optcom.c:74-109: p90 of |adj| unless the tail is heavy."""
    mag = np.sort(np.abs(adj.ravel(order="F")).astype(F32))
    n = mag.size
    median = F32(mag[n // 2] / F32(rescale))
    p90 = F32(mag[int(math.trunc(n * 0.9))] / F32(rescale))
    mx = F32(mag[n - 1] / F32(rescale))
    return float(p90 if (mx - p90) < 2 * (p90 - median) else mx)


class SenseOracle:
    """A = NUFFT o S (sense_nc_init, src/sense/modelnc.c:28-67)."""

    def __init__(self, traj, sens, toeplitz=True, periodic=False):
        sens = _as4(sens)
        self.sens = sens
        self.toeplitz = toeplitz
        self.nufft = NufftOracle(traj, sens.shape[:3], periodic=periodic)

    def forward(self, x):
        x = _as4(x)[..., :1]
        return self.nufft.forward(x * self.sens)

    def adjoint(self, y):
        return np.sum(np.conj(self.sens) * self.nufft.adjoint(y), axis=3, keepdims=True)

    def normal(self, x):
        x = _as4(x)[..., :1]
        cx = x * self.sens
        if self.toeplitz:
            n = self.nufft.normal_toeplitz(cx)
        else:
            n = self.nufft.normal_explicit(cx)
        return np.sum(np.conj(self.sens) * n, axis=3, keepdims=True)


def conjgrad(normal, b, lam, maxiter, x0=None, tol=0.0, f32_scalars=False):
    """Plain CG on (normal + lam I) x = b (src/iter/italgos.c:497-572), float64.

    The reference keeps vectors in float32 with float64 dot accumulation and
    float32 alpha/beta; this restatement keeps the vectors in float64. With
    ``f32_scalars`` the squared norms, <p, A p>, alpha and beta are rounded
    to float32 as the reference stores them (src/iter/italgos.c:518-520,
    542-554): that rounding, not the vectors', is what moves unconverged
    iterates (at 30 iterations it puts the oracle within 2e-4 of the
    reference's pics, against 1e-2 with float64 scalars).
    Returns (x, number of iterations run).
    """
    rnd = (lambda v: float(F32(v))) if f32_scalars else float
    x = np.zeros_like(b) if x0 is None else x0.astype(np.complex128).copy()
    r = b - (normal(x) + lam * x)
    p = r.copy()
    rsold = rnd(np.vdot(r, r).real)
    eps2 = (tol * math.sqrt(float(np.vdot(b, b).real))) ** 2
    it = 0
    if rsold == 0.0:
        return x, 0
    for it in range(1, maxiter + 1):
        Ap = normal(p) + lam * p
        pAp = rnd(np.vdot(p, Ap).real)
        if pAp == 0.0:
            break
        alpha = rnd(rsold / pAp)
        x = x + alpha * p
        r = r - alpha * Ap
        rsnew = rnd(np.vdot(r, r).real)
        beta = rnd(rsnew / rsold)
        rsold = rsnew
        if rsnew <= eps2:
            break
        p = beta * p + r
    return x, it


def pics_l2(traj, ksp, sens, lam=0.01, maxiter=30, toeplitz=True, scaling=0.0, rescale=False,
            periodic=False, f32_scalars=False):
    """``bart pics -l2 -r lam -i maxiter -t traj ksp sens out`` (src/pics.c).

    Data scaling by estimate_scaling_norm of the adjoint unless ``scaling``
    is given (``-w``), ksp /= scale (src/pics.c:499-530), then CG from zero
    on (A^H A + lam) x = A^H y (src/iter/lsqr.c:52-62, src/grecon/italgo.c:84-103).
    Returns (image [X,Y,Z,1], scale used).
    """
    A = SenseOracle(traj, sens, toeplitz=toeplitz, periodic=periodic)
    y = np.asarray(ksp).reshape(A.nufft.M, -1).astype(np.complex128)
    if scaling == 0.0:
        adj = A.adjoint(y)
        scaling = estimate_scaling_norm(adj)
        if scaling == 0.0:
            scaling = 1.0
    y = y * float(F32(1.0 / scaling))
    b = A.adjoint(y)
    x, _ = conjgrad(A.normal, b, lam, maxiter, f32_scalars=f32_scalars)
    if rescale:
        x = x * scaling
    return x, scaling


def normal_residual(A, x, b, lam):
    """True relative normal-equation residual ||b - (A^H A + lam) x|| / ||b||."""
    r = b - (A.normal(x) + lam * _as4(x)[..., :1])
    return float(np.linalg.norm(r) / np.linalg.norm(b))


# ---------------------------------------------------------------------------
# FP64 direct NDFT (exact transform the NUFFT approximates)
# ---------------------------------------------------------------------------

def ndft_forward(traj, img):
    """y_m = N^-1/2 sum_n x_n exp(-2 pi i k_m . (n - N/2) / N), float64."""
    img = _as4(img)
    dims3 = img.shape[:3]
    traj = np.asarray(traj, dtype=np.float64).reshape(3, -1)
    E = []
    for ax in range(3):
        n = dims3[ax]
        grid = np.arange(n) - n // 2
        E.append(np.exp(-2j * np.pi * np.outer(traj[ax], grid) / n))
    scale = 1.0 / math.sqrt(float(np.prod(dims3)))
    return np.einsum("mx,my,mz,xyzc->mc", E[0], E[1], E[2], img, optimize=True) * scale


def ndft_adjoint(traj, ksp, dims3):
    traj = np.asarray(traj, dtype=np.float64).reshape(3, -1)
    ksp = np.asarray(ksp).reshape(traj.shape[1], -1).astype(np.complex128)
    E = []
    for ax in range(3):
        n = dims3[ax]
        grid = np.arange(n) - n // 2
        E.append(np.exp(2j * np.pi * np.outer(traj[ax], grid) / n))
    scale = 1.0 / math.sqrt(float(np.prod(dims3)))
    return np.einsum("mx,my,mz,mc->xyzc", E[0], E[1], E[2], ksp, optimize=True) * scale

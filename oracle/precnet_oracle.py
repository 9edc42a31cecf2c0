"""CPU oracle of the learned preconditioner network (test infrastructure only).

The network has no counterpart in the reference: it plugs into the
preconditioner slot that the reference's lsqr2_create chains in front of CG
(src/iter/lsqr.c:126-143). This is a NumPy statement of the forward pass,
the loss and the backward pass the library runs on the GPU: 6 layers of
3x3 convolutions with zero padding, 2 -> 32 -> 32 -> 32 -> 32 -> 32 -> 2
channels, ReLU after layers 1-5, loss (1/nimg) sum |out - target|^2.

`bf16=True` rounds exactly where the GPU path stores bfloat16 (weights,
layer 1-5 activations, the gradients entering layers 5..1) so the two agree
up to float32 summation order; `bf16=False` is the plain float64 network
used for the finite-difference check of the backward pass.
"""

from __future__ import annotations

import numpy as np

C = 32
CIN = [2, C, C, C, C, C]
COUT = [C, C, C, C, C, 2]


def offsets():
    """(weight offset, bias offset, end) per layer in the parameter vector."""
    out, o = [], 0
    for ci, co in zip(CIN, COUT):
        w = co * 9 * ci
        out.append((o, o + w, o + w + co))
        o += w + co
    return out


NPARAMS = offsets()[-1][2]


def init_params(rng, scale=1.0):
    """He-style initial weights (fan-in 9 cin), zero biases."""
    p = np.zeros(NPARAMS, dtype=np.float32)
    for (wo, bo, _), ci, co in zip(offsets(), CIN, COUT):
        p[wo:bo] = (rng.standard_normal(bo - wo) * scale * np.sqrt(2.0 / (9 * ci))).astype(np.float32)
    return p


def bf16(a):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(p, round_bf16):
    layers = []
    for (wo, bo, e), ci, co in zip(offsets(), CIN, COUT):
        w = np.asarray(p[wo:bo], dtype=np.float64).reshape(co, 3, 3, ci)
        if round_bf16:
            w = bf16(w.astype(np.float32))
        layers.append((w.astype(np.float64), np.asarray(p[bo:e], dtype=np.float64)))
    return layers


def to_channels(z):
    """complex [X, Y, n] (BART order) -> float [n, Y, X, 2] (NHWC)."""
    z = np.asarray(z).reshape(z.shape[0], z.shape[1], -1, order="F")
    return np.stack([z.real, z.imag], axis=-1).transpose(2, 1, 0, 3).astype(np.float64)


def from_channels(a):
    """float [n, Y, X, 2] -> complex [X, Y, n]."""
    return (a[..., 0] + 1j * a[..., 1]).transpose(2, 1, 0)


def conv3(a, w):
    """3x3 'same' convolution, a [n, Y, X, ci], w [co, 3, 3, ci] ->
    out[n, y, x, co] = sum w[co, ky, kx, ci] a[n, y + ky - 1, x + kx - 1, ci]."""
    n, Y, X, ci = a.shape
    ap = np.zeros((n, Y + 2, X + 2, ci))
    ap[:, 1:-1, 1:-1] = a
    out = 0.
    for ky in range(3):
        for kx in range(3):
            out = out + np.einsum("nyxc,oc->nyxo", ap[:, ky:ky + Y, kx:kx + X], w[:, ky, kx], optimize=True)
    return out


def conv3_wgrad(a, g):
    """dW[co, ky, kx, ci] = sum g[n, y, x, co] a[n, y + ky - 1, x + kx - 1, ci]."""
    n, Y, X, ci = a.shape
    ap = np.zeros((n, Y + 2, X + 2, ci))
    ap[:, 1:-1, 1:-1] = a
    dw = np.zeros((g.shape[-1], 3, 3, ci))
    for ky in range(3):
        for kx in range(3):
            dw[:, ky, kx] = np.einsum("nyxo,nyxc->oc", g, ap[:, ky:ky + Y, kx:kx + X], optimize=True)
    return dw


def conv3_dgrad(g, w):
    """Gradient of conv3 with respect to its input: correlation of g with the
    flipped, transposed kernel."""
    wt = w[:, ::-1, ::-1, :].transpose(3, 1, 2, 0)
    return conv3(g, wt)


def forward(p, x, bf16_mode=True):
    """x: float [n, Y, X, 2]; returns (out [n, Y, X, 2], activations)."""
    rnd = bf16 if bf16_mode else (lambda v: v)
    layers = unpack(p, bf16_mode)
    acts = [x]
    a = x
    for i, (w, b) in enumerate(layers):
        u = conv3(a, w) + b
        if i < 5:
            a = rnd(np.maximum(u, 0.0)).astype(np.float64)
            acts.append(a)
        else:
            a = u
    return a, acts


def loss_and_grad(p, x, target, bf16_mode=True):
    """loss = (1/n) sum |out - target|^2 and d loss / d params (float64)."""
    rnd = bf16 if bf16_mode else (lambda v: v)
    layers = unpack(p, bf16_mode)
    n = x.shape[0]
    out, acts = forward(p, x, bf16_mode)
    d = out - target
    loss = float(np.sum(d * d) / n)
    g = 2.0 / n * d
    grads = np.zeros(NPARAMS)
    offs = offsets()
    for i in range(5, -1, -1):
        w, _ = layers[i]
        a = acts[i]
        wo, bo, e = offs[i]
        grads[wo:bo] = conv3_wgrad(a, g).ravel()
        grads[bo:e] = g.sum(axis=(0, 1, 2))
        if i > 0:
            ga = conv3_dgrad(g, w)
            g = rnd(np.where(a > 0, ga, 0.0)).astype(np.float64)
    return loss, grads

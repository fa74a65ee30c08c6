"""FP64 restatement of the CNN closure (new; no reference counterpart) with the
BF16 rounding of weights and activations emulated, for checking the tensor-core
kernels.  Test infrastructure only (see ``oracle/__init__.py``).

The network: input channels (u_x, u_y, u_z, z) with z = (log Re_Delta - mu)/sigma,
Re_Delta = Delta^2 sqrt(<|grad u|^2>)/nu (the ``fullchain`` convention,
src/nets.jl:311-331); four 3x3x3 periodic cross-correlations
4->32->32->32->6 with GELU between them.  GELU is the activation the
reference's networks use (``gelu`` in src/nets.jl:187, 191, 549-551, from
NNlib through Lux), the tanh form 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))).
"""

from __future__ import annotations

import math

import numpy as np

from .spectral import Grid, getenergy, twothirds, vectorgradient

__all__ = ["bf16", "f16", "split_parts", "gelu", "gelu_grad", "cnn_redelta_channel", "cnn_rows", "cnn_field",
           "cnn_rows_split"]

_GELU_C = math.sqrt(2.0 / math.pi)
_GELU_A = 0.044715


def gelu(x):
    """NNlib ``gelu`` (tanh form), used by the reference's convolutional nets."""
    x = np.asarray(x, dtype=np.float64)
    return 0.5 * x * (1.0 + np.tanh(_GELU_C * (x + _GELU_A * x ** 3)))


def gelu_grad(x):
    """d gelu / dx of the tanh form."""
    x = np.asarray(x, dtype=np.float64)
    t = np.tanh(_GELU_C * (x + _GELU_A * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * _GELU_C * (1.0 + 3.0 * _GELU_A * x * x)


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    b = f.view(np.uint32).astype(np.uint64)
    lsb = (b >> 16) & 1
    b = ((b + 0x7FFF + lsb) & 0xFFFF0000).astype(np.uint32)
    return b.view(np.float32).astype(np.float64)


def f16(x):
    """Round to the nearest FP16 value (ties to even, subnormals kept), returned as float64."""
    return np.asarray(x, dtype=np.float64).astype(np.float16).astype(np.float64)


def split_parts(x, rnd=f16):
    """The split precision's two parts of x: hi = rnd(x), lo = rnd(x - hi)."""
    x = np.asarray(x, dtype=np.float64)
    hi = rnd(x)
    return hi, rnd(x - hi)


def cnn_redelta_channel(u, g: Grid, delta, nu, mu=0.0, sigma=1.0):
    A = vectorgradient(u, g)
    a2 = sum(getenergy(twothirds(v, g)) for v in A.values())
    return (math.log(delta * delta * math.sqrt(a2) / nu) - mu) / sigma


def _conv(act, w, b, z_lo, z_hi, y_lo, y_hi):
    """Periodic 3x3x3 cross-correlation on the window; act: (C, Z, Y, X) covering
    rows z_lo-1..z_hi+1, y_lo-1..y_hi+1 (window-relative), full periodic x."""
    cout = w.shape[0]
    Z = z_hi - z_lo + 1
    Y = y_hi - y_lo + 1
    X = act.shape[-1]
    out = np.zeros((cout, Z, Y, X))
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                sl = act[:, z_lo + kz - 1:z_lo + kz - 1 + Z, y_lo + ky - 1:y_lo + ky - 1 + Y, :]
                sl = np.roll(sl, -(kx - 1), axis=-1)
                out += np.einsum("oc,czyx->ozyx", w[:, :, kz, ky, kx], sl)
    return out + b[:, None, None, None]


def cnn_rows(uphys, zval, weights, biases, rows, round_bf16=True):
    """tau (6, len(rows), n) at the x-rows ``rows`` = [(y, z), ...] of the periodic grid.

    uphys: (3, n, n, n) physical velocity indexed [c, z, y, x].  With
    ``round_bf16=False`` the network is evaluated in FP64 without rounding.
    """
    n = uphys.shape[-1]
    rnd = bf16 if round_bf16 else (lambda x: np.asarray(x, dtype=np.float64))
    ws = [rnd(w) for w in weights]
    out = []
    for (y0, z0) in rows:
        idx_z = [(z0 + d) % n for d in range(-4, 5)]
        idx_y = [(y0 + d) % n for d in range(-4, 5)]
        win = uphys[:, idx_z][:, :, idx_y]  # (3, 9, 9, n)
        act = np.concatenate([rnd(win), np.full((1,) + win.shape[1:], rnd(np.array([zval]))[0])], 0)
        for li in range(4):
            h = 4 - li  # input window half-width
            act = _conv(act, ws[li], biases[li].astype(np.float64), 1, 2 * h - 1, 1, 2 * h - 1)
            if li < 3:
                act = rnd(gelu(act))
        out.append(act[:, 0, 0, :])
    return np.stack(out, 1)


def cnn_field(uphys, zval, weights, biases, round_bf16=True):
    """tau (6, n, n, n) of the CNN closure on the whole periodic grid (the same
    network and BF16 roundings as :func:`cnn_rows`); each 3x3x3 tap is one
    (C_out x C_in) by (C_in x n^3) product of a rolled activation."""
    rnd = bf16 if round_bf16 else (lambda x: np.asarray(x, dtype=np.float64))
    act = np.concatenate([rnd(uphys), np.full((1,) + uphys.shape[1:], rnd(np.array([zval]))[0])], 0)
    for li, (w, b) in enumerate(zip(weights, biases)):
        w = rnd(w)
        out = np.zeros((w.shape[0],) + act.shape[1:])
        for kz in range(3):
            for ky in range(3):
                for kx in range(3):
                    sl = np.roll(act, shift=(1 - kz, 1 - ky, 1 - kx), axis=(1, 2, 3))
                    out += np.tensordot(w[:, :, kz, ky, kx], sl, axes=(1, 0))
        act = out + np.asarray(b, dtype=np.float64)[:, None, None, None]
        if li < 3:
            act = rnd(gelu(act))
    return act


def cnn_rows_split(uphys, zval, weights, biases, rows, wscale=64.0):
    """tau at ``rows`` as the split precision computes it: every operand x =
    hi + lo in FP16 parts (weights scaled by ``wscale`` before the split and
    the sum scaled back), each convolution the three products A_hi W_hi +
    A_lo W_hi + A_hi W_lo accumulated exactly (FP64 here), GELU unrounded and
    its output split again.  Emulates the rounding of the parts, not the FP32
    accumulation order of the tensor cores."""
    out = []
    n = uphys.shape[-1]
    wparts = [split_parts(np.asarray(w, dtype=np.float64) * wscale) for w in weights]
    for (y0, z0) in rows:
        idx_z = [(z0 + d) % n for d in range(-4, 5)]
        idx_y = [(y0 + d) % n for d in range(-4, 5)]
        win = uphys[:, idx_z][:, :, idx_y]
        act = np.concatenate([np.asarray(win, dtype=np.float64), np.full((1,) + win.shape[1:], zval)], 0)
        for li in range(4):
            h = 4 - li
            ah, al = split_parts(act)
            wh, wl = wparts[li]
            zero = np.zeros_like(np.asarray(biases[li], dtype=np.float64))
            acc = sum(_conv(a_, w_, zero, 1, 2 * h - 1, 1, 2 * h - 1) for a_, w_ in ((ah, wh), (al, wh), (ah, wl)))
            act = acc / wscale + np.asarray(biases[li], dtype=np.float64)[:, None, None, None]
            if li < 3:
                act = gelu(act)
        out.append(act[:, 0, 0, :])
    return np.stack(out, 1)

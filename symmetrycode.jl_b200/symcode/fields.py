"""Seeded synthetic initial fields on the host (the reference's ``randomfield``,
src/solver.jl:576-641), in the solver's compact 2/3 layout.

The reference draws complex normal coefficients, makes the kx = 0 plane
Hermitian (``symmetrize!``), projects them onto divergence-free fields
(``project!``), drops the mean (``twothirds!``) and rescales every integer
shell ``s <= |k| < s + 1`` so that its energy is ``totalenergy * profile(s) /
sum(profile)`` over ``s = 0 .. floor(sqrt(D) n/2)``.  Modes outside the 2/3
cube are zeroed by the reference's final ``twothirds!``, so only the retained
cube is drawn here.  The stream is numpy ``PCG64(seed)``: per component x, y[, z],
all real parts then all imaginary parts, each N(0, 1/2), over the compact array
in C order (Julia's Xoshiro stream is not reproduced).

Compact layout (numpy C order): ``(K2, K2, K1)`` in 3D, ``(K2, K1)`` in 2D, with
``K1 = n//3 + 1`` (kx = 0 .. n//3) and ``K2 = 2 (n//3) + 1`` (k = 0 .. n//3, then
-n//3 .. -1).  :func:`compact_to_full` scatters it into the full RFFT layout
``(n, n, n//2 + 1)`` / ``(n, n//2 + 1)`` the C ABI takes.
"""

from __future__ import annotations

import math

import numpy as np

__all__ = ["compact_shape", "peak_profile", "random_field_compact", "compact_to_full"]


def compact_shape(D: int, n: int):
    k = n // 3
    return (2 * k + 1,) * (D - 1) + (k + 1,)


def peak_profile(k, kpeak):
    """``peak_profile`` (src/solver.jl:523): k^4 exp(-2 (k/kpeak)^2)."""
    return k ** 4 * math.exp(-2 * (k / kpeak) ** 2)


def _signed_wavenumbers(n: int) -> np.ndarray:
    """Signed wavenumber of each compact y/z index."""
    k = n // 3
    i = np.arange(2 * k + 1)
    return np.where(i <= k, i, i - (2 * k + 1))


def _hermitian_plane(c: np.ndarray, n: int, D: int) -> None:
    """Make the kx = 0 plane Hermitian in place: of each pair (k, -k) the
    member with the larger FFT index (y first, then z) takes the conjugate of
    the other; the k = 0 coefficient becomes real."""
    s = _signed_wavenumbers(n)
    fft = s % n                       # FFT index of each compact index
    partner = np.where(s == 0, 0, np.where(s > 0, len(s) - s, -s))  # compact index of -s
    if D == 2:
        plane = c[:, 0].copy()
        take = fft > (-fft) % n
        new = plane.copy()
        new[take] = np.conj(plane[partner[take]])
        new[0] = plane[0].real
        c[:, 0] = new
        return
    plane = c[:, :, 0].copy()
    fz, fy = np.meshgrid(fft, fft, indexing="ij")
    pz, py = (-fz) % n, (-fy) % n
    take = (fy > py) | ((fy == py) & (fz > pz))
    iz, iy = np.meshgrid(np.arange(len(s)), np.arange(len(s)), indexing="ij")
    new = plane.copy()
    new[take] = np.conj(plane[partner[iz[take]], partner[iy[take]]])
    new[0, 0] = plane[0, 0].real
    c[:, :, 0] = new


def random_field_compact(D: int, n: int, seed: int, kpeak: float = 4.0, totalenergy: float = 1.0,
                         profile=None, dtype=np.complex128):
    """Seeded solenoidal random field with shell spectrum E(k) ~ profile(k)
    (default ``peak_profile(k, kpeak)``), as a list of D compact arrays."""
    if profile is None:
        def profile(kk):
            return peak_profile(kk, kpeak)
    shape = compact_shape(D, n)
    rng = np.random.Generator(np.random.PCG64(seed))
    half = math.sqrt(0.5)
    u = []
    for _ in range(D):
        re = rng.standard_normal(shape)
        im = rng.standard_normal(shape)
        u.append((re + 1j * im) * half)
    for c in u:
        _hermitian_plane(c, n, D)
    # divergence-free part: u - k (k . u) / |k|^2, mean dropped
    s = _signed_wavenumbers(n).astype(np.float64)
    kx = np.arange(n // 3 + 1, dtype=np.float64)
    ks = [kx[None, :], s[:, None]] if D == 2 else [kx[None, None, :], s[None, :, None], s[:, None, None]]
    k2 = sum(a * a for a in ks)
    with np.errstate(invalid="ignore", divide="ignore"):
        kdotu = sum(a * c for a, c in zip(ks, u)) / k2
    kdotu.flat[0] = 0
    u = [c - a * kdotu for a, c in zip(ks, u)]
    for c in u:
        c.flat[0] = 0
    # shell energies (kx > 0 counted twice: their conjugates are not stored)
    weight = np.ones(shape)
    weight[..., 1:] = 2.0
    energy = sum(np.abs(c) ** 2 for c in u) / 2
    k2i = np.rint(k2).astype(np.int64)
    shell = np.floor(np.sqrt(k2i)).astype(np.int64)
    shell = np.where((shell + 1) ** 2 <= k2i, shell + 1, shell)
    shell = np.where(shell ** 2 > k2i, shell - 1, shell)
    smax = int(math.floor(math.sqrt(D) * (n // 2)))
    prof = np.array([profile(j) for j in range(smax + 1)])
    eshell = np.bincount(shell.ravel(), weights=(weight * energy).ravel(), minlength=smax + 1)[: smax + 1]
    target = totalenergy * prof / prof.sum()
    with np.errstate(invalid="ignore", divide="ignore"):
        scale = np.where(eshell > 0, np.sqrt(target / eshell), 0.0)
    f = scale[shell]
    return [(c * f).astype(dtype) for c in u]


def compact_to_full(cc: np.ndarray, n: int) -> np.ndarray:
    """Scatter one compact component into the full RFFT layout (zeros elsewhere)."""
    D = cc.ndim
    k = n // 3
    fft = _signed_wavenumbers(n) % n
    full = np.zeros((n,) * (D - 1) + (n // 2 + 1,), dtype=cc.dtype)
    if D == 2:
        full[np.ix_(fft, np.arange(k + 1))] = cc
    else:
        full[np.ix_(fft, fft, np.arange(k + 1))] = cc
    return full

"""Exact triad-sum oracle for sparse spectral fields (no FFT).

Test infrastructure only (see ``oracle/__init__.py``).  For a velocity field
with a few hundred retained Fourier modes the pseudo-spectral products of
``nonlinearity!`` (src/solver.jl:434-456) are finite sums over mode pairs:

    σ_ij(k) = F[(P u_i)(P u_j)](k) / n^D = Σ_{p + q ≡ k (mod n)} û_i(p) û_j(q),

where the sum runs over the full Hermitian mode set (each stored mode and its
conjugate partner) and ``mod n`` per axis is the aliasing of the n-point grid.
With that, ``viscosity!`` (:458-476), ``tensordivergence!`` (:509-521),
``twothirds!`` (:371-389), ``project!`` (:350-368), ``cutoff!`` and
``gaussianfilter!`` (src/filtering.jl:9-67) and ``sfs!`` (src/data.jl:625-642)
become pointwise operations on the sparse output set.  The sums are exact in
FP64 (no transform roundoff), at any n, so they pin the FFT-based paths at the
production size 810^3 where a dense FFT oracle is expensive.

A sparse field is a pair ``(k, u)``: ``k`` an (M, 3) int array of wavevectors
in the RFFT half space (kx > 0, or kx = 0 with (ky, kz) > 0 lexicographically)
and ``u`` an (M, 3) complex array of the velocity at those modes; the conjugate
half is implied.
"""

from __future__ import annotations

import math

import numpy as np

__all__ = ["random_sparse_field", "full_modes", "triad_products", "convectiondiffusion",
           "rk4_rhs", "sfs", "to_rfft_index", "dense_rfft"]

_PAIRS = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (2, 0)]  # xx yy zz xy yz zx


def _canonical(k):
    """True for wavevectors in the RFFT half space used to store a sparse field."""
    kx, ky, kz = k[:, 0], k[:, 1], k[:, 2]
    return (kx > 0) | ((kx == 0) & ((ky > 0) | ((ky == 0) & (kz > 0))))


def random_sparse_field(n, nmodes, seed, kmax=None, extra=()):
    """Seeded solenoidal sparse field with ``nmodes`` random retained modes
    (|k_i| <= kmax, default n÷3) plus the wavevectors ``extra`` (edge cases:
    the cube's faces and corners, kx = 0, the forced band).  Amplitudes decay
    like |k|^-1 so that the field looks like a turbulent spectrum, not noise."""
    kmax = n // 3 if kmax is None else kmax
    rng = np.random.Generator(np.random.PCG64(seed))
    cand = rng.integers(-kmax, kmax + 1, size=(4 * nmodes, 3))
    cand[:, 0] = np.abs(cand[:, 0])
    ks = [tuple(e) for e in extra] + [tuple(c) for c in cand]
    seen, keep = set(), []
    for kk in ks:
        a = np.array(kk)
        if not _canonical(a[None])[0]:
            a = -a
        if not _canonical(a[None])[0]:
            continue  # k = 0
        t = tuple(int(x) for x in a)
        if t in seen:
            continue
        seen.add(t)
        keep.append(t)
        if len(keep) >= nmodes + len(extra):
            break
    k = np.array(keep, dtype=np.int64)
    z = (rng.standard_normal((len(k), 3)) + 1j * rng.standard_normal((len(k), 3))) * math.sqrt(0.5)
    kf = k.astype(np.float64)
    k2 = (kf ** 2).sum(1)
    z -= kf * ((kf * z).sum(1) / k2)[:, None]  # Leray projection per mode
    z *= (1.0 / np.sqrt(k2))[:, None]
    return k, z


def full_modes(k, u):
    """The full Hermitian mode set: the stored modes and their conjugates."""
    return np.concatenate([k, -k]), np.concatenate([u, np.conj(u)])


def _wrap(k, n):
    """Wavevector modulo the n-point grid, into [-n/2, n/2)."""
    return (k + n // 2) % n - n // 2


def triad_products(k, u, n, keep):
    """σ_ij at every output wavevector ``keep(kout)`` accepts (kout in the RFFT
    half: kx >= 0 after wrapping).  Returns (kout (K, 3), sigma (K, 6))."""
    kf, uf = full_modes(k, u)
    P = len(kf)
    ko = _wrap(kf[:, None, :] + kf[None, :, :], n).reshape(-1, 3)
    sel = (ko[:, 0] >= 0) & keep(ko)
    ko = ko[sel]
    ii, jj = np.nonzero(sel.reshape(P, P))
    base = n + 1
    key = ((ko[:, 0] + n // 2) * base + (ko[:, 1] + n // 2)) * base + (ko[:, 2] + n // 2)
    uniq, inv = np.unique(key, return_inverse=True)
    kout = np.stack([uniq // (base * base) - n // 2, (uniq // base) % base - n // 2, uniq % base - n // 2], 1)
    sig = np.zeros((len(uniq), 6), dtype=np.complex128)
    for c, (i, j) in enumerate(_PAIRS):
        v = uf[ii, i] * uf[jj, j]
        sig[:, c] = np.bincount(inv, weights=v.real, minlength=len(uniq)) + \
            1j * np.bincount(inv, weights=v.imag, minlength=len(uniq))
    return kout, sig


def _retained(n):
    kc = n // 3

    def keep(ko):
        return (np.abs(ko) <= kc).all(1) & (np.abs(ko).sum(1) > 0)
    return keep


def _lookup(kout, k, u):
    """u at the wavevectors kout (zero where the sparse field has no mode);
    kout in the RFFT half, so stored modes or conjugates of kx = 0 modes."""
    kf, uf = full_modes(k, u)
    table = {tuple(int(x) for x in kk): i for i, kk in enumerate(kf)}
    out = np.zeros((len(kout), 3), dtype=np.complex128)
    for r, kk in enumerate(kout):
        i = table.get((int(kk[0]), int(kk[1]), int(kk[2])))
        if i is not None:
            out[r] = uf[i]
    return out


def convectiondiffusion(k, u, n, visc):
    """``twothirds!(convectiondiffusion!(u))`` (src/solver.jl:949-953) of a sparse
    field on an n-point grid (l = 2π): returns (kout, du (K, 3)) over the
    retained output modes, including the input modes themselves."""
    kout, sig = triad_products(k, u, n, _retained(n))
    # add the input modes (and the conjugates of kx = 0 ones) that no triad reaches
    kf, _ = full_modes(k, u)
    extra = kf[kf[:, 0] >= 0]
    base = n + 1

    def keyof(a):
        return ((a[:, 0] + n // 2) * base + (a[:, 1] + n // 2)) * base + (a[:, 2] + n // 2)
    missing = ~np.isin(keyof(extra), keyof(kout))
    if missing.any():
        kout = np.concatenate([kout, extra[missing]])
        sig = np.concatenate([sig, np.zeros((int(missing.sum()), 6), dtype=np.complex128)])
    uk = _lookup(kout, k, u)
    ks = kout.astype(np.float64)
    idx = {}
    for c, (i, j) in enumerate(_PAIRS):
        idx[(i, j)] = c
        idx[(j, i)] = c
    du = np.zeros((len(kout), 3), dtype=np.complex128)
    for i in range(3):
        for j in range(3):
            s = sig[:, idx[(i, j)]]
            visc_ij = visc * 1j * (ks[:, j] * uk[:, i] + ks[:, i] * uk[:, j])
            du[:, i] += -1j * ks[:, j] * (s - visc_ij)
    return kout, du


def rk4_rhs(k, u, n, visc, eps=None):
    """The RK4 stage derivative P(twothirds(convectiondiffusion(u))) + A u|band of
    ``oracle.spectral.rk4_rhs``, on a sparse field."""
    kout, du = convectiondiffusion(k, u, n, visc)
    ks = kout.astype(np.float64)
    k2 = (ks ** 2).sum(1)
    p = (ks * du).sum(1) / k2
    du = du - ks * p[:, None]
    if eps is not None:
        uk = _lookup(kout, k, u)
        band = (k2 >= 1) & (k2 < 9)
        w = np.where(kout[:, 0] > 0, 2.0, 1.0)
        ef = float(np.sum((w * (np.abs(uk) ** 2).sum(1))[band])) / 2
        A = eps / (2 * ef) if ef > 0 else 0.0
        du[band] += A * uk[band]
    return kout, du


def sfs(k, u, n, nb, delta):
    """``sfs!`` (src/data.jl:625-642) from a sparse n-grid field to an nb grid at
    filter width Δ (``None``: no Gaussian).  Returns (kout, ubar (K, 3),
    tau (K, 6)) on the retained LES modes (|k_i| <= nb÷3, k != 0, kx >= 0)."""
    kc = nb // 3

    def keep(ko):
        return (np.abs(ko) <= kc).all(1) & (np.abs(ko).sum(1) > 0)

    def gauss(ks):
        if delta is None:
            return np.ones(len(ks))
        k2 = (ks.astype(np.float64) ** 2).sum(1)
        return np.where(k2 < 9.0, 1.0, np.exp(-delta ** 2 * k2 / 24))

    # ubar = P_les G cutoff(u): the retained LES modes of u, filtered
    kb = k[(np.abs(k) <= kc).all(1)]
    ub = u[(np.abs(k) <= kc).all(1)] * gauss(kb)[:, None]
    kd, sd = triad_products(k, u, n, keep)  # DNS products at the LES modes
    kl, sl = triad_products(kb, ub, nb, keep)  # LES products of ubar
    base = n + 1

    def keyof(a):
        return ((a[:, 0] + n // 2) * base + (a[:, 1] + n // 2)) * base + (a[:, 2] + n // 2)
    kbf, _ = full_modes(kb, ub)
    kbf = kbf[kbf[:, 0] >= 0]
    allk = np.unique(np.concatenate([keyof(kd), keyof(kl), keyof(kbf)]))
    kout = np.stack([allk // (base * base) - n // 2, (allk // base) % base - n // 2, allk % base - n // 2], 1)
    pos = {int(x): i for i, x in enumerate(allk)}
    tau = np.zeros((len(kout), 6), dtype=np.complex128)
    g = gauss(kout)
    s1 = np.zeros_like(tau)
    s2 = np.zeros_like(tau)
    for kk, s in zip(keyof(kd), sd):
        s1[pos[int(kk)]] = s
    for kk, s in zip(keyof(kl), sl):
        s2[pos[int(kk)]] = s
    tau = g[:, None] * s1 - s2
    tr = (tau[:, 0] + tau[:, 1] + tau[:, 2]) / 3
    tau[:, :3] -= tr[:, None]
    ubar = _lookup(kout, kb, ub)
    return kout, ubar, tau


def to_rfft_index(kout, n):
    """(iz, iy, ix) of wavevectors (kx >= 0) in the full RFFT layout (n, n, n/2+1)."""
    return kout[:, 2] % n, kout[:, 1] % n, kout[:, 0]


def dense_rfft(k, u, n):
    """The sparse field in the full RFFT layout (3 arrays (n, n, n/2+1)), for small n."""
    kf, uf = full_modes(k, u)
    m = kf[:, 0] >= 0
    out = [np.zeros((n, n, n // 2 + 1), dtype=np.complex128) for _ in range(3)]
    iz, iy, ix = to_rfft_index(kf[m], n)
    for c in range(3):
        out[c][iz, iy, ix] = uf[m][:, c]
    return out

"""DNS -> LES filter and sub-filter stress: FP64 restatement of
``src/filtering.jl`` and ``sfs!`` (``src/data.jl:614-642``).

Test infrastructure only (see ``oracle/__init__.py``).
"""

from __future__ import annotations

import math

import numpy as np

from .spectral import (Grid, make_tracefree, nonlinearity, twothirds,
                       wavenumbers_full)

__all__ = ["cutoff_index", "cutoff", "inverse_cutoff", "gaussianfilter", "sfs", "filter_reynolds"]


def cutoff_index(nbar, n, i0, is1):
    """``cutoff_index`` (src/filtering.jl:9-13), 0-based: coarse index -> fine index."""
    imax = nbar // 2 + (1 if is1 else 0)  # 1-based bound
    i1 = np.asarray(i0) + 1
    return np.where(i1 > imax, n - nbar + i1, i1) - 1


def _fine_indices(g_dns: Grid, g_les: Grid):
    nb, n = g_les.n, g_dns.n
    ix = cutoff_index(nb, n, np.arange(nb // 2 + 1), True)
    iy = cutoff_index(nb, n, np.arange(nb), False)
    return ix, iy


def cutoff(u, g_dns: Grid, g_les: Grid):
    """``cutoff!`` (src/filtering.jl:28-34): copy the LES-grid modes out of a DNS spectrum."""
    ix, iy = _fine_indices(g_dns, g_les)
    if g_dns.D == 2:
        return np.ascontiguousarray(u[np.ix_(iy, ix)])
    return np.ascontiguousarray(u[np.ix_(iy, iy, ix)])


def inverse_cutoff(ubar, g_dns: Grid, g_les: Grid):
    """``inverse_cutoff!`` (src/filtering.jl:36-42) into a zero DNS array."""
    ix, iy = _fine_indices(g_dns, g_les)
    out = np.zeros(g_dns.spec_shape, dtype=ubar.dtype)
    if g_dns.D == 2:
        out[np.ix_(iy, ix)] = ubar
    else:
        out[np.ix_(iy, iy, ix)] = ubar
    return out


def gaussianfilter(u, delta, g: Grid):
    """``gaussianfilter!`` (src/filtering.jl:44-67): × exp(-Δ² k² / 24), except k² < (3·2π/l)²."""
    ks = wavenumbers_full(g)
    k2 = sum(k * k for k in ks)
    w = np.exp(-delta ** 2 * k2 / 24)
    kbound2 = (2 * math.pi / g.l * 3) ** 2
    w = np.where(k2 < kbound2, 1.0, w)
    return u * w


def sfs(u, g_dns: Grid, g_les: Grid, delta):
    """``sfs!`` (src/data.jl:625-642).

    Returns ``(ubar, tau)``: ``ubar = P_les G_Δ cutoff(u)``,
    ``tau = tracefree(P_les[G_Δ cutoff(σ_dns) - σ_les(ubar)])`` with ``σ`` the
    (untruncated) ``nonlinearity!`` outputs.  ``delta=None`` skips the Gaussian.
    """
    sig_dns = nonlinearity(u, g_dns)
    ubar = []
    for c in u:
        b = cutoff(c, g_dns, g_les)
        if delta is not None:
            b = gaussianfilter(b, delta, g_les)
        ubar.append(twothirds(b, g_les))
    sbar1 = []
    for s in sig_dns:
        b = cutoff(s, g_dns, g_les)
        if delta is not None:
            b = gaussianfilter(b, delta, g_les)
        sbar1.append(b)
    sbar2 = nonlinearity(ubar, g_les)
    tau = [twothirds(a - b, g_les) for a, b in zip(sbar1, sbar2)]
    return ubar, make_tracefree(tau, g_dns.D)


def filter_reynolds(ubar, g: Grid, visc, delta):
    """``filter_reynolds`` (src/solver.jl:768-774): Δ² √(Σ_ab getenergy(twothirds(i k_b ū_a))) / ν."""
    from .spectral import getenergy, vectorgradient
    A = vectorgradient(ubar, g)
    a2 = sum(getenergy(twothirds(v, g)) for v in A.values())
    return delta ** 2 * math.sqrt(a2) / visc

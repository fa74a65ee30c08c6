"""Classical LES closures: FP64 restatement of ``src/closures.jl``.

Test infrastructure only (see ``oracle/__init__.py``).

A physical velocity-gradient field ``G`` is a dict keyed ``'xx', 'xy', ...``
with ``G['ab'] = ∂_b u_a`` (``vectorgradient!``, src/solver.jl:711-733), the
reference's ``tensorat`` convention ``G[i, j] = GG.ij`` (src/closures.jl:6-11).
Closures return the packed physical stress, an array of shape
``(tensordim, *phys_shape)`` in the order xx, yy, zz, xy, yz, zx -- the memory
layout of the reference's ``(n, n, n, 6)`` column-major ``τpack``.
"""

from __future__ import annotations

import math

import numpy as np
import scipy.fft as sfft

from .filtering import gaussianfilter
from .spectral import (WORKERS, Grid, nonlinearity, pairs, strainrate, to_phys,
                       twothirds, make_tracefree)

__all__ = ["mlp_fullchain", "tbnn", "GRAD_ORDER", "grad_matrix", "store_sym", "clark", "smagorinsky", "verstappen",
           "bardina", "dynamic_smagorinsky", "smagorinsky_tensor", "smagorinsky_ml_mm",
           "dynsmag_coefficient", "test_filter_phys"]

# ``tensorfield_nonsym`` component order (src/solver.jl:264-277): xx yx zx xy yy zy xz yz zz
GRAD_ORDER = ["xx", "yx", "zx", "xy", "yy", "zy", "xz", "yz", "zz"]


def grad_matrix(G, D):
    """Stack G into an array ``[..., i, j] = G_ij`` (``tensorat``, src/closures.jl:6-11)."""
    names = "xyz"[:D]
    return np.stack([np.stack([G[names[i] + names[j]] for j in range(D)], -1) for i in range(D)], -2)


def store_sym(tau_mat, D):
    """``store_symtensor!`` (src/closures.jl:14-28): packed upper triangle."""
    return np.stack([tau_mat[..., i, j] for (i, j) in pairs(D)], 0)


def clark(G, delta, D):
    """``clark_kernel!`` (src/closures.jl:37-42): τ = Δ²/12 · G Gᵀ."""
    A = grad_matrix(G, D)
    tau = delta ** 2 / 12 * np.einsum("...ik,...jk->...ij", A, A)
    return store_sym(tau, D)


def smagorinsky(G, CS, delta, D):
    """``smagorinsky_kernel!`` (src/closures.jl:44-51): τ = -2 C_s²Δ² √(2 S:S) S."""
    A = grad_matrix(G, D)
    S = (A + np.swapaxes(A, -1, -2)) / 2
    nu = CS ** 2 * delta ** 2 * np.sqrt(2 * np.sum(S * S, axis=(-1, -2)))
    return store_sym(-2 * nu[..., None, None] * S, D)


def verstappen(G, C, delta, D):
    """``verstappen_kernel!`` (src/closures.jl:53-62); 3D only (``create_verstappen`` asserts)."""
    if D != 3:
        raise AssertionError("Q-R model is only defined in 3D")
    A = grad_matrix(G, D)
    S = (A + np.swapaxes(A, -1, -2)) / 2
    SS = S @ S
    q = np.trace(SS, axis1=-2, axis2=-1) / 2
    r = np.trace(SS @ S, axis1=-2, axis2=-1) / 3
    nu = C ** 2 * delta ** 2 * np.abs(r) / q
    return store_sym(-2 * nu[..., None, None] * S, D)


def test_filter_phys(phys, delta, g: Grid):
    """``test_filter_phys!`` (src/solver.jl:226-232): r2c, Gaussian(Δ), 2/3 rule, normalised c2r."""
    spec = sfft.rfftn(phys, workers=WORKERS)
    spec = twothirds(gaussianfilter(spec, delta, g), g)
    return sfft.irfftn(spec, s=g.phys_shape, workers=WORKERS)


def _dealias_phys(phys, g):
    spec = sfft.rfftn(phys, workers=WORKERS)
    return sfft.irfftn(twothirds(spec, g), s=g.phys_shape, workers=WORKERS)


def bardina(u, s, delta, g: Grid):
    """``create_bardina`` model (src/closures.jl:81-115): scale similarity with test width sΔ, trace-free."""
    dt_ = s * delta
    ut = [twothirds(gaussianfilter(c, dt_, g), g) for c in u]
    sig = nonlinearity(u, g)
    sigt = nonlinearity(ut, g)
    sig = [twothirds(gaussianfilter(c, dt_, g), g) for c in sig]
    tau = [to_phys(a, g) - to_phys(b, g) for a, b in zip(sig, sigt)]
    return np.stack(make_tracefree(tau, g.D), 0)


def smagorinsky_tensor(S, delta, D):
    """``smagorinsky_tensor!`` (src/closures.jl:117-150) with C_s = 1; S packed list."""
    S2 = sum(S[i] ** 2 for i in range(D)) + 2 * sum(S[i] ** 2 for i in range(D, len(S)))
    nu = delta ** 2 * np.sqrt(2 * S2)
    return [-2 * nu * c for c in S]


def smagorinsky_ml_mm(M, L, D):
    """``smagorinsky_ml_mm!`` (src/closures.jl:152-179): pointwise M:L (L made trace-free) and M:M."""
    L = list(L)
    tr = sum(L[i] for i in range(D)) / D
    for i in range(D):
        L[i] = L[i] - tr
    ml = sum(M[i] * L[i] for i in range(D)) + 2 * sum(M[i] * L[i] for i in range(D, len(M)))
    mm = sum(M[i] * M[i] for i in range(D)) + 2 * sum(M[i] * M[i] for i in range(D, len(M)))
    return ml, mm


def dynsmag_coefficient(sum_ml, sum_mm):
    """Global Lilly coefficient with the ⟨MM⟩ = 0 guard (src/closures.jl:260-262)."""
    if sum_mm == 0:
        return 0.0
    return max(-sum_ml / sum_mm, 0.0)


def dynamic_smagorinsky(u, delta, g: Grid, return_coeff=False):
    """``create_dynamic_smagorinsky`` model (src/closures.jl:188-272).

    Test filter Gaussian(2Δ)∘P, combined width √((2Δ)² + Δ²); c = max(-ΣML/ΣMM, 0)
    (0 when ΣMM = 0); τ = c · P(m1), not trace-free.
    """
    D = g.D
    dtl = 2 * delta
    ddb = math.sqrt(dtl ** 2 + delta ** 2)
    ut = [twothirds(gaussianfilter(c, dtl, g), g) for c in u]
    sig = nonlinearity(u, g)
    sigt = nonlinearity(ut, g)
    sig = [twothirds(gaussianfilter(c, dtl, g), g) for c in sig]
    L = [to_phys(a, g) - to_phys(b, g) for a, b in zip(sig, sigt)]
    Shat = strainrate(u, g)
    S, St = [], []
    for c in Shat:
        c = twothirds(c, g)
        S.append(to_phys(c, g))
        c = twothirds(gaussianfilter(c, dtl, g), g)
        St.append(to_phys(c, g))
    m1 = smagorinsky_tensor(S, delta, D)
    m2 = smagorinsky_tensor(St, ddb, D)
    m1 = [_dealias_phys(c, g) for c in m1]
    M = [test_filter_phys(c, dtl, g) - b for c, b in zip(m1, m2)]
    ml, mm = smagorinsky_ml_mm(M, L, D)
    c = dynsmag_coefficient(float(ml.sum()), float(mm.sum()))
    tau = np.stack([c * a for a in m1], 0)
    if return_coeff:
        return tau, c
    return tau


def mlp_fullchain(G, delta, visc, weights, biases, D, use_redelta=False, mu=0.0, sigma=1.0, eps=np.finfo(np.float64).eps):
    """``fullchain(setup, mlp(...), ...)`` (src/nets.jl:311-331 wrapping
    src/nets.jl:248-296): a pointwise MLP on the normalised velocity gradient.

    ``G``: dict of physical VGT components ('xy' = d_y u_x).  Input channels are
    G stacked with the first index fastest (xx, yx, zx, xy, ...), divided by
    (|G| + eps) pointwise; with ``use_redelta`` the standardised
    log Re_Delta = (log(Delta^2 sqrt(mean |G|^2) / visc) - mu) / sigma is
    appended (``append_redelta``, src/data.jl:689-695).  Layers
    (``PointwiseConv``, src/nets.jl:37-80): y = act(W^T x + b) with W of shape
    (c_in, c_out); GELU (NNlib, tanh form) on every layer but the last, which
    has no bias; the output's trace is removed and it is scaled by Delta^2 |G|^2.
    ``weights[l]``: array (c_out, c_in); ``biases[l]``: (c_out,) or None."""
    from .cnn import gelu
    names = "xyz"[:D]
    x = np.stack([G[names[a] + names[b]] for b in range(D) for a in range(D)], 0)
    A2 = np.sum(x * x, axis=0)
    x = x / (np.sqrt(A2) + eps)
    if use_redelta:
        re = delta ** 2 * np.sqrt(np.mean(A2)) / visc
        z = (np.log(re) - mu) / sigma
        x = np.concatenate([x, np.full((1,) + A2.shape, z)], 0)
    nl = len(weights)
    for l, W in enumerate(weights):
        y = np.einsum("oc,c...->o...", np.asarray(W, dtype=np.float64), x)
        if biases[l] is not None:
            y = y + np.asarray(biases[l], dtype=np.float64).reshape((-1,) + (1,) * A2.ndim)
        x = gelu(y) if l < nl - 1 else y
    if D == 3:
        t = (x[0] + x[1] + x[2]) / 3
        x = np.stack([x[0] - t, x[1] - t, x[2] - t, x[3], x[4], x[5]], 0)
    else:
        t = (x[0] + x[1]) / 2
        x = np.stack([x[0] - t, x[1] - t, x[2]], 0)
    return x * (delta ** 2 * A2)


def _dev(M, D):
    tr = np.trace(M, axis1=-2, axis2=-1)[..., None, None]
    return M - tr / D * np.eye(D)


def tbnn(G, delta, visc, weights, biases, D, use_redelta=False, mu=0.0, sigma=1.0, eps=np.finfo(np.float64).eps):
    """``tbnn(net, ps, st, Delta, g; use_redelta, redelta_norm, visc)``
    (src/nets.jl:560-588) with ``build_tensorbasis`` / ``tb_kernel!``
    (src/nets.jl:393-505): A = grad u normalised by (|A| + eps), S and R its
    symmetric and antisymmetric parts; invariants tr(SS), tr(RR) [, tr(SSS),
    tr(SRR), tr(SSRR)] (+ the standardised log Re_Delta) feed a pointwise MLP
    (GELU, bias-free last layer) whose outputs weight the deviatoric basis
    dev(S), dev(SR - RS) (2D) or dev(S), dev(SS), dev(RR), dev(SR - RS), dev(RSR),
    dev(RSS - SSR), dev(RSRR - RRSR) (3D); tau = sum * Delta^2 |A|^2, packed."""
    from .cnn import gelu
    names = "xyz"[:D]
    A = np.stack([np.stack([G[names[a] + names[b]] for b in range(D)], -1) for a in range(D)], -2)
    A2 = np.sum(A * A, axis=(-1, -2))
    A = A / (np.sqrt(A2) + eps)[..., None, None]
    S = (A + np.swapaxes(A, -1, -2)) / 2
    R = (A - np.swapaxes(A, -1, -2)) / 2
    mm = lambda *Ms: __import__("functools").reduce(lambda x, y: x @ y, Ms)  # noqa: E731
    tr = lambda M: np.trace(M, axis1=-2, axis2=-1)  # noqa: E731
    if D == 2:
        inv = [tr(mm(S, S)), tr(mm(R, R))]
        basis = [_dev(S, D), _dev(mm(S, R) - mm(R, S), D)]
    else:
        inv = [tr(mm(S, S)), tr(mm(R, R)), tr(mm(S, S, S)), tr(mm(S, R, R)), tr(mm(S, S, R, R))]
        basis = [_dev(S, D), _dev(mm(S, S), D), _dev(mm(R, R), D), _dev(mm(S, R) - mm(R, S), D),
                 _dev(mm(R, S, R), D), _dev(mm(R, S, S) - mm(S, S, R), D),
                 _dev(mm(R, S, R, R) - mm(R, R, S, R), D)]
    x = np.stack(inv, 0)
    if use_redelta:
        re = delta ** 2 * np.sqrt(np.mean(A2)) / visc
        x = np.concatenate([x, np.full((1,) + A2.shape, (np.log(re) - mu) / sigma)], 0)
    nl = len(weights)
    for l, W in enumerate(weights):
        y = np.einsum("oc,c...->o...", np.asarray(W, dtype=np.float64), x)
        if biases[l] is not None:
            y = y + np.asarray(biases[l], dtype=np.float64).reshape((-1,) + (1,) * A2.ndim)
        x = gelu(y) if l < nl - 1 else y
    M = sum(x[k][..., None, None] * basis[k] for k in range(len(basis)))
    return np.stack([M[..., i, j] for (i, j) in pairs(D)], 0) * (delta ** 2 * A2)

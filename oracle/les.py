"""LES right-hand side with a closure: FP64 restatement of ``les!`` (``src/les.jl:4-33``).

Test infrastructure only (see ``oracle/__init__.py``).
"""

from __future__ import annotations

import numpy as np

from .spectral import (Grid, get_dissipation, getenergy, k2_int, make_tracefree, pairs, spectrum, stress,
                       tensordivergence, to_phys, to_spec, twothirds, vectorgradient)

__all__ = ["physical_gradient", "les_rhs", "strain_from_gradient", "contract_dissipation", "les_aposteriori"]


def physical_gradient(u, g: Grid):
    """Physical VGT as in ``les!`` (src/les.jl:12-16): to_phys(twothirds(i k_b u_a))."""
    G = vectorgradient(u, g)
    return {k: to_phys(twothirds(v, g), g) for k, v in G.items()}


def les_rhs(u, g: Grid, model, visc):
    """``les!`` (src/les.jl:4-33): du = div(stress(u) + F[model(u, G)]).

    ``model(u, G)`` returns the packed physical stress ``(tensordim, *phys)``.
    ``model=None`` gives ``convectiondiffusion!``.
    """
    sig = stress(u, visc, g)
    if model is not None:
        GG = physical_gradient(u, g)
        y = model(u, GG)
        sig = [s + to_spec(y[i], g) for i, s in enumerate(sig)]
    return tensordivergence(sig, g)


def strain_from_gradient(G, D):
    """``strain_from_gradient`` (src/solver.jl:742-750), packed in pair order."""
    names = "xyz"[:D]
    return [G[names[i] + names[i]] if i == j else (G[names[i] + names[j]] + G[names[j] + names[i]]) / 2
            for (i, j) in pairs(D)]


def contract_dissipation(tau, S, D):
    """``contract_dissipation`` (src/solver.jl:753-759): tau : S, off-diagonals twice."""
    return sum((1.0 if i == j else 2.0) * tau[m] * S[m] for m, (i, j) in enumerate(pairs(D)))


def les_aposteriori(u, uref, g: Grid, model, visc, nshell=None):
    """The a-posteriori reductions of one LES state in ``solve_les!`` (``reduce!``,
    src/les.jl:94-148): e_post against the 2/3-truncated reference snapshot,
    kinetic energy, viscous dissipation, spectrum, SFS dissipation
    eps_sfs = -mean(tau_dev : S) with the closure re-evaluated on ``u``, and the
    shell-resolved transfer sum_shell Re(conj(u) . clo), clo_i = -i k_j tau_dev_ij
    (twothirds applied), summed over the shell's RFFT indices plus the conjugate
    interior (``getshells``, src/solver.jl:1080-1129).  ``model=None`` is ``:nomo``."""
    D = g.D
    nshell = nshell or g.n // 3
    out = {}
    if uref is not None:
        ur = [twothirds(c, g) for c in uref]
        num = np.sqrt(sum(float(np.sum(np.abs(a - b) ** 2)) for a, b in zip(u, ur)))
        den = np.sqrt(sum(float(np.sum(np.abs(b) ** 2)) for b in ur))
        out["e_post"] = num / den
    out["ke"] = sum(getenergy(c) for c in u) / 2
    out["eps_visc"] = get_dissipation(u, visc, g)
    out["spectrum"] = spectrum(u, g, nshell)
    if model is None:
        out["eps_sfs"] = 0.0
        out["transfer"] = [0.0] * nshell
        return out
    AA = physical_gradient(u, g)
    S = strain_from_gradient(AA, D)
    tau = make_tracefree(list(model(u, AA)), D)
    out["eps_sfs"] = -float(np.mean(contract_dissipation(tau, S, D)))
    ts = [twothirds(to_spec(t, g), g) for t in tau]
    clo = tensordivergence(ts, g)
    tloc = np.real(sum(np.conj(a) * b for a, b in zip(u, clo)))
    K = g.n // 2 + 1
    w = np.ones(g.spec_shape)
    w[..., 1:K - 1] = 2.0
    k2 = k2_int(g)
    out["transfer"] = [float((tloc * w)[(k2 >= i * i) & (k2 < (i + 1) * (i + 1))].sum()) for i in range(1, nshell + 1)]
    return out

"""LES right-hand side with a closure: FP64 restatement of ``les!`` (``src/les.jl:4-33``).

Test infrastructure only (see ``oracle/__init__.py``).
"""

from __future__ import annotations

from .spectral import (Grid, stress, tensordivergence, to_phys, to_spec, twothirds,
                       vectorgradient)

__all__ = ["physical_gradient", "les_rhs"]


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

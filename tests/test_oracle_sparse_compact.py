"""The two FP64 oracles used at 810^3 against the reference-following FFT oracle (CPU).

``oracle.triad`` (exact triad sums of a sparse field, with the n-point grid's
aliasing) and ``oracle.compact`` (the FFT oracle on the compact 2/3 cube) must
reproduce ``oracle.spectral`` / ``oracle.filtering`` -- the line-by-line
restatement of src/solver.jl, src/filtering.jl and src/data.jl -- at sizes the
full-layout oracle finishes in a second, including the cube's edge modes where
the products alias (p_i = q_i = n/3).
"""

import numpy as np
import pytest

import oracle as O
from oracle import triad as T
from oracle.compact import CompactOracle


def _edges(n):
    kc = n // 3
    return [(kc, kc, kc), (kc, -kc, 3), (0, kc, -kc), (0, 1, 0), (1, 1, 1), (0, 0, 1), (kc, 0, 0), (2, -kc, kc)]


def _scatter(kout, vals, g):
    out = [np.zeros(g.spec_shape, dtype=np.complex128) for _ in range(vals.shape[1])]
    iz, iy, ix = T.to_rfft_index(kout, g.n)
    for c in range(vals.shape[1]):
        out[c][iz, iy, ix] = vals[:, c]
    return out


@pytest.mark.parametrize("n", [24, 30, 36])
def test_triad_matches_fft_oracle(n):
    k, u = T.random_sparse_field(n, 60, 5, extra=_edges(n))
    g = O.Grid(3, n)
    dense = T.dense_rfft(k, u, n)
    ref = [O.twothirds(c, g) for c in O.convectiondiffusion(dense, g, 2e-3)]
    ko, du = T.convectiondiffusion(k, u, n, 2e-3)
    assert O.rel_l2(_scatter(ko, du, g), ref) < 1e-13
    ko, du = T.rk4_rhs(k, u, n, 2e-3, 0.1)
    assert O.rel_l2(_scatter(ko, du, g), O.rk4_rhs(dense, g, 2e-3, 0.1)) < 1e-13
    gl = O.Grid(3, 12)
    for d in (None, 0.9):
        ub, ta = O.sfs(dense, g, gl, d)
        ko, ubar, tau = T.sfs(k, u, n, 12, d)
        assert O.rel_l2(_scatter(ko, ubar, gl), ub) < 1e-13
        assert O.rel_l2(_scatter(ko, tau, gl), ta) < 1e-13


def test_triad_field_is_hermitian_and_solenoidal():
    k, u = T.random_sparse_field(30, 40, 9, extra=_edges(30))
    g = O.Grid(3, 30)
    dense = T.dense_rfft(k, u, 30)
    assert np.abs(O.vectordivergence(dense, g)).max() < 1e-12
    np.testing.assert_allclose(O.symmetrize(dense[0], g), dense[0], atol=1e-15)


@pytest.mark.parametrize("n", [30, 48])
def test_compact_matches_fft_oracle(n):
    g = O.Grid(3, n)
    uc = O.random_field_compact(3, n, 3)
    full = [O.unpack_retained(c, g) for c in uc]
    o = CompactOracle(n, workers=4)
    r1 = o.convectiondiffusion(uc, 2e-3)
    ref = [O.twothirds(c, g) for c in O.convectiondiffusion(full, g, 2e-3)]
    assert O.rel_l2([O.unpack_retained(c, g) for c in r1], ref) < 1e-14
    a = o.rk4_step(uc, 1e-2, 2e-3, 0.1)
    b = O.rk4_step(full, 1e-2, g, 2e-3, 0.1)
    assert O.rel_l2([O.unpack_retained(c, g) for c in a], b) < 1e-14
    gl = O.Grid(3, 16)
    for d in (None, 2 * 2 * np.pi / 16):
        ((ub, ta, scale),) = o.sfs(uc, 16, [d])
        ub2, ta2 = O.sfs(full, g, gl, d)
        assert O.rel_l2(ub, ub2) < 1e-14 and O.rel_l2(ta, ta2) < 1e-13
        assert scale > 0

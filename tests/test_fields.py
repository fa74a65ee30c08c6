"""The host-side initial-condition generator (symcode.fields, the reference's
``randomfield``) against the oracle's restatement: the same seed gives the
same coefficients, and the field is solenoidal with the prescribed shell energies."""

import numpy as np
import pytest

import oracle as O
from symcode import fields as F


@pytest.mark.parametrize("D,n,seed", [(3, 24, 0), (3, 48, 7), (2, 96, 3), (2, 64, 11)])
def test_random_field_matches_oracle(D, n, seed):
    a = F.random_field_compact(D, n, seed, kpeak=4.0)
    b = O.random_field_compact(D, n, seed, kpeak=4.0)
    for x, y in zip(a, b):
        assert x.shape == y.shape
        np.testing.assert_allclose(x, y, rtol=0, atol=1e-15 * np.abs(y).max())
    g = O.Grid(D, n)
    for x, y in zip(a, O.random_field(g, seed, kpeak=4.0)):
        np.testing.assert_allclose(F.compact_to_full(x, n), y, rtol=0, atol=1e-15 * np.abs(y).max())


def test_random_field_is_solenoidal_with_unit_energy():
    n = 48
    u = F.random_field_compact(3, n, 5, kpeak=4.0, totalenergy=1.0)
    full = [F.compact_to_full(c, n) for c in u]
    assert abs(O.energy(full) - 1.0) < 1e-12
    k = n // 3
    s = np.where(np.arange(2 * k + 1) <= k, np.arange(2 * k + 1), np.arange(2 * k + 1) - (2 * k + 1))
    kx = np.arange(k + 1)
    div = kx[None, None, :] * u[0] + s[None, :, None] * u[1] + s[:, None, None] * u[2]
    assert np.abs(div).max() < 1e-12 * max(np.abs(c).max() for c in u)

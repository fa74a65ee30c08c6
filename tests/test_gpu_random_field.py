"""randomfield (src/solver.jl:576-641) on the device (sc_random_field).

With the caller's draws (numpy PCG64, the generator of symcode.fields) the
device construction equals the host restatement (and so the oracle's) to FP64
roundoff; with the device's own counter-based draws the field has the
reference's properties: Hermitian kx = 0 plane, solenoidal, zero mean, every
retained shell at exactly its target energy, total energy as requested.
"""

import math

import numpy as np
import pytest
import torch

import oracle as O
import symcode as S
from symcode import fields
from _util import to_np

pytestmark = pytest.mark.gpu


def _draws(D, n, seed):
    """The host generator's coefficients (symcode.fields.random_field_compact's first step)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    shape = fields.compact_shape(D, n)
    out = []
    for _ in range(D):
        re = rng.standard_normal(shape)
        im = rng.standard_normal(shape)
        out.append((re + 1j * im) * math.sqrt(0.5))
    return out


@pytest.mark.parametrize("D,n,dtype,tol", [(3, 48, torch.float64, 1e-13), (2, 96, torch.float64, 1e-13),
                                           (3, 64, torch.float32, 2e-7)])
def test_device_random_field_equals_host_construction(D, n, dtype, tol):
    g = S.Grid(D, n, dtype=dtype, device="cuda:0")
    draws = [torch.from_numpy(c).cuda(0) for c in _draws(D, n, 7)]
    u = S.random_field(g, kpeak=4.0, totalenergy=1.0, draws=draws)
    ref = [fields.compact_to_full(c, n) for c in fields.random_field_compact(D, n, 7, kpeak=4.0, totalenergy=1.0)]
    assert O.rel_l2([to_np(c) for c in u], ref) < tol
    # the plan's state holds it too
    st = S.State(g)
    assert math.isclose(st.energy(), 1.0, rel_tol=1e-6 if dtype == torch.float32 else 1e-12)
    g.close()


@pytest.mark.parametrize("D,n", [(3, 64), (2, 128)])
def test_device_generator_field_has_the_reference_properties(D, n):
    g, go = S.Grid(D, n, dtype=torch.float64, device="cuda:0"), O.Grid(D, n)
    u = [to_np(c) for c in S.random_field(g, seed=11, kpeak=3.0, totalenergy=0.2)]
    u2 = [to_np(c) for c in S.random_field(g, seed=11, kpeak=3.0, totalenergy=0.2)]
    # deterministic per seed (the draws are; the shell sums are FP64 atomics, so
    # the rescale may differ in the last bit)
    assert O.rel_l2(u2, u) < 1e-14
    u3 = [to_np(c) for c in S.random_field(g, seed=12, kpeak=3.0, totalenergy=0.2)]
    assert O.rel_l2(u3, u) > 0.5  # another seed, another field
    assert np.abs(O.vectordivergence(u, go)).max() < 1e-12
    for c in u:
        np.testing.assert_allclose(O.symmetrize(c, go), c, atol=1e-15)
        assert c.flat[0] == 0
    np.testing.assert_array_equal(O.twothirds(u[0], go), u[0])
    assert math.isclose(O.energy(u), 0.2, rel_tol=1e-12)
    # every retained shell at its target: totalenergy * prof(s) / sum prof
    smax = int(math.floor(math.sqrt(D) * (n // 2)))
    prof = np.array([O.peak_profile(k, 3.0) for k in range(smax + 1)])
    spec = O.spectrum(u, go, nshell=n // 3)
    target = 0.2 * prof / prof.sum()
    np.testing.assert_allclose(spec, target[1:n // 3 + 1], rtol=1e-10)
    g.close()

"""Property checks of the oracle for the parts the reference's tests do not pin
(RHS values, steppers, forcing, filter, dynamic Smagorinsky)."""

import math

import numpy as np
import pytest

import oracle as O


def _wsum(a, b, g):
    """Re Σ_k w(k) conj(a)·b with the RFFT double count (interior kx twice)."""
    K = g.n // 2 + 1
    w = np.ones(g.spec_shape)
    w[..., 1:K - 1] = 2.0
    return float(sum(np.sum(w * (np.conj(x) * y).real) for x, y in zip(a, b)))


@pytest.mark.parametrize("D,n", [(2, 32), (3, 16)])
def test_energy_budget_unforced(D, n):
    """Dealiased Galerkin NS: dE/dt = -ε exactly (n not divisible by 3: no edge aliasing)."""
    g = O.Grid(D, n)
    u = O.random_field(g, seed=5, kpeak=3)
    du = [O.twothirds(c, g) for c in O.convectiondiffusion(u, g, 0.01)]
    dEdt = _wsum(u, du, g)
    eps = O.get_dissipation(u, 0.01, g)
    assert abs(dEdt + eps) < 1e-12 * max(1.0, eps)


def test_stress_form_matches_advective_form():
    """-∂_j(u_i u_j) (reference stress form) equals -(u·∇)u on retained modes for div-free u."""
    g = O.Grid(3, 16)
    u = O.random_field(g, seed=6, kpeak=3)
    du = [O.twothirds(c, g) for c in O.convectiondiffusion(u, g, 0.0)]
    ks = O.wavenumbers_full(g)
    v = [O.to_phys(c, g) for c in u]
    adv = []
    for i in range(3):
        a = sum(v[j] * O.to_phys(1j * ks[j] * u[i], g) for j in range(3))
        adv.append(-O.twothirds(O.to_spec(a, g), g))
    assert O.rel_l2(du, adv) < 1e-12


def test_taylor_green_divergence_free_and_real():
    g = O.Grid(3, 16)
    u = O.taylorgreen(g)
    assert np.max(np.abs(O.vectordivergence(u, g))) < 1e-12
    assert math.isclose(O.energy(u), 1 / 8, rel_tol=1e-12)


def test_random_field_properties():
    g = O.Grid(3, 24)
    u = O.random_field(g, seed=1, kpeak=4, totalenergy=1.0)
    assert np.max(np.abs(O.vectordivergence(u, g))) < 1e-12
    for c in u:  # Hermitian on kx = 0, zero outside the 2/3 cube
        np.testing.assert_allclose(O.symmetrize(c, g), c, atol=1e-15)
        np.testing.assert_array_equal(O.twothirds(c, g), c)
    # all shells up to the 2/3 corner are populated, so E matches the profile sum
    kmax = g.n // 2
    kdiag = int(math.floor(math.sqrt(3) * kmax))
    prof = np.array([O.peak_profile(k, 4) for k in range(kdiag + 1)])
    populated = [k for k in range(kdiag + 1) if k <= math.sqrt(3) * g.kcut]
    assert math.isclose(O.energy(u), prof[populated].sum() / prof.sum(), rel_tol=1e-10)


def test_wray3_third_order():
    g = O.Grid(2, 32)
    u0 = O.random_field(g, seed=2, kpeak=3)
    visc = 0.01

    def run(dt, nsteps):
        u = u0
        for _ in range(nsteps):
            u = O.wray3(O.convectiondiffusion, u, dt, g, visc=visc)
        return [O.twothirds(c, g) for c in u]

    ref = run(0.0025, 16)
    e1 = O.rel_l2(run(0.02, 2), ref)
    e2 = O.rel_l2(run(0.01, 4), ref)
    assert 5.5 < e1 / e2 < 11  # ~2^3


def test_rk4_fourth_order_and_forcing_rate():
    g = O.Grid(3, 16)
    u0 = O.random_field(g, seed=3, kpeak=3)
    visc, eps = 0.01, 0.1

    def run(dt, nsteps):
        u = u0
        for _ in range(nsteps):
            u = O.rk4_step(u, dt, g, visc, eps)
        return u

    ref = run(0.0125, 8)
    e1 = O.rel_l2(run(0.1, 1), ref)
    e2 = O.rel_l2(run(0.05, 2), ref)
    assert 11 < e1 / e2 < 22  # ~2^4
    # the band forcing injects exactly ε
    A = O.linear_forcing_coeff(u0, g, eps)
    m = O.band_mask(g)
    f = [np.where(m, A * c, 0) for c in u0]
    assert math.isclose(_wsum(u0, f, g), eps, rel_tol=1e-12)


def test_sfs_identity_filter_vanishes():
    """Same grid and no Gaussian: ū = P u and τ = P[σ(Pu) - σ(ū)] = 0."""
    g = O.Grid(3, 16)
    u = O.random_field(g, seed=4, kpeak=3)
    ubar, tau = O.sfs(u, g, g, None)
    assert O.rel_l2(ubar, u) < 1e-15
    assert max(np.max(np.abs(t)) for t in tau) < 1e-15


def test_sfs_trace_free_and_truncated():
    gd, gl = O.Grid(3, 24), O.Grid(3, 12)
    u = O.random_field(gd, seed=7, kpeak=3)
    ubar, tau = O.sfs(u, gd, gl, 2 * gl.l / gl.n)
    assert np.max(np.abs(tau[0] + tau[1] + tau[2])) < 1e-15
    for c in ubar + tau:
        np.testing.assert_array_equal(O.twothirds(c, gl), c)


def test_dynsmag_nonnegative_coefficient():
    g = O.Grid(3, 16)
    u = O.random_field(g, seed=8, kpeak=3)
    tau, c = O.dynamic_smagorinsky(u, 2 * g.l / g.n, g, return_coeff=True)
    assert c >= 0 and np.isfinite(tau).all()
    assert tau.shape == (6,) + g.phys_shape

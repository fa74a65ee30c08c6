"""Parity of the CUDA path (through the C ABI) with the FP64 oracle.

Tolerances: FP64 path <= 1e-12 relative L2 against the oracle (FFT roundoff of
pocketfft vs our mixed-radix kernels); FP32 path <= 1e-5 relative L2 per RHS
call against the FP64 oracle.
"""

import math

import numpy as np
import pytest
import torch

import oracle as O
import symcode as S
from _util import rel_l2, to_dev, to_np

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5


def _grid(D, n, dtype, l=2 * math.pi):
    return S.Grid(D, n, l, dtype=dtype, device="cuda:0"), O.Grid(D, n, l)


def _hermitian_spec(go, seed):
    r = np.random.default_rng(seed)
    c = (r.standard_normal(go.spec_shape) + 1j * r.standard_normal(go.spec_shape)) * math.sqrt(0.5)
    return O.symmetrize(c, go)


# ---------------------------------------------------------------- FFT wrappers
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("D,n,l", [(2, 16, 2 * math.pi), (3, 8, 1.0)])
def test_fft_roundtrip_and_scaling(dtype, D, n, l):
    """test/test_fft.jl:5-24: to_spec -> to_phys is the identity; a constant 1.5 gives spec[1] = 1.5."""
    g, go = _grid(D, n, dtype, l)
    phys = np.random.default_rng(0).standard_normal(go.phys_shape)
    spec = S.scalarfield(g)
    out = S.spacescalarfield(g)
    S.to_spec_(spec, to_dev(phys, g), g)
    S.to_phys_(out, spec, g)
    tol = TOL64 if dtype == torch.float64 else 1e-6
    assert rel_l2(to_np(out), phys) < tol
    S.to_spec_(spec, torch.full(go.phys_shape, 1.5, dtype=dtype, device=g.device), g)
    assert abs(complex(spec.flatten()[0].item()) - 1.5) < tol


@pytest.mark.parametrize("D,n", [(3, 24), (3, 30), (3, 64), (2, 256), (3, 90)])
def test_fft_matches_pocketfft(D, n):
    g, go = _grid(D, n, torch.float64)
    spec = _hermitian_spec(go, 1)
    phys = S.spacescalarfield(g)
    S.to_phys_(phys, to_dev(spec, g), g)
    assert rel_l2(to_np(phys), O.to_phys(spec, go)) < TOL64
    x = np.random.default_rng(2).standard_normal(go.phys_shape)
    sp = S.scalarfield(g)
    S.to_spec_(sp, to_dev(x, g), g)
    assert rel_l2(to_np(sp), O.to_spec(x, go)) < TOL64


@pytest.mark.parametrize("D,n", [(3, 64), (3, 128), (2, 256), (2, 810)])
def test_fft_fp32_matches_pocketfft(D, n):
    g, go = _grid(D, n, torch.float32)
    spec = _hermitian_spec(go, 3)
    phys = S.spacescalarfield(g)
    S.to_phys_(phys, to_dev(spec, g), g)
    assert rel_l2(to_np(phys), O.to_phys(spec, go)) < 1e-6
    x = np.random.default_rng(4).standard_normal(go.phys_shape)
    sp = S.scalarfield(g)
    S.to_spec_(sp, to_dev(x, g), g)
    assert rel_l2(to_np(sp), O.to_spec(x, go)) < 1e-6


# ------------------------------------------------------------- point kernels
def test_twothirds_and_project():
    g, go = _grid(2, 24, torch.float64)
    u = np.random.default_rng(0).standard_normal(go.spec_shape) + 0j
    t = to_dev(u, g)
    S.twothirds_(t, g)
    np.testing.assert_array_equal(to_np(t), O.twothirds(u, go))
    g3, go3 = _grid(3, 8, torch.float64)
    r = np.random.default_rng(1)
    v = [r.standard_normal(go3.spec_shape) + 1j * r.standard_normal(go3.spec_shape) for _ in range(3)]
    tv = [to_dev(c, g3) for c in v]
    S.project_(tv, g3)
    assert rel_l2([to_np(c) for c in tv], O.project(v, go3)) < 1e-14
    div = O.vectordivergence([to_np(c) for c in tv], go3)
    assert np.max(np.abs(div)) < 1e-10  # test/test_solver_kernels.jl:19-29


# --------------------------------------------------------------------- RHS
def _rhs_case(D, n, dtype, seed=0, visc=2e-3, full_input=False):
    g, go = _grid(D, n, dtype)
    if full_input:
        r = np.random.default_rng(seed)
        u = [O.symmetrize((r.standard_normal(go.spec_shape) + 1j * r.standard_normal(go.spec_shape)) * 0.01, go)
             for _ in range(D)]
        u = O.project(u, go)
    else:
        u = O.random_field(go, seed=seed, kpeak=max(2, n // 16))
    ref = [O.twothirds(c, go) for c in O.convectiondiffusion(u, go, visc)]
    du = S.vectorfield(g)
    S.convectiondiffusion_(du, [to_dev(c, g) for c in u], g, visc)
    return rel_l2([to_np(c) for c in du], ref)


@pytest.mark.parametrize("D,n", [(2, 256), (2, 32), (3, 8), (3, 16), (3, 30), (3, 64)])
def test_rhs_fp64_matches_oracle(D, n):
    assert _rhs_case(D, n, torch.float64) < TOL64


@pytest.mark.parametrize("D,n", [(2, 256), (2, 810), (3, 16), (3, 64), (3, 128)])
def test_rhs_fp32_within_tolerance(D, n):
    assert _rhs_case(D, n, torch.float32) < TOL32


@pytest.mark.parametrize("D,n", [(2, 24), (3, 12)])
def test_rhs_untruncated_input(D, n):
    """Modes outside the 2/3 cube and the k = 0 mode of u never reach retained du."""
    assert _rhs_case(D, n, torch.float64, full_input=True) < TOL64


def test_rhs_ignores_mean_mode():
    g, go = _grid(3, 16, torch.float64)
    u = O.random_field(go, seed=3, kpeak=3)
    u[0][0, 0, 0] = 0.7  # a mean flow: masked out of the products by twothirds!
    ref = [O.twothirds(c, go) for c in O.convectiondiffusion(u, go, 1e-2)]
    du = S.vectorfield(g)
    S.convectiondiffusion_(du, [to_dev(c, g) for c in u], g, 1e-2)
    assert rel_l2([to_np(c) for c in du], ref) < TOL64


# ----------------------------------------------------------------- steppers
@pytest.mark.parametrize("D,n", [(2, 64), (3, 24)])
def test_wray3_matches_oracle(D, n):
    g, go = _grid(D, n, torch.float64)
    u = O.random_field(go, seed=4, kpeak=3)
    ref = O.wray3(O.convectiondiffusion, u, 0.01, go, visc=5e-3)
    ref = [O.twothirds(c, go) for c in ref]
    ut = [to_dev(c, g) for c in u]
    S.wray3_(ut, 0.01, g, 5e-3)
    assert rel_l2([to_np(c) for c in ut], ref) < TOL64


@pytest.mark.parametrize("dtype,tol", [(torch.float64, TOL64), (torch.float32, 2e-5)])
def test_rk4_forced_matches_oracle(dtype, tol):
    g, go = _grid(3, 24, dtype)
    u = O.random_field(go, seed=5, kpeak=3)
    ref = u
    for _ in range(2):
        ref = O.rk4_step(ref, 0.01, go, 5e-3, eps=0.1)
    ut = [to_dev(c, g) for c in u]
    S.rk4_(ut, 0.01, g, 5e-3, nsteps=2, eps=0.1)
    assert rel_l2([to_np(c) for c in ut], ref) < tol


def test_rk4_unforced_2d():
    g, go = _grid(2, 256, torch.float64)
    u = O.random_field(go, seed=0, kpeak=5)
    ref = u
    for _ in range(3):
        ref = O.rk4_step(ref, 1e-3, go, 5e-4)
    ut = [to_dev(c, g) for c in u]
    S.rk4_(ut, 1e-3, g, 5e-4, nsteps=3)
    assert rel_l2([to_np(c) for c in ut], ref) < TOL64


def test_config0_2d_decaying_200_steps():
    """The 2D decaying case: 256^2 FP64, nu = 5e-4, RK4 dt = 1e-3, 200 steps from
    the seeded k^4 exp(-2 (k/5)^2) field (seed 0), against the oracle on the same
    field; the tolerance allows 200 steps of round-off growth."""
    g, go = _grid(2, 256, torch.float64)
    u = O.random_field(go, seed=0, kpeak=5)
    ref = u
    for _ in range(200):
        ref = O.rk4_step(ref, 1e-3, go, 5e-4)
    ut = [to_dev(c, g) for c in u]
    S.rk4_(ut, 1e-3, g, 5e-4, nsteps=200)
    assert rel_l2([to_np(c) for c in ut], ref) < 1e-11
    assert math.isclose(S.energy(ut, g), O.energy(ref), rel_tol=1e-12)


# -------------------------------------------------------------- diagnostics
def test_energy_and_dissipation():
    g, go = _grid(3, 32, torch.float64)
    u = O.random_field(go, seed=6, kpeak=4, totalenergy=1.0)
    r = np.random.default_rng(9)
    u[0] = u[0] + 0.01 * O.symmetrize(r.standard_normal(go.spec_shape) + 0j, go)  # populate Nyquist planes
    ut = [to_dev(c, g) for c in u]
    assert math.isclose(S.energy(ut, g), O.energy(u), rel_tol=1e-12)
    assert math.isclose(S.get_dissipation(ut, 1e-3, g), O.get_dissipation(u, 1e-3, go), rel_tol=1e-12)

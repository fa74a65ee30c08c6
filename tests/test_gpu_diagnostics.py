"""CFL step, shell-energy clamp, spectrum and statistics through the C ABI vs the oracle."""

import math

import numpy as np
import pytest
import torch

import oracle as O
import symcode as S
from _util import rel_l2, to_dev, to_np

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("D,n,dtype,tol", [(3, 32, torch.float64, 1e-12), (2, 64, torch.float64, 1e-12),
                                           (3, 64, torch.float32, 1e-6)])
def test_propose_timestep(D, n, dtype, tol):
    g, go = S.Grid(D, n, dtype=dtype, device="cuda:0"), O.Grid(D, n)
    u = O.random_field(go, seed=50, kpeak=3)
    for visc in (1e-3, 10.0):  # convective and diffusive limit
        dt = S.propose_timestep([to_dev(c, g) for c in u], g, visc)
        assert math.isclose(dt, O.propose_timestep(u, go, visc), rel_tol=tol)


def test_shell_clamp_matches_oracle():
    g, go = S.Grid(3, 32, dtype=torch.float64, device="cuda:0"), O.Grid(3, 32)
    u0 = O.random_field(go, seed=51, kpeak=3)
    u1 = O.random_field(go, seed=52, kpeak=3)
    shells = O.energy_shells(go, [1, 2], u0)
    eref = S.energy_shells(g, [to_dev(c, g) for c in u0])
    assert np.allclose(eref, [s[2] for s in shells], rtol=1e-13)
    ut = [to_dev(c, g) for c in u1]
    S.maintain_shell_energy_(ut, eref, g)
    ref = O.maintain_shell_energy(u1, shells)
    assert rel_l2([to_np(c) for c in ut], ref) < 1e-13


def test_spectrum_and_statistics():
    g, go = S.Grid(3, 48, dtype=torch.float64, device="cuda:0"), O.Grid(3, 48)
    u = O.random_field(go, seed=53, kpeak=4)
    ut = [to_dev(c, g) for c in u]
    s = S.spectrum(ut, g)
    assert np.allclose(s, O.spectrum(u, go), rtol=1e-12, atol=1e-16)
    st = S.turbulence_statistics(ut, 1e-3, g)
    ref = O.turbulence_statistics(u, 1e-3, go)
    for k in ("e", "diss", "l_kol", "Re_tay"):
        assert math.isclose(st[k], ref[k], rel_tol=1e-12)


def test_wray3_with_shell_clamp_is_the_reference_dns_loop():
    """create_dns inner loop (src/data.jl:60-78): CFL dt, wray3!, maintain_shell_energy!."""
    g, go = S.Grid(3, 24, dtype=torch.float64, device="cuda:0"), O.Grid(3, 24)
    u = O.random_field(go, seed=54, kpeak=3)
    shells = O.energy_shells(go, [1, 2], u)
    ut = [to_dev(c, g) for c in u]
    eref = S.energy_shells(g, ut)
    ref = u
    for _ in range(2):
        dt = 0.35 * O.propose_timestep(ref, go, 2e-3)
        ref = O.wray3(O.convectiondiffusion, ref, dt, go, visc=2e-3)
        ref = O.maintain_shell_energy(ref, shells)
        dtg = 0.35 * S.propose_timestep(ut, g, 2e-3)
        assert math.isclose(dt, dtg, rel_tol=1e-11)
        S.wray3_(ut, dtg, g, 2e-3)
        S.maintain_shell_energy_(ut, eref, g)
    assert rel_l2([to_np(c) for c in ut], [O.twothirds(c, go) for c in ref]) < 1e-11

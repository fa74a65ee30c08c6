"""Tensor-core CNN closure (tcgen05, BF16 x BF16 -> FP32) against the FP64
oracle with BF16 rounding emulated, on sampled output rows of a 128^3 field.

Tolerance: 5e-3 relative L2 -- accumulation order (FP32 on the tensor cores vs
FP64 in the oracle) occasionally moves a pre-activation across a BF16 rounding
boundary, a one-ulp (0.4 %) change of that activation.
"""

import math

import numpy as np
import pytest
import torch

import oracle as O
import symcode as S
from _util import rel_l2, to_dev, to_np

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    n = 128
    g = S.Grid(3, n, dtype=torch.float32, device="cuda:0")
    go = O.Grid(3, n)
    u = O.random_field(go, seed=40, kpeak=4)
    delta, nu = 4 * go.l / n, 3e-4
    ws, bs = S.kaiming_cnn_weights(7)
    bs = [b + 0.05 * np.arange(b.size, dtype=np.float32) for b in bs]  # exercise the bias path
    cl = S.create_cnn_closure(delta, nu, g, ws, bs, mu=1.0, sigma=2.0)
    return g, go, u, delta, nu, ws, bs, cl


def test_cnn_closure_matches_oracle(setup):
    g, go, u, delta, nu, ws, bs, cl = setup
    ut = [to_dev(c, g) for c in u]
    tau = to_np(cl(ut, None))
    uphys = np.stack([to_np(S.to_phys_(S.spacescalarfield(g), c, g)) for c in ut], 0)
    # the closure sees u through twothirds! (k = 0 removed); the field has no mean
    zval = O.cnn_redelta_channel(u, go, delta, nu, mu=1.0, sigma=2.0)
    rows = [(0, 0), (17, 5), (64, 127), (101, 63), (127, 90)]
    ref = O.cnn_rows(uphys, zval, ws, bs, rows)
    got = np.stack([tau[:, z, y, :] for (y, z) in rows], 1)
    assert np.isfinite(got).all()
    assert rel_l2(got, ref) < 5e-3
    st = torch.zeros(1)
    import ctypes as ct
    status = ct.c_int()
    S.lib().sc_closure_status(cl.ptr, ct.byref(status))
    assert status.value == 0


def test_les_rhs_with_cnn_adds_divergence_of_tau(setup):
    g, go, u, delta, nu, ws, bs, cl = setup
    ut = [to_dev(c, g) for c in u]
    du_c = S.vectorfield(g)
    du_0 = S.vectorfield(g)
    S.les_(du_c, ut, g, cl, nu)
    S.les_(du_0, ut, g, None, nu)
    tau = to_np(cl(ut, None))
    sig = [O.twothirds(O.to_spec(t, go), go) for t in tau]
    extra = O.tensordivergence(sig, go)
    diff = [to_np(a) - to_np(b) for a, b in zip(du_c, du_0)]
    assert rel_l2(diff, [O.twothirds(e, go) for e in extra]) < 1e-4


def test_cnn_closure_64_matches_oracle():
    """n = 64: M = 128 tiles of which rows 0..63 are the x-row."""
    n = 64
    g, go = S.Grid(3, n, dtype=torch.float32, device="cuda:0"), O.Grid(3, n)
    u = O.random_field(go, seed=41, kpeak=3)
    delta, nu = 4 * go.l / n, 1e-3
    ws, bs = S.kaiming_cnn_weights(8)
    bs = [b + 0.05 * np.arange(b.size, dtype=np.float32) for b in bs]
    cl = S.create_cnn_closure(delta, nu, g, ws, bs, mu=1.0, sigma=2.0)
    ut = [to_dev(c, g) for c in u]
    tau = to_np(cl(ut, None))
    uphys = np.stack([to_np(S.to_phys_(S.spacescalarfield(g), c, g)) for c in ut], 0)
    zval = O.cnn_redelta_channel(u, go, delta, nu, mu=1.0, sigma=2.0)
    rows = [(0, 0), (17, 5), (63, 63), (31, 40)]
    ref = O.cnn_rows(uphys, zval, ws, bs, rows)
    got = np.stack([tau[:, z, y, :] for (y, z) in rows], 1)
    assert np.isfinite(got).all()
    assert rel_l2(got, ref) < 5e-3
    # the parameter vector round-trips: setting the same weights gives the same stress
    S.closure_set_params(cl, S.pack_cnn_params(ws, bs))
    assert rel_l2(to_np(cl(ut, None)), tau) < 1e-7


@pytest.mark.parametrize("n,seed", [(128, 40), (64, 41)])
def test_cnn_closure_split_matches_unrounded_oracle(n, seed):
    """Split precision (SC_CLOPT_CNN_SPLIT): three tensor-core passes over
    FP16 hi/lo parts per convolution against the FP64 network without any
    rounding.  The parts carry 22 significant bits, so the bar is the FP32
    level, not the BF16 one (measured on a B200: 2.1e-6 at n = 128, 2.7e-6 at
    n = 64)."""
    g, go = S.Grid(3, n, dtype=torch.float32, device="cuda:0"), O.Grid(3, n)
    u = O.random_field(go, seed=seed, kpeak=4)
    delta, nu = 4 * go.l / n, 3e-4
    ws, bs = S.kaiming_cnn_weights(7)
    bs = [b + 0.05 * np.arange(b.size, dtype=np.float32) for b in bs]
    cl = S.create_cnn_closure(delta, nu, g, ws, bs, mu=1.0, sigma=2.0, split=True)
    ut = [to_dev(c, g) for c in u]
    tau = to_np(cl(ut, None))
    uphys = np.stack([to_np(S.to_phys_(S.spacescalarfield(g), c, g)) for c in ut], 0)
    zval = O.cnn_redelta_channel(u, go, delta, nu, mu=1.0, sigma=2.0)
    rows = [(0, 0), (17, 5), (n - 1, n - 1), (n // 2 + 3, n // 3)]
    ref = O.cnn_rows(uphys, zval, ws, bs, rows, round_bf16=False)
    got = np.stack([tau[:, z, y, :] for (y, z) in rows], 1)
    err = rel_l2(got, ref)
    print(f"split precision n={n}: tau relative L2 vs unrounded FP64 {err:.2e}")
    assert np.isfinite(got).all()
    assert err < 1e-5
    # back to BF16: the one-pass result, BF16-level error again
    S.closure_set_option(cl, S.SC_CLOPT_CNN_SPLIT, 0)
    tau_bf = to_np(cl(ut, None))
    S.closure_set_option(cl, S.SC_CLOPT_CNN_SPLIT, 1)
    assert rel_l2(to_np(cl(ut, None)), tau) < 1e-7
    ref_bf = O.cnn_rows(uphys, zval, ws, bs, rows)
    assert rel_l2(np.stack([tau_bf[:, z, y, :] for (y, z) in rows], 1), ref_bf) < 5e-3
    import ctypes as ct
    status = ct.c_int()
    S.lib().sc_closure_status(cl.ptr, ct.byref(status))
    assert status.value == 0
    cl.close()
    g.close()


def test_closure_option_rejects_other_closures():
    g = S.Grid(3, 32, dtype=torch.float32, device="cuda:0")
    ws, bs = S.kaiming_cnn_weights(3)
    cl = S.create_cnn_fp_closure(4 * g.l / 32, 1e-3, g, ws, bs)
    with pytest.raises(S.SymcodeError):
        S.closure_set_option(cl, S.SC_CLOPT_CNN_SPLIT, 1)
    cl.close()
    g.close()


@pytest.mark.parametrize("target_scale", [1.3])
def test_tensor_core_adjoint_matches_fp64_gradient(target_scale):
    """The BF16 tensor-core adjoint (roundings taken as identities) against the
    FP64 CUDA-core adjoint of the same network on the same rollout.  The target
    closure has weights x target_scale, so the trajectory residual, which the
    gradient is proportional to, is large against the BF16 rounding of weights
    and activations (with a 1 % perturbation the two residuals, and hence the
    gradients, differ by tens of percent through the rounding alone)."""
    n, nsteps, ck, dt, nu = 64, 3, 2, 5e-3, 1e-3
    go = O.Grid(3, n)
    u0n = O.random_field(go, seed=42, kpeak=3)
    ws, bs = S.kaiming_cnn_weights(9)
    theta = S.pack_cnn_params(ws, bs)
    theta_t = theta * target_scale
    out = {}
    for kind, dtype in (("tc", torch.float32), ("fp64", torch.float64)):
        g = S.Grid(3, n, dtype=dtype, device="cuda:0")
        u0 = [to_dev(c, g) for c in u0n]
        make = S.create_cnn_closure if kind == "tc" else S.create_cnn_fp_closure
        cl = make(4 * go.l / n, nu, g, ws, bs, mu=5.0, sigma=2.0)
        S.closure_set_params(cl, theta_t)
        traj = S.rollout_record(g, cl, u0, dt, nu, nsteps)
        S.closure_set_params(cl, theta)
        out[kind] = S.rollout_adjoint(g, cl, u0, traj, dt, nu, nsteps, ckpt_every=ck)
    (l_tc, g_tc), (l_64, g_64) = out["tc"], out["fp64"]
    assert np.isfinite(g_tc).all()
    err = np.linalg.norm(g_tc - g_64) / np.linalg.norm(g_64)
    assert err < 5e-2, err
    assert abs(l_tc - l_64) <= 5e-2 * abs(l_64)

"""FP32/FP64 CUDA-core CNN closure and the hand-written adjoint of the LES
rollout (a-posteriori training).  The gradient is checked against central
finite differences in FP64 on random weight directions."""

import math

import numpy as np
import pytest
import torch

import oracle as O
import symcode as S
from _util import rel_l2, to_dev, to_np

pytestmark = pytest.mark.gpu


def _weights(seed, scale_last=1.0):
    ws, bs = S.kaiming_cnn_weights(seed)
    ws[3] = ws[3] * scale_last
    bs = [b + 0.01 * np.arange(b.size, dtype=np.float32) for b in bs]
    return ws, bs


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-11), (torch.float32, 2e-5)])
def test_cnn_fp_closure_matches_oracle(dtype, tol):
    n = 32
    g, go = S.Grid(3, n, dtype=dtype, device="cuda:0"), O.Grid(3, n)
    u = O.random_field(go, seed=60, kpeak=3)
    delta, nu = 4 * go.l / n, 1e-3
    ws, bs = _weights(8)
    cl = S.create_cnn_fp_closure(delta, nu, g, ws, bs, mu=2.0, sigma=1.5)
    ut = [to_dev(c, g) for c in u]
    tau = to_np(cl(ut, None))
    uphys = np.stack([O.to_phys(O.twothirds(c, go), go) for c in u], 0)
    zval = O.cnn_redelta_channel(u, go, delta, nu, mu=2.0, sigma=1.5)
    rows = [(y, z) for y in (0, 9, 31) for z in (0, 17)]
    ref = O.cnn_rows(uphys, zval, ws, bs, rows, round_bf16=False)
    got = np.stack([tau[:, z, y, :] for (y, z) in rows], 1)
    assert rel_l2(got, ref) < tol


def test_rollout_adjoint_matches_finite_differences():
    n, nsteps, ck, dt, nu = 16, 4, 2, 2e-3, 2e-3
    g, go = S.Grid(3, n, dtype=torch.float64, device="cuda:0"), O.Grid(3, n)
    u0 = [to_dev(c, g) for c in O.random_field(go, seed=61, kpeak=2)]
    delta = 4 * go.l / n
    ws, bs = _weights(9, scale_last=0.3)
    theta = S.pack_cnn_params(ws, bs)
    rng = np.random.default_rng(62)
    theta_t = theta * (1 + 0.01 * rng.standard_normal(theta.size))  # target: perturbed closure
    cl = S.create_cnn_fp_closure(delta, nu, g, ws, bs, mu=1.0, sigma=2.0)
    S.closure_set_params(cl, theta_t)
    traj = S.rollout_record(g, cl, u0, dt, nu, nsteps)
    S.closure_set_params(cl, theta)
    loss, grad = S.rollout_adjoint(g, cl, u0, traj, dt, nu, nsteps, ckpt_every=ck)
    assert loss > 0 and np.isfinite(grad).all() and np.abs(grad).max() > 0
    assert math.isclose(loss, S.rollout_loss(g, cl, u0, traj, dt, nu, nsteps), rel_tol=1e-12)
    for k in range(16):
        d = rng.standard_normal(theta.size)
        d /= np.linalg.norm(d)
        h = 1e-4 * np.linalg.norm(theta) / math.sqrt(theta.size)
        S.closure_set_params(cl, theta + h * d)
        lp = S.rollout_loss(g, cl, u0, traj, dt, nu, nsteps)
        S.closure_set_params(cl, theta - h * d)
        lm = S.rollout_loss(g, cl, u0, traj, dt, nu, nsteps)
        fd = (lp - lm) / (2 * h)
        ad = float(grad @ d)
        assert abs(fd - ad) <= 1e-6 * abs(ad) + 1e-14, (k, fd, ad)
    S.closure_set_params(cl, theta)


def test_rollout_adjoint_batch_matches_single_jobs():
    """Concurrent jobs (own plan, closure and stream each) give the single-job results."""
    n, nsteps, ck, dt = 16, 3, 2, 2e-3
    go = O.Grid(3, n)
    ws, bs = _weights(11, scale_last=0.3)
    theta = S.pack_cnn_params(ws, bs)
    jobs, ref = [], []
    for i, nu in enumerate((2e-3, 1e-3, 5e-4)):
        g = S.Grid(3, n, dtype=torch.float64, device="cuda:0")
        u0 = [to_dev(c, g) for c in O.random_field(go, seed=70 + i, kpeak=2)]
        cl = S.create_cnn_fp_closure(4 * go.l / n, nu, g, ws, bs, mu=1.0, sigma=2.0)
        S.closure_set_params(cl, theta * (1 + 0.01 * np.random.default_rng(80 + i).standard_normal(theta.size)))
        traj = S.rollout_record(g, cl, u0, dt, nu, nsteps)
        S.closure_set_params(cl, theta)
        ref.append(S.rollout_adjoint(g, cl, u0, traj, dt, nu, nsteps, ckpt_every=ck))
        jobs.append(dict(grid=g, closure=cl, u0=u0, traj=traj, dt=dt, visc=nu, nsteps=nsteps, ckpt_every=ck))
    for _ in range(2):
        got = S.rollout_adjoint_batch(jobs)
        for (l, gr), (lr, grr) in zip(got, ref):
            assert math.isclose(l, lr, rel_tol=1e-12)
            assert np.linalg.norm(gr - grr) <= 1e-12 * np.linalg.norm(grr)


def test_rollout_adjoint_batch_rejects_shared_plans():
    n = 16
    g = S.Grid(3, n, dtype=torch.float64, device="cuda:0")
    ws, bs = _weights(12)
    cl = S.create_cnn_fp_closure(4 * g.l / n, 1e-3, g, ws, bs)
    u0 = [to_dev(c, g) for c in O.random_field(O.Grid(3, n), seed=90, kpeak=2)]
    traj = S.rollout_record(g, cl, u0, 2e-3, 1e-3, 2)
    job = dict(grid=g, closure=cl, u0=u0, traj=traj, dt=2e-3, visc=1e-3, nsteps=2)
    with pytest.raises(S.SymcodeError):
        S.rollout_adjoint_batch([job, job])


# ---------------------------------------------------------------- the a-posteriori training configuration
# 64^3, 40 RK4 steps (dt = 5e-3), checkpoints every 5 steps, nu = 1e-3,
# Delta/h = 4, the CNN closure, target rollout of the closure with weights
# x (1 + 0.01 N(0, 1)).
T_N, T_STEPS, T_CK, T_DT, T_NU = 64, 40, 5, 5e-3, 1e-3


def _training_case(dtype, seed=101, split=False):
    g, go = S.Grid(3, T_N, dtype=dtype, device="cuda:0"), O.Grid(3, T_N)
    u0 = [to_dev(c, g) for c in O.random_field(go, seed=seed, kpeak=4)]
    ws, bs = S.kaiming_cnn_weights(5)
    theta = S.pack_cnn_params(ws, bs)
    if split:  # the tensor-core CNN in split precision
        cl = S.create_cnn_closure(4 * go.l / T_N, T_NU, g, ws, bs, mu=5.0, sigma=2.0, split=True)
    else:
        cl = S.create_cnn_fp_closure(4 * go.l / T_N, T_NU, g, ws, bs, mu=5.0, sigma=2.0)
    rng = np.random.default_rng(seed + 1)
    S.closure_set_params(cl, theta * (1 + 0.01 * rng.standard_normal(theta.size)))
    traj = S.rollout_record(g, cl, u0, T_DT, T_NU, T_STEPS)
    S.closure_set_params(cl, theta)
    return g, cl, u0, traj, theta


def test_training_adjoint_matches_finite_differences_at_64():
    """FP64 gradient by the adjoint (checkpoints every 5 of 40 steps) against
    central finite differences of the FP64 loss on 4 random weight directions."""
    g, cl, u0, traj, theta = _training_case(torch.float64)
    loss, grad = S.rollout_adjoint(g, cl, u0, traj, T_DT, T_NU, T_STEPS, ckpt_every=T_CK)
    rng = np.random.default_rng(103)
    h = 1e-4 * np.linalg.norm(theta) / math.sqrt(theta.size)
    for k in range(4):
        d = rng.standard_normal(theta.size)
        d /= np.linalg.norm(d)
        S.closure_set_params(cl, theta + h * d)
        lp = S.rollout_loss(g, cl, u0, traj, T_DT, T_NU, T_STEPS)
        S.closure_set_params(cl, theta - h * d)
        lm = S.rollout_loss(g, cl, u0, traj, T_DT, T_NU, T_STEPS)
        fd = (lp - lm) / (2 * h)
        ad = float(grad @ d)
        print(f"direction {k}: adjoint {ad:.10e}  central FD {fd:.10e}  rel {abs(fd - ad) / abs(ad):.2e}")
        assert abs(fd - ad) <= 1e-5 * abs(ad), (k, fd, ad)
    S.closure_set_params(cl, theta)
    cl.close()
    g.close()


def test_training_adjoint_fp32_matches_fp64():
    """The FP32 CUDA-core adjoint (the batched training path's precision) against
    the FP64 adjoint on the same initial field, target and weights."""
    res = {}
    for dtype in (torch.float64, torch.float32):
        g, cl, u0, traj, theta = _training_case(dtype)
        res[dtype] = S.rollout_adjoint(g, cl, u0, traj, T_DT, T_NU, T_STEPS, ckpt_every=T_CK)
        cl.close()
        g.close()
    (l64, g64), (l32, g32) = res[torch.float64], res[torch.float32]
    e_loss = abs(l32 - l64) / l64
    e_grad = float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64))
    print(f"FP32 vs FP64: loss {e_loss:.2e}, gradient {e_grad:.2e}")
    # measured: loss 5.3e-7, gradient 6.8e-6
    assert e_loss < 1e-5
    assert e_grad < 1e-4


def test_training_adjoint_split_tensor_cores_matches_fp64():
    """The tensor-core adjoint in split precision (FP16 hi/lo forward passes,
    BF16 hi/lo input-gradient passes, FP32 accumulation) at the training
    geometry against the FP64 CUDA-core adjoint: the configuration's 1 % weight
    perturbation, where the one-pass BF16 gradient is 0.16-0.22 off."""
    res = {}
    for dtype, split in ((torch.float64, False), (torch.float32, True)):
        g, cl, u0, traj, theta = _training_case(dtype, split=split)
        res[dtype] = S.rollout_adjoint(g, cl, u0, traj, T_DT, T_NU, T_STEPS, ckpt_every=T_CK)
        cl.close()
        g.close()
    (l64, g64), (l32, g32) = res[torch.float64], res[torch.float32]
    e_loss = abs(l32 - l64) / l64
    e_grad = float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64))
    print(f"split tensor cores vs FP64: loss {e_loss:.2e}, gradient {e_grad:.2e}")
    # measured on a B200: loss 1.4e-5, gradient 1.9e-5
    assert np.isfinite(g32).all()
    assert e_loss < 1e-4
    assert e_grad < 1e-4

"""Time one sweep kernel on synthetic buffers (``sc_microbench``).

    python -m symcode.microbench --kernel x --n 810 --count 65610 [--dtype f32] [--reps 5]

kernel: ``yinv`` (y-inverse sweep over COUNT z planes), ``yfwd`` (y-forward
sweep over COUNT z planes), ``x`` (3D x sweep with products over COUNT rows),
``zinv`` / ``zfwd`` (z sweeps of one component over COUNT ky columns of a
full-size cube, so the lines keep the solver's plane stride).
Prints one JSON line with ms per launch, algorithmic bytes and GB/s.  Used to
make small, self-contained cases of the exact kernels the solver runs (for
ncu) and to compare tile shapes.

``--kernel sfs`` runs sfs! from an n^3 FP32 field to ``--n-les`` at three filter
widths; ``--kernel clark`` / ``dynsmag`` evaluate that closure's ``model(u, G)``
at n^3 (FP32).

``--kernel cnn`` evaluates the tensor-core CNN closure (n = 128, FP32) COUNT
times on a seeded random field and reports ms per evaluation and the
convolutions' TFLOP/s (2 x 27 x sum(C_in C_out) flops per grid point);
``--split`` in split precision (three passes per convolution; the TFLOP/s
count one pass's flops).

``--kernel adjoint`` runs one a-posteriori training rollout of the tensor-core
CNN closure at n^3 (default n = 64 with ``--n 64``): record a target
trajectory of COUNT RK4 steps, then loss and adjoint with checkpoints every 5
steps, timed over REPS repetitions of the adjoint (``--split`` for the split
precision).
"""

import argparse
import ctypes as ct
import json
import sys

from ._lib import check, lib

KERNELS = {"yinv": 0, "yfwd": 1, "x": 2, "zinv": 3, "zfwd": 4}
CNN_LAYERS = ((4, 32), (32, 32), (32, 32), (32, 6))


def run_cnn(n, count, reps=5, split=False):
    import torch

    from . import Grid, create_cnn_closure, kaiming_cnn_weights

    g = Grid(3, n, dtype=torch.float32, device="cuda:0")
    gen = torch.Generator(device="cuda:0").manual_seed(3)
    u = [torch.randn(g.spec_shape, dtype=g.cdtype, device=g.device, generator=gen) * 1e-3 for _ in range(3)]
    ws, bs = kaiming_cnn_weights(7, CNN_LAYERS)
    cl = create_cnn_closure(2 * g.l / n, 1e-3, g, ws, bs, split=split)
    cl(u)
    torch.cuda.synchronize()
    best = None
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(count):
            cl(u)
        e1.record()
        e1.synchronize()
        t = e0.elapsed_time(e1) / count
        best = t if best is None else min(best, t)
    flops = 2.0 * 27 * n ** 3 * sum(ci * co for ci, co in CNN_LAYERS)
    cl.close()
    return {"kernel": "cnn", "n": n, "count": count, "dtype": "f16 split" if split else "bf16", "ms": best,
            "flops": flops, "tflops": flops / (best / 1e3) / 1e12}


def run_adjoint(n, nsteps, reps=1, split=False):
    import time

    import numpy as np
    import torch

    from . import (Grid, closure_set_params, create_cnn_closure, kaiming_cnn_weights, pack_cnn_params,
                   rollout_adjoint, rollout_record)

    g = Grid(3, n, dtype=torch.float32, device="cuda:0")
    gen = torch.Generator(device="cuda:0").manual_seed(5)
    u0 = [torch.randn(g.spec_shape, dtype=g.cdtype, device=g.device, generator=gen) * 1e-3 for _ in range(3)]
    ws, bs = kaiming_cnn_weights(5, CNN_LAYERS)
    theta = pack_cnn_params(ws, bs)
    cl = create_cnn_closure(4 * g.l / n, 1e-3, g, ws, bs, mu=5.0, sigma=2.0, split=split)
    closure_set_params(cl, theta * (1 + 0.01 * np.random.default_rng(6).standard_normal(theta.size)))
    traj = rollout_record(g, cl, u0, 5e-3, 1e-3, nsteps)
    closure_set_params(cl, theta)
    rollout_adjoint(g, cl, u0, traj, 5e-3, 1e-3, nsteps, ckpt_every=5)  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        loss, grad = rollout_adjoint(g, cl, u0, traj, 5e-3, 1e-3, nsteps, ckpt_every=5)
    torch.cuda.synchronize()
    t = (time.perf_counter() - t0) / reps
    cl.close()
    g.close()
    return {"kernel": "adjoint", "n": n, "steps": nsteps, "precision": "split" if split else "bf16",
            "s_per_rollout": t, "ms_per_step": 1e3 * t / nsteps, "loss": loss,
            "grad_finite": bool(np.isfinite(grad).all())}


def run_sfs(n, nl, count, reps=3):
    """sfs! of a seeded n^3 FP32 field to nl^3 at Delta/h in {2, 4, 8}, COUNT calls."""
    import torch

    from . import Grid, random_field, scalarfield, sfs_

    g = Grid(3, n, dtype=torch.float32, device="cuda:0")
    gl = Grid(3, nl, dtype=torch.float32, device="cuda:0")
    u = random_field(g, seed=2, kpeak=4.0)
    deltas = [dh * gl.l / nl for dh in (2, 4, 8)]
    ub = [[scalarfield(gl) for _ in range(3)] for _ in deltas]
    ta = [[scalarfield(gl) for _ in range(6)] for _ in deltas]
    sfs_(ub, ta, u, g, gl, deltas)
    torch.cuda.synchronize()
    best = None
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(count):
            sfs_(ub, ta, u, g, gl, deltas)
        e1.record()
        e1.synchronize()
        t = e0.elapsed_time(e1) / count
        best = t if best is None else min(best, t)
    return {"kernel": "sfs", "n": n, "n_les": nl, "count": count, "ms": best}


def run_closure(kind, n, count, reps=3):
    """One classical closure's tau = model(u, G) on a seeded n^3 FP32 field, COUNT evaluations."""
    import torch

    from . import Grid, create_clark, create_dynamic_smagorinsky, random_field, spacescalarfield, to_phys_

    g = Grid(3, n, dtype=torch.float32, device="cuda:0")
    u = random_field(g, seed=3, kpeak=4.0)
    delta = 2 * g.l / n
    cl = create_clark(delta, g) if kind == "clark" else create_dynamic_smagorinsky(delta, g)
    # physical velocity gradient G[a + 3 b] = to_phys(i k_b u_a), the les! input of model(u, G)
    f = torch.fft.fftfreq(n, 1.0 / n, device=g.device).to(torch.float32)
    ks = (torch.arange(n // 2 + 1, device=g.device, dtype=torch.float32)[None, None, :], f[None, :, None],
          f[:, None, None])
    G = [to_phys_(spacescalarfield(g), (1j * ks[b] * u[a]).contiguous(), g) for b in range(3) for a in range(3)]
    cl(u, G)
    torch.cuda.synchronize()
    best = None
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(count):
            cl(u, G)
        e1.record()
        e1.synchronize()
        t = e0.elapsed_time(e1) / count
        best = t if best is None else min(best, t)
    cl.close()
    return {"kernel": kind, "n": n, "count": count, "ms": best}


def run(kernel, n, count, dtype="f32", reps=5, variant=0):
    ms, by = ct.c_double(), ct.c_double()
    code = KERNELS[kernel] | (int(variant) << 8)  # the sweep's autotuner variant in bits 8..
    check(lib().sc_microbench(code, n, 0 if dtype == "f32" else 1, count, reps, ct.byref(ms), ct.byref(by)))
    return {"kernel": kernel, "variant": variant, "n": n, "count": count, "dtype": dtype, "ms": ms.value,
            "bytes": by.value, "gbs": by.value / (ms.value / 1e3) / 1e9}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel", choices=sorted(KERNELS) + ["cnn", "sfs", "clark", "dynsmag", "adjoint"], required=True)
    ap.add_argument("--n-les", type=int, default=128)
    ap.add_argument("--n", type=int, default=810)
    ap.add_argument("--count", type=int, required=True)
    ap.add_argument("--dtype", choices=["f32", "f64"], default="f32")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--variant", type=int, default=0, help="autotuner variant of the sweep (sc_plan_num_variants)")
    ap.add_argument("--split", action="store_true", help="cnn, adjoint: the CNN's split precision")
    a = ap.parse_args(argv)
    if a.kernel == "cnn":
        print(json.dumps(run_cnn(a.n, a.count, a.reps, a.split)))
    elif a.kernel == "adjoint":
        print(json.dumps(run_adjoint(a.n, a.count, a.reps, a.split)))
    elif a.kernel == "sfs":
        print(json.dumps(run_sfs(a.n, a.n_les, a.count, a.reps)))
    elif a.kernel in ("clark", "dynsmag"):
        print(json.dumps(run_closure(a.kernel, a.n, a.count, a.reps)))
    else:
        print(json.dumps(run(a.kernel, a.n, a.count, a.dtype, a.reps, a.variant)))
    return 0


if __name__ == "__main__":
    sys.exit(main())

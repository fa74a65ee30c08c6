"""Time one sweep kernel on synthetic buffers (``sc_microbench``).

    python -m symcode.microbench --kernel x --n 810 --count 65610 [--dtype f32] [--reps 5]

kernel: ``yinv`` (y-inverse sweep over COUNT z planes), ``yfwd`` (y-forward
sweep over COUNT z planes), ``x`` (3D x sweep with products over COUNT rows),
``zinv`` / ``zfwd`` (z sweeps of one component over COUNT ky columns of a
full-size cube, so the lines keep the solver's plane stride).
Prints one JSON line with ms per launch, algorithmic bytes and GB/s.  Used to
make small, self-contained cases of the exact kernels the solver runs (for
ncu) and to compare tile shapes.

``--kernel cnn`` evaluates the tensor-core CNN closure (n = 128, FP32) COUNT
times on a seeded random field and reports ms per evaluation and the
convolutions' TFLOP/s (2 x 27 x sum(C_in C_out) flops per grid point).
"""

import argparse
import ctypes as ct
import json
import sys

from ._lib import check, lib

KERNELS = {"yinv": 0, "yfwd": 1, "x": 2, "zinv": 3, "zfwd": 4}
CNN_LAYERS = ((4, 32), (32, 32), (32, 32), (32, 6))


def run_cnn(n, count, reps=5):
    import torch

    from . import Grid, create_cnn_closure, kaiming_cnn_weights

    g = Grid(3, n, dtype=torch.float32, device="cuda:0")
    gen = torch.Generator(device="cuda:0").manual_seed(3)
    u = [torch.randn(g.spec_shape, dtype=g.cdtype, device=g.device, generator=gen) * 1e-3 for _ in range(3)]
    ws, bs = kaiming_cnn_weights(7, CNN_LAYERS)
    cl = create_cnn_closure(2 * g.l / n, 1e-3, g, ws, bs)
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
    return {"kernel": "cnn", "n": n, "count": count, "dtype": "bf16", "ms": best, "flops": flops,
            "tflops": flops / (best / 1e3) / 1e12}


def run(kernel, n, count, dtype="f32", reps=5, variant=0):
    ms, by = ct.c_double(), ct.c_double()
    code = KERNELS[kernel] | (int(variant) << 8)  # the sweep's autotuner variant in bits 8..
    check(lib().sc_microbench(code, n, 0 if dtype == "f32" else 1, count, reps, ct.byref(ms), ct.byref(by)))
    return {"kernel": kernel, "variant": variant, "n": n, "count": count, "dtype": dtype, "ms": ms.value,
            "bytes": by.value, "gbs": by.value / (ms.value / 1e3) / 1e9}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel", choices=sorted(KERNELS) + ["cnn"], required=True)
    ap.add_argument("--n", type=int, default=810)
    ap.add_argument("--count", type=int, required=True)
    ap.add_argument("--dtype", choices=["f32", "f64"], default="f32")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--variant", type=int, default=0, help="autotuner variant of the sweep (sc_plan_num_variants)")
    a = ap.parse_args(argv)
    if a.kernel == "cnn":
        print(json.dumps(run_cnn(a.n, a.count, a.reps)))
    else:
        print(json.dumps(run(a.kernel, a.n, a.count, a.dtype, a.reps, a.variant)))
    return 0


if __name__ == "__main__":
    sys.exit(main())

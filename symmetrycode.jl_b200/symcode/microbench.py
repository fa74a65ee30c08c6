"""Time one sweep kernel on synthetic buffers (``sc_microbench``).

    python -m symcode.microbench --kernel x --n 810 --count 65610 [--dtype f32] [--reps 5]

kernel: ``yinv`` (y-inverse sweep over COUNT z planes), ``yfwd`` (y-forward
sweep over COUNT z planes) or ``x`` (3D x sweep with products over COUNT rows).
Prints one JSON line with ms per launch, algorithmic bytes and GB/s.  Used to
make small, self-contained cases of the exact kernels the solver runs (for
ncu) and to compare tile shapes.
"""

import argparse
import ctypes as ct
import json
import sys

from ._lib import check, lib

KERNELS = {"yinv": 0, "yfwd": 1, "x": 2}


def run(kernel, n, count, dtype="f32", reps=5):
    ms, by = ct.c_double(), ct.c_double()
    check(lib().sc_microbench(KERNELS[kernel], n, 0 if dtype == "f32" else 1, count, reps, ct.byref(ms), ct.byref(by)))
    return {"kernel": kernel, "n": n, "count": count, "dtype": dtype, "ms": ms.value,
            "bytes": by.value, "gbs": by.value / (ms.value / 1e3) / 1e9}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel", choices=sorted(KERNELS), required=True)
    ap.add_argument("--n", type=int, default=810)
    ap.add_argument("--count", type=int, required=True)
    ap.add_argument("--dtype", choices=["f32", "f64"], default="f32")
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args(argv)
    print(json.dumps(run(a.kernel, a.n, a.count, a.dtype, a.reps)))
    return 0


if __name__ == "__main__":
    sys.exit(main())

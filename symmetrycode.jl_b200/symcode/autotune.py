"""Autotuner of the FP32 sweep kernels: tile shapes, FFT splits and x-sweep kernels.

The reference gets its transform plan from cuFFT / FFTW planning
(``plan_rfft``, src/solver.jl:432).  Here each of the five sweeps of the 3D
product pipeline of an FP32 plan (z-inverse, y-inverse, x, y-forward,
z-forward) has a few kernel variants -- the same transform with another
column-tile width, the transposed two-level split N = N1 N2, or another
x-sweep kernel (``sc_plan_num_variants``).  ``tune`` times every variant of
every sweep on the plan's own buffers with CUDA events
(``sc_state_profile_rhs``, one right-hand side of the plan's state per
repetition), keeps the fastest per sweep (``sc_plan_set_option``) and records
the choice and the timings in a JSON cache keyed by device, grid and
precision, so later plans of the same shape reuse it without timing.

Usage::

    g = Grid(3, 810, dtype=torch.float32)
    State(g).load(u)                      # any field: the timing does not depend on it
    report = autotune.tune(g, visc=6e-4)  # {"variants": {...}, "ms": {...}, "source": ...}
"""

from __future__ import annotations

import ctypes as ct
import json
import os
import tempfile

from ._lib import SC_OPT_VARIANT_ZINV, check, lib

SWEEPS = ("z_inverse", "y_inverse", "x_sweep", "y_forward", "z_forward")


def num_variants(g):
    """Variant count of each sweep of the plan (1: nothing to choose)."""
    out = []
    for s in range(len(SWEEPS)):
        c = ct.c_int()
        check(lib().sc_plan_num_variants(g.plan, s, ct.byref(c)))
        out.append(c.value)
    return out


def set_variants(g, variants):
    """Apply {sweep name: variant} to the plan."""
    for s, name in enumerate(SWEEPS):
        if name in variants:
            check(lib().sc_plan_set_option(g.plan, SC_OPT_VARIANT_ZINV + s, int(variants[name])))


def choose(timings, counts):
    """The fastest variant of each sweep.

    timings: {variant: {sweep name: ms}} (a sweep appears under the variants it
    has); counts: variants per sweep.  Ties keep the lower variant (0 is the
    default).  Returns {sweep name: variant} for the sweeps with a choice."""
    best = {}
    for s, name in enumerate(SWEEPS):
        if counts[s] <= 1:
            continue
        cand = [(timings[v][name], v) for v in sorted(timings) if v < counts[s] and name in timings[v]]
        if cand:
            best[name] = min(cand)[1]
    return best


def cache_key(device_name, D, n, dtype_name):
    return f"{device_name}|D={D}|n={n}|{dtype_name}"


def default_cache_path():
    return os.environ.get("SC_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "symcode_tune.json"))


def load_cache(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save_cache(path, key, entry):
    """Merge one entry into the cache file, written to a temporary file and
    renamed over the old one (the atomic write of the reference's
    ``jldsave_atomic``, src/solver.jl:76-86)."""
    data = load_cache(path)
    data[key] = entry
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    fd, tmp = tempfile.mkstemp(dir=d, prefix=".symcode_tune_")
    try:
        with os.fdopen(fd, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except BaseException:
        if os.path.exists(tmp):
            os.remove(tmp)
        raise


def measure(g, visc, reps, counts):
    """{variant: {sweep: ms}}: every sweep runs variant v where it has one (the
    default elsewhere), one right-hand side per repetition after a warm-up."""
    from . import State
    st = State(g)
    timings = {}
    for v in range(max(counts)):
        set_variants(g, {name: (v if v < counts[s] else 0) for s, name in enumerate(SWEEPS)})
        st.profile_rhs(visc, 1)  # warm-up (first launch of the variant)
        ms = st.profile_rhs(visc, reps)
        timings[v] = {name: ms[s] for s, name in enumerate(SWEEPS) if v < counts[s]}
    return timings


def tune(g, visc=1e-3, reps=3, cache=None, force=False):
    """Pick and apply the fastest variant of each sweep of the plan of `g`.

    cache: JSON path (default ``$SC_TUNE_CACHE`` or ``~/.cache/symcode_tune.json``;
    ``False`` disables it).  A cached choice for the same device, grid and
    precision is applied without timing unless `force`."""
    import torch
    counts = num_variants(g)
    if max(counts) <= 1:
        return {"variants": {}, "ms": {}, "source": "no choice"}
    dname = torch.cuda.get_device_name(g.device)
    key = cache_key(dname, g.D, g.n, str(g.dtype).replace("torch.", ""))
    path = default_cache_path() if cache is None else cache
    if path and not force:
        hit = load_cache(path).get(key)
        if hit and all(name in hit.get("variants", {}) for s, name in enumerate(SWEEPS) if counts[s] > 1):
            set_variants(g, hit["variants"])
            return {"variants": hit["variants"], "ms": hit.get("ms", {}), "source": "cache"}
    timings = measure(g, visc, reps, counts)
    best = choose(timings, counts)
    set_variants(g, {name: best.get(name, 0) for name in SWEEPS})
    entry = {"variants": best, "ms": {str(v): t for v, t in timings.items()}}
    if path:
        save_cache(path, key, entry)
    return {"variants": best, "ms": entry["ms"], "source": "timed"}

"""DNS -> LES filter (sfs!) through the C ABI against the FP64 oracle."""

import math

import numpy as np
import pytest
import torch

import oracle as O
import symcode as S
from _util import rel_l2, to_dev, to_np

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("D,nd,nl,dtype,tol", [
    (3, 48, 24, torch.float64, 1e-12),
    (3, 64, 32, torch.float64, 1e-12),
    (2, 256, 64, torch.float64, 1e-12),
    (3, 128, 64, torch.float32, 1e-5),
    (3, 64, 64, torch.float64, 1e-12),
])
def test_sfs_matches_oracle(D, nd, nl, dtype, tol):
    gd, gl = S.Grid(D, nd, dtype=dtype, device="cuda:0"), S.Grid(D, nl, dtype=dtype, device="cuda:0")
    od, ol = O.Grid(D, nd), O.Grid(D, nl)
    u = O.random_field(od, seed=11, kpeak=3)
    h = ol.l / ol.n
    deltas = [None, 2 * h, 4 * h]
    ub = [S.vectorfield(gl) for _ in deltas]
    ta = [[S.scalarfield(gl) for _ in range(gl.tensordim)] for _ in deltas]
    S.sfs_(ub, ta, [to_dev(c, gd) for c in u], gd, gl, deltas)
    sig_dns = O.nonlinearity(u, od)
    for d, b, t in zip(deltas, ub, ta):
        rb, rt = O.sfs(u, od, ol, d)
        assert rel_l2([to_np(c) for c in b], rb) < tol
        # tau is a difference of two nearly equal product spectra: its error is
        # measured against the size of the filtered DNS products it cancels
        s1 = [O.twothirds(O.cutoff(c, od, ol) if d is None else O.gaussianfilter(O.cutoff(c, od, ol), d, ol), ol)
              for c in sig_dns]
        scale = math.sqrt(sum(float(np.sum(np.abs(c) ** 2)) for c in s1))
        err = math.sqrt(sum(float(np.sum(np.abs(to_np(x) - y) ** 2)) for x, y in zip(t, rt)))
        assert err < tol * scale
        re = S.filter_reynolds(b, gl, 1e-3, 2 * h)
        assert math.isclose(re, O.filter_reynolds(rb, ol, 1e-3, 2 * h), rel_tol=max(tol, 1e-12))


def test_sfs_rejects_same_plan_and_finer_les():
    g = S.Grid(3, 16, dtype=torch.float64, device="cuda:0")
    g2 = S.Grid(3, 32, dtype=torch.float64, device="cuda:0")
    u = S.vectorfield(g)
    with pytest.raises(S.SymcodeError):
        S.sfs_(S.vectorfield(g), S.tensorfield(g), u, g, g, 0.1)
    with pytest.raises(S.SymcodeError):
        S.sfs_(S.vectorfield(g2), S.tensorfield(g2), u, g, g2, 0.1)


def test_sfs_810_fp32_matches_fp64_path():
    """At 810^3 -> 128^3 the FP32 filter runs the 810 kernels with a pruned
    output width (the product spectra are formed only up to the LES cutoff);
    it agrees with the FP64 path (pinned to the oracle at smaller sizes) on the
    same input bytes."""
    nd, nl = 810, 128
    gen = torch.Generator(device="cuda:0").manual_seed(5)
    g32 = S.Grid(3, nd, dtype=torch.float32, device="cuda:0")
    u64 = [torch.randn(g32.spec_shape, dtype=torch.complex128, device="cuda:0", generator=gen) * 1e-3
           for _ in range(3)]
    u32 = [c.to(torch.complex64) for c in u64]
    del u64
    h = 2 * math.pi / nl
    deltas = [None, 2 * h, 4 * h]

    def run(gd, u, dtype):
        gl = S.Grid(3, nl, dtype=dtype, device="cuda:0")
        ub = [S.vectorfield(gl) for _ in deltas]
        ta = [[S.scalarfield(gl) for _ in range(gl.tensordim)] for _ in deltas]
        S.sfs_(ub, ta, u, gd, gl, deltas)
        out = ([[c.to(torch.complex128) for c in b] for b in ub], [[c.to(torch.complex128) for c in t] for t in ta])
        gl.close()
        return out

    ub32, ta32 = run(g32, u32, torch.float32)
    g32.close()
    g64 = S.Grid(3, nd, dtype=torch.float64, device="cuda:0")
    ub64, ta64 = run(g64, [c.to(torch.complex128) for c in u32], torch.float64)
    g64.close()

    def rel(a, b):
        num = sum(float((x - y).abs().pow(2).sum()) for x, y in zip(a, b))
        den = sum(float(y.abs().pow(2).sum()) for y in b)
        return (num / den) ** 0.5

    # measured: ubar 3.5e-8, tau 4.8e-7 .. 7.9e-7 (relative L2 per width)
    for b32, b64, t32, t64 in zip(ub32, ub64, ta32, ta64):
        assert rel(b32, b64) < 1e-6
        assert rel(t32, t64) < 1e-5

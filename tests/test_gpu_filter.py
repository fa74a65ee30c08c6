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

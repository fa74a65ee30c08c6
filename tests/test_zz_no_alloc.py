"""sc_spectrum_static (allocation-free spectrum, fixed device scratch) against sc_spectrum.

Collected last on purpose: it must give the same shells whether it runs alone
or after every other test has used the device.
"""

import ctypes as ct

import numpy as np
import pytest
import torch

import oracle as O
import symcode as S
from symcode import _lib as L
from _util import to_dev


def _spectrum_static(u, n, D, dtype, nshell):
    pu, _keep = L.ptr_array([c.data_ptr() for c in u])
    s = (ct.c_double * nshell)()
    L.check(L.lib().sc_spectrum_static(pu, n, D, dtype, nshell, s, None))
    return np.array(s)


@pytest.mark.gpu
@pytest.mark.parametrize("D,n,dtype", [(3, 48, torch.float64), (3, 64, torch.float32), (2, 96, torch.float64),
                                       (2, 120, torch.float32)])
def test_static_spectrum_matches_sc_spectrum(D, n, dtype):
    g, go = S.Grid(D, n, dtype=dtype, device="cuda:0"), O.Grid(D, n)
    u = O.random_field(go, seed=60, kpeak=4)
    ut = [to_dev(c, g) for c in u]
    nshell = n // 3
    ref = np.array(S.spectrum(ut, g, nshell))
    code = L.SC_FLOAT64 if dtype == torch.float64 else L.SC_FLOAT32
    # two calls in a row: the scratch is re-zeroed by each call
    for _ in range(2):
        s = _spectrum_static(ut, n, D, code, nshell)
        assert np.allclose(s, ref, rtol=1e-12, atol=1e-300)
    # the defining property: further calls take no device memory (neither the
    # device's free memory nor torch's caching pool moves)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    res0 = torch.cuda.memory_reserved()
    for _ in range(3):
        s = _spectrum_static(ut, n, D, code, nshell)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0 and torch.cuda.memory_reserved() == res0
    assert np.allclose(s, ref, rtol=1e-12, atol=1e-300)
    # fewer shells than the plan's n/3 reads the same leading shells
    s = _spectrum_static(ut, n, D, code, 5)
    assert np.allclose(s, ref[:5], rtol=1e-12, atol=1e-300)


def test_static_spectrum_rejects_oversize_requests():
    # argument checks run before any CUDA call, so no device is touched here
    dummy = [ct.c_void_p(16)] * 3
    pu = ct.cast((ct.c_void_p * 3)(*dummy), ct.POINTER(ct.c_void_p))
    s = (ct.c_double * 600)()
    lib = L.lib()
    rc = lib.sc_spectrum_static(pu, 2048, 3, L.SC_FLOAT64, 513, s, None)
    assert rc == L.SC_ERR_SIZE
    assert b"static shell scratch" in lib.sc_last_error_string()
    assert lib.sc_spectrum_static(pu, 48, 3, L.SC_FLOAT64, 17, s, None) == L.SC_ERR_INVALID
    assert lib.sc_spectrum_static(pu, 47, 3, L.SC_FLOAT64, 5, s, None) == L.SC_ERR_SIZE

"""The C-ABI library loads and exports every entry point include/symcode.h declares (no GPU needed)."""

import ctypes as ct

import pytest
import torch

from symcode import _lib


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = _lib.header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(_lib._SIGS), "ctypes signatures out of sync with include/symcode.h"


def test_abi_version_and_sizes():
    L = _lib.lib()
    assert L.sc_abi_version() == 1
    for n in (4, 8, 16, 24, 30, 64, 90, 128, 256, 810):
        assert L.sc_fft_size_supported(n) == 1
    for n in (7, 14, 22, 26, 1000):
        assert L.sc_fft_size_supported(n) == 0


def test_plan_create_rejects_bad_arguments():
    L = _lib.lib()
    p = ct.c_void_p()
    assert L.sc_plan_create(ct.byref(p), 3, 7, 1.0, 0, None) == _lib.SC_ERR_SIZE
    assert b"even" in L.sc_last_error_string()
    assert L.sc_plan_create(ct.byref(p), 4, 8, 1.0, 0, None) == _lib.SC_ERR_INVALID
    assert L.sc_plan_create(ct.byref(p), 3, 22, 1.0, 0, None) == _lib.SC_ERR_SIZE
    assert L.sc_plan_create(ct.byref(p), 3, 8, 1.0, 5, None) == _lib.SC_ERR_INVALID
    assert L.sc_plan_create(None, 3, 8, 1.0, 0, None) == _lib.SC_ERR_INVALID
    assert L.sc_plan_destroy(None) == 0


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device error path")
def test_plan_create_without_device_fails_loudly():
    L = _lib.lib()
    p = ct.c_void_p()
    st = L.sc_plan_create(ct.byref(p), 3, 8, 1.0, 0, None)
    assert st == _lib.SC_ERR_CUDA
    import symcode
    with pytest.raises(RuntimeError):
        symcode.Grid(3, 8)


def test_closure_set_option_rejects_a_null_closure():
    # the null check runs before any CUDA call
    L = _lib.lib()
    assert L.sc_closure_set_option(None, _lib.SC_CLOPT_CNN_SPLIT, 1) == _lib.SC_ERR_INVALID
    assert b"null" in L.sc_last_error_string()

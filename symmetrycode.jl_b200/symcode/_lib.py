"""ctypes binding of ``libsymcode.so`` (declarations in include/symcode.h).

The library is loaded from the package directory; there is no fallback: if it
is missing, or no CUDA device is present, the calls that need it raise.
"""

from __future__ import annotations

import ctypes as ct
import os
import re

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libsymcode.so")
HEADER = os.path.join(os.path.dirname(PKG_DIR), "include", "symcode.h")

SC_OK, SC_ERR_INVALID, SC_ERR_SIZE, SC_ERR_CUDA, SC_ERR_OOM, SC_ERR_DIVERGED, SC_ERR_UNSUPPORTED, SC_ERR_TIMEOUT = range(8)
SC_FLOAT32, SC_FLOAT64 = 0, 1
SC_OPT_USE_GRAPH, SC_OPT_WAIT_LIMIT = 1, 2  # sc_plan_set_option
SC_OPT_VARIANT_ZINV = 3  # ... SC_OPT_VARIANT_ZFWD = 7: sweep variants (z-inv, y-inv, x, y-fwd, z-fwd)
SC_CLOPT_CNN_SPLIT = 1  # sc_closure_set_option: split-precision tensor-core CNN


class SymcodeError(RuntimeError):
    """Raised when a C-ABI call returns a non-zero sc_status."""

    def __init__(self, status, msg):
        super().__init__(f"[sc_status {status}] {msg}")
        self.status = status


class sc_forcing(ct.Structure):
    _fields_ = [("enabled", ct.c_int), ("eps", ct.c_double)]


class sc_les_instance(ct.Structure):
    _fields_ = [("plan", ct.c_void_p), ("closure", ct.c_void_p), ("visc", ct.c_double), ("dt", ct.c_double),
                ("forced", ct.c_int), ("eps", ct.c_double)]


class sc_rollout_job(ct.Structure):
    _fields_ = [("plan", ct.c_void_p), ("closure", ct.c_void_p), ("u0", ct.c_void_p * 3), ("traj", ct.c_void_p),
                ("dt", ct.c_double), ("visc", ct.c_double), ("nsteps", ct.c_int), ("ckpt_every", ct.c_int),
                ("loss", ct.POINTER(ct.c_double)), ("grad", ct.POINTER(ct.c_double))]


_vp = ct.c_void_p
_pp = ct.POINTER(ct.c_void_p)

_SIGS = {
    "sc_abi_version": ([], ct.c_int),
    "sc_last_error_string": ([], ct.c_char_p),
    "sc_fft_size_supported": ([ct.c_int], ct.c_int),
    "sc_plan_create": ([ct.POINTER(_vp), ct.c_int, ct.c_int, ct.c_double, ct.c_int, ct.POINTER(ct.c_size_t)], ct.c_int),
    "sc_plan_destroy": ([_vp], ct.c_int),
    "sc_plan_info": ([_vp, ct.POINTER(ct.c_int), ct.POINTER(ct.c_int), ct.POINTER(ct.c_int), ct.POINTER(ct.c_int)], ct.c_int),
    "sc_to_phys": ([_vp, _vp, _vp, _vp], ct.c_int),
    "sc_to_spec": ([_vp, _vp, _vp, _vp], ct.c_int),
    "sc_twothirds": ([_vp, _pp, ct.c_int, _vp], ct.c_int),
    "sc_project": ([_vp, _pp, _vp], ct.c_int),
    "sc_rhs": ([_vp, _pp, _pp, ct.c_double, _vp], ct.c_int),
    "sc_wray3_step": ([_vp, _pp, ct.c_double, ct.c_double, _vp], ct.c_int),
    "sc_rk4_steps": ([_vp, _pp, ct.c_double, ct.c_double, ct.c_int, ct.POINTER(sc_forcing), _vp], ct.c_int),
    "sc_state_load": ([_vp, _pp, _vp], ct.c_int),
    "sc_state_store": ([_vp, _pp, _vp], ct.c_int),
    "sc_state_rk4": ([_vp, ct.c_double, ct.c_double, ct.c_int, ct.POINTER(sc_forcing), _vp], ct.c_int),
    "sc_state_energy": ([_vp, ct.POINTER(ct.c_double), _vp], ct.c_int),
    "sc_state_rk4_launches_per_step": ([_vp, ct.c_int], ct.c_int),
    "sc_state_profile_rhs": ([_vp, ct.c_double, ct.c_int, ct.POINTER(ct.c_double), ct.POINTER(ct.c_int), _vp], ct.c_int),
    "sc_microbench": ([ct.c_int, ct.c_int, ct.c_int, ct.c_longlong, ct.c_int, ct.POINTER(ct.c_double), ct.POINTER(ct.c_double)], ct.c_int),
    "sc_filter_sfs": ([_vp, _vp, _pp, ct.POINTER(ct.c_double), ct.c_int, _pp, _pp, _vp], ct.c_int),
    "sc_filter_reynolds": ([_vp, _pp, ct.c_double, ct.c_double, ct.POINTER(ct.c_double), _vp], ct.c_int),
    "sc_closure_create": ([ct.POINTER(_vp), _vp, ct.c_int, ct.c_double, ct.POINTER(ct.c_double), ct.c_int], ct.c_int),
    "sc_closure_destroy": ([_vp], ct.c_int),
    "sc_cnn_closure_create": ([ct.POINTER(_vp), _vp, ct.c_double, ct.c_double, ct.POINTER(ct.POINTER(ct.c_float)),
                               ct.POINTER(ct.POINTER(ct.c_float)), ct.c_double, ct.c_double], ct.c_int),
    "sc_closure_status": ([_vp, ct.POINTER(ct.c_int)], ct.c_int),
    "sc_cnn_fp_closure_create": ([ct.POINTER(_vp), _vp, ct.c_double, ct.c_double, ct.POINTER(ct.POINTER(ct.c_float)),
                                  ct.POINTER(ct.POINTER(ct.c_float)), ct.c_double, ct.c_double], ct.c_int),
    "sc_closure_num_params": ([_vp, ct.POINTER(ct.c_longlong)], ct.c_int),
    "sc_closure_set_params": ([_vp, ct.POINTER(ct.c_double)], ct.c_int),
    "sc_closure_set_option": ([_vp, ct.c_int, ct.c_longlong], ct.c_int),
    "sc_rollout_traj_bytes": ([_vp, ct.c_int], ct.c_size_t),
    "sc_rollout_record": ([_vp, _vp, _pp, ct.c_double, ct.c_double, ct.c_int, _vp, _vp], ct.c_int),
    "sc_rollout_loss": ([_vp, _vp, _pp, _vp, ct.c_double, ct.c_double, ct.c_int, ct.POINTER(ct.c_double), _vp], ct.c_int),
    "sc_rollout_adjoint": ([_vp, _vp, _pp, _vp, ct.c_double, ct.c_double, ct.c_int, ct.c_int, ct.POINTER(ct.c_double),
                            ct.POINTER(ct.c_double), _vp], ct.c_int),
    "sc_closure_eval": ([_vp, _pp, _pp, _pp, _vp], ct.c_int),
    "sc_les_rhs": ([_vp, _vp, _pp, _pp, ct.c_double, _vp], ct.c_int),
    "sc_les_wray3_step": ([_vp, _vp, _pp, ct.c_double, ct.c_double, _vp], ct.c_int),
    "sc_les_rk4_steps": ([_vp, _vp, _pp, ct.c_double, ct.c_double, ct.c_int, ct.POINTER(sc_forcing), _vp], ct.c_int),
    "sc_state_les_rk4": ([_vp, _vp, ct.c_double, ct.c_double, ct.c_int, ct.POINTER(sc_forcing), _vp], ct.c_int),
    "sc_les_batch_create": ([ct.POINTER(_vp), ct.POINTER(sc_les_instance), ct.c_int], ct.c_int),
    "sc_les_batch_run": ([_vp, ct.c_int, _vp], ct.c_int),
    "sc_les_batch_status": ([_vp, ct.POINTER(ct.c_int), ct.POINTER(ct.c_double), ct.c_int, _vp], ct.c_int),
    "sc_les_batch_set_snapshots": ([_vp, ct.c_int, ct.c_int, ct.c_int], ct.c_int),
    "sc_random_field": ([_vp, ct.c_ulonglong, _pp, ct.c_double, ct.c_double, _pp, _vp], ct.c_int),
    "sc_les_batch_snapshots": ([_vp, ct.POINTER(ct.c_int), ct.POINTER(ct.c_double), _vp], ct.c_int),
    "sc_les_batch_destroy": ([_vp], ct.c_int),
    "sc_plan_set_option": ([_vp, ct.c_int, ct.c_longlong], ct.c_int),
    "sc_plan_num_variants": ([_vp, ct.c_int, ct.POINTER(ct.c_int)], ct.c_int),
    "sc_plan_status": ([_vp, ct.POINTER(ct.c_int)], ct.c_int),
    "sc_propose_timestep": ([_vp, _pp, ct.c_double, ct.POINTER(ct.c_double), _vp], ct.c_int),
    "sc_shell_energies": ([_vp, _pp, ct.POINTER(ct.c_double), _vp], ct.c_int),
    "sc_maintain_shell_energy": ([_vp, _pp, ct.POINTER(ct.c_double), _vp], ct.c_int),
    "sc_state_maintain_shell_energy": ([_vp, ct.POINTER(ct.c_double), _vp], ct.c_int),
    "sc_spectrum": ([_vp, _pp, ct.c_int, ct.POINTER(ct.c_double), _vp], ct.c_int),
    "sc_rollout_adjoint_batch": ([ct.c_int, ct.POINTER(sc_rollout_job), ct.POINTER(ct.c_int), _vp], ct.c_int),
    "sc_les_diagnostics": ([_vp, _vp, _pp, _pp, ct.c_double, ct.c_int, ct.POINTER(ct.c_double),
                            ct.POINTER(ct.c_double), ct.POINTER(ct.c_double), _vp], ct.c_int),
    "sc_mlp_closure_create": ([ct.POINTER(ct.c_void_p), _vp, ct.c_double, ct.c_double, ct.c_int,
                               ct.POINTER(ct.c_int), ct.POINTER(ct.c_double), ct.c_int, ct.c_double, ct.c_double],
                              ct.c_int),
    "sc_tbnn_closure_create": ([ct.POINTER(ct.c_void_p), _vp, ct.c_double, ct.c_double, ct.c_int,
                                ct.POINTER(ct.c_int), ct.POINTER(ct.c_double), ct.c_int, ct.c_double, ct.c_double],
                               ct.c_int),
    "sc_spectrum_static": ([_pp, ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.POINTER(ct.c_double), _vp], ct.c_int),
    "sc_energy": ([_vp, _pp, ct.POINTER(ct.c_double), _vp], ct.c_int),
    "sc_dissipation": ([_vp, _pp, ct.c_double, ct.POINTER(ct.c_double), _vp], ct.c_int),
}

_lib = None


def header_functions(path=HEADER):
    """Names of every entry point declared in include/symcode.h."""
    txt = open(path).read()
    return re.findall(r"^SC_API\s+(?:const\s+)?\w+\*?\s+(sc_\w+)\s*\(", txt, flags=re.M)


def lib():
    """Load libsymcode.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python symmetrycode.jl_b200/build.py` "
                "(the CUDA path has no fallback)")
        L = ct.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def check(status):
    if status != SC_OK:
        msg = lib().sc_last_error_string()
        raise SymcodeError(status, msg.decode() if msg else "")


def ptr_array(ptrs):
    arr = (ct.c_void_p * len(ptrs))(*[ct.c_void_p(int(p)) for p in ptrs])
    return ct.cast(arr, _pp), arr

"""The bounded-wait failure path of the tensor-core CNN closure, made to run out on purpose.

Every mbarrier wait of the tcgen05 convolution kernels is bounded.  With the
plan option SC_OPT_WAIT_LIMIT = 0 each wait of the row pipeline gives up at
once: the kernel sets the closure's error flag, gives the MMAs it already
issued one more wait with the full default bound, frees its tensor memory and
returns.  Nothing hangs and nothing faults; sc_closure_status reports
SC_ERR_TIMEOUT, and the context stays usable: with the default bound restored a
fresh closure on the same plan evaluates correctly.
"""

import ctypes as ct

import numpy as np
import pytest
import torch

import oracle as O
import symcode as S
from symcode import _lib as L
from _util import rel_l2, to_dev, to_np

pytestmark = pytest.mark.gpu


def _status(cl):
    st = ct.c_int(-1)
    L.check(L.lib().sc_closure_status(cl.ptr, ct.byref(st)))
    return st.value


def test_cnn_wait_timeout_is_reported_and_the_context_recovers():
    n = 64
    g = S.Grid(3, n, dtype=torch.float32, device="cuda:0")
    go = O.Grid(3, n)
    u = O.random_field(go, seed=44, kpeak=4)
    ut = [to_dev(c, g) for c in u]
    delta, nu = 4 * go.l / n, 5e-4
    ws, bs = S.kaiming_cnn_weights(9)

    S.set_option(g, L.SC_OPT_WAIT_LIMIT, 0)  # every pipeline wait gives up at once
    cl = S.create_cnn_closure(delta, nu, g, ws, bs, mu=1.0, sigma=2.0)
    with pytest.raises(S.SymcodeError) as err:  # the evaluation reports the timeout
        cl(ut, None)
    assert err.value.status == L.SC_ERR_TIMEOUT
    torch.cuda.synchronize()  # the kernels returned: no hang, no fault
    assert _status(cl) == L.SC_ERR_TIMEOUT
    cl.close()

    S.set_option(g, L.SC_OPT_WAIT_LIMIT, -1)  # back to the default bound
    cl2 = S.create_cnn_closure(delta, nu, g, ws, bs, mu=1.0, sigma=2.0)
    tau = to_np(cl2(ut, None))
    assert _status(cl2) == L.SC_OK
    uphys = np.stack([to_np(S.to_phys_(S.spacescalarfield(g), c, g)) for c in ut], 0)
    zval = O.cnn_redelta_channel(u, go, delta, nu, mu=1.0, sigma=2.0)
    rows = [(0, 0), (13, 7), (63, 32)]
    ref = O.cnn_rows(uphys, zval, ws, bs, rows)
    got = np.stack([tau[:, z, y, :] for (y, z) in rows], 1)
    assert rel_l2(got, ref) < 5e-3
    cl2.close()
    g.close()

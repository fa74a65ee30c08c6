"""The 810^3 FP32 production kernels against the FP64 oracles, on the benchmark's own input.

At n = 810 every sweep of the solver runs its production kernel: the z and y
column sweeps (two-level 27 x 30 register FFTs on the 2/3-rule compact layout)
and the three-level 9 x 9 x 10 x sweep with the six products.  These tests pin
them (and the FP64 path at 810) to two independent FP64 oracles:

* ``oracle.triad``: exact triad sums of a sparse field (a few hundred retained
  modes, including the cube's faces and corners, kx = 0, kx = 270 and the forced
  band), no FFT at all, so the comparison covers every output mode exactly;
* ``oracle.compact``: the FFT oracle on the compact 2/3 cube, run at full size
  on the host on the seeded field of the 810^3 benchmark (spectrum
  k^4 exp(-2 (k/4)^2), solenoidal, unit energy, seed 2).

Tolerances: FP64 <= 1e-12 relative L2; FP32 <= 1e-5 per right-hand side
against the exact triad oracle, 1.2e-5 on the benchmark field (the FP32 floor
of this RHS at 810^3, see the test), and 2e-5 on one RK4 step of the state
(with the increment u1 - u0 within 1e-4);
filter: ubar <= 1e-6, tau within 1e-5 of the filtered DNS products it cancels.
"""

import math

import numpy as np
import pytest
import torch

import symcode as S
from oracle import triad as T
from oracle.compact import CompactOracle
from symcode import fields

pytestmark = pytest.mark.gpu

N, NU, DT, EPS, SEED = 810, 6e-4, 2e-3, 0.1, 2
DEV = "cuda:0"


def _compact_t(t, n):
    """Retained 2/3 cube of a full-layout (n, n, n/2+1) device tensor, on the host (complex128)."""
    k = n // 3
    idx = torch.cat([torch.arange(k + 1), torch.arange(n - k, n)]).to(t.device)
    c = t.index_select(0, idx).index_select(1, idx)[:, :, : k + 1]
    return c.to(torch.complex128).cpu().numpy()


def _rel(a, b):
    num = sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(a, b))
    den = sum(float(np.sum(np.abs(y) ** 2)) for y in b)
    return math.sqrt(num / den)


def _full_dev(uc, n, dtype):
    cd = np.complex64 if dtype == torch.float32 else np.complex128
    return [torch.from_numpy(fields.compact_to_full(c.astype(cd), n)).to(DEV) for c in uc]


@pytest.fixture(scope="module")
def bench_field():
    return fields.random_field_compact(3, N, SEED, kpeak=4.0, totalenergy=1.0)


@pytest.fixture(scope="module")
def oracle810():
    o = CompactOracle(N)
    yield o
    o.release()


def _triad_err(du, ref, idx):
    """Relative L2 error of the device spectra du against the triad oracle's
    values ref at the oracle's modes idx; every other mode must be zero, so its
    energy counts as error (summed directly: a difference of two large sums
    would lose it to rounding)."""
    num = den = 0.0
    for c in range(3):
        got = du[c][idx].to(torch.complex128)
        num += float((got - ref[c]).abs().pow(2).sum())
        den += float(ref[c].abs().pow(2).sum())
        rest = du[c].clone()
        rest[idx] = 0
        num += float(rest.abs().to(torch.float64).pow(2).sum())
        del rest
    return math.sqrt(num / den)


# --------------------------------------------------------------- exact (triad) oracle
EDGES = [(270, 270, 270), (270, -270, 270), (270, 0, -270), (0, 270, -270), (0, 270, 270), (0, 1, 0),
         (0, 0, 1), (1, 1, 1), (2, 0, -1), (1, -2, 1), (135, 270, -3), (269, -1, 270), (3, -270, -270)]


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 1e-5)])
def test_rhs_810_matches_triad_oracle(dtype, tol):
    k, u = T.random_sparse_field(N, 300, 21, extra=EDGES)
    kout, du_ref = T.convectiondiffusion(k, u, N, NU)
    g = S.Grid(3, N, dtype=dtype, device=DEV)
    kf, uf = T.full_modes(k, u)
    m = kf[:, 0] >= 0
    iz, iy, ix = (torch.from_numpy(a).to(DEV) for a in T.to_rfft_index(kf[m], N))
    uin = []
    for c in range(3):
        t = torch.zeros(g.spec_shape, dtype=g.cdtype, device=DEV)
        t[iz, iy, ix] = torch.from_numpy(uf[m][:, c]).to(g.cdtype).to(DEV)
        uin.append(t)
    du = S.vectorfield(g)
    S.convectiondiffusion_(du, uin, g, NU)
    del uin
    oz, oy, ox = (torch.from_numpy(a).to(DEV) for a in T.to_rfft_index(kout, N))
    ref = [torch.from_numpy(du_ref[:, c]).to(DEV) for c in range(3)]
    err = _triad_err(du, ref, (oz, oy, ox))
    g.close()
    print(f"810^3 {dtype} rhs vs triad oracle: {err:.3e} over {len(kout)} modes")
    assert err < tol


# --------------------------------------------------------------- dense FFT oracle
def test_rhs_810_matches_oracle_on_bench_field(bench_field, oracle810):
    uc = bench_field
    ref = oracle810.convectiondiffusion(uc, NU)
    errs = {}
    # FP32: the rounding of the product spectra is spread over all retained modes
    # and multiplied by |k| in the divergence, so the FP32 error of this RHS grows
    # with n (pocketfft's FP32 transforms: 7.0e-7 / 1.3e-6 / 2.8e-6 at n = 64 /
    # 128 / 256, about 9e-6 extrapolated to 810); measured here 1.02e-5
    for dtype, tol in ((torch.float32, 1.2e-5), (torch.float64, 1e-12)):
        g = S.Grid(3, N, dtype=dtype, device=DEV)
        u = _full_dev(uc, N, dtype)
        du = S.vectorfield(g)
        S.convectiondiffusion_(du, u, g, NU)
        del u
        got = [_compact_t(c, N) for c in du]
        del du
        g.close()
        torch.cuda.empty_cache()
        errs[dtype] = _rel(got, ref)
        print(f"810^3 {dtype} rhs vs oracle (bench field): {errs[dtype]:.3e}")
        assert errs[dtype] < tol


def test_rk4_810_fp32_matches_oracle(bench_field, oracle810):
    """One forced RK4 step of the production stepper (graph-captured, compact
    state, fused stage epilogues) against the oracle's RK4 step."""
    uc = bench_field
    ref = oracle810.rk4_step(uc, DT, NU, EPS)
    g = S.Grid(3, N, dtype=torch.float32, device=DEV)
    st = S.State(g)
    u = _full_dev(uc, N, torch.float32)
    st.load(u)
    st.rk4(DT, NU, 1, EPS)
    st.store(u)
    got = [_compact_t(c, N) for c in u]
    del u
    g.close()
    torch.cuda.empty_cache()
    e_state = _rel(got, ref)
    e_inc = _rel([a - b for a, b in zip(got, uc)], [a - b for a, b in zip(ref, uc)])
    print(f"810^3 fp32 RK4 step vs oracle: state {e_state:.3e}, increment {e_inc:.3e}")
    assert e_state < 2e-5
    assert e_inc < 1e-4


def test_sfs_810_fp32_matches_oracle(bench_field, oracle810):
    """sfs! 810^3 -> 128^3 at Delta/h in {2, 4, 8} (the DNS filtering workload)."""
    uc = bench_field
    nl = 128
    h = 2 * math.pi / nl
    deltas = [2 * h, 4 * h, 8 * h]
    ref = oracle810.sfs(uc, nl, deltas)
    gd = S.Grid(3, N, dtype=torch.float32, device=DEV)
    gl = S.Grid(3, nl, dtype=torch.float32, device=DEV)
    u = _full_dev(uc, N, torch.float32)
    ub = [S.vectorfield(gl) for _ in deltas]
    ta = [S.tensorfield(gl) for _ in deltas]
    S.sfs_(ub, ta, u, gd, gl, deltas)
    for b, t, (rb, rt, scale) in zip(ub, ta, ref):
        eb = _rel([c.to(torch.complex128).cpu().numpy() for c in b], rb)
        et = math.sqrt(sum(float(np.sum(np.abs(x.to(torch.complex128).cpu().numpy() - y) ** 2))
                           for x, y in zip(t, rt))) / scale
        print(f"810^3 -> 128^3 sfs fp32: ubar {eb:.3e}, tau {et:.3e} of the cancelled products")
        assert eb < 1e-6
        assert et < 1e-5
    gd.close()
    gl.close()


def test_every_810_sweep_variant_matches_triad_oracle():
    """Every kernel variant the autotuner may pick at 810 (column tiles 8 / 4 /
    16, the 30 x 27 split, the three TMA-fed column sweeps, the four x-sweep
    kernels) computes the same FP32 right-hand side, pinned to the exact triad
    oracle."""
    from symcode import autotune as A
    k, u = T.random_sparse_field(N, 200, 23, extra=EDGES)
    kout, du_ref = T.convectiondiffusion(k, u, N, NU)
    g = S.Grid(3, N, dtype=torch.float32, device=DEV)
    kf, uf = T.full_modes(k, u)
    m = kf[:, 0] >= 0
    iz, iy, ix = (torch.from_numpy(a).to(DEV) for a in T.to_rfft_index(kf[m], N))
    uin = []
    for c in range(3):
        t = torch.zeros(g.spec_shape, dtype=g.cdtype, device=DEV)
        t[iz, iy, ix] = torch.from_numpy(uf[m][:, c]).to(g.cdtype).to(DEV)
        uin.append(t)
    oz, oy, ox = (torch.from_numpy(a).to(DEV) for a in T.to_rfft_index(kout, N))
    ref = [torch.from_numpy(du_ref[:, c]).to(DEV) for c in range(3)]
    counts = A.num_variants(g)
    assert counts == [4, 7, 4, 7, 7]
    du = S.vectorfield(g)
    for s, name in enumerate(A.SWEEPS):
        for v in range(counts[s]):
            A.set_variants(g, {nm: (v if nm == name else 0) for nm in A.SWEEPS})
            S.convectiondiffusion_(du, uin, g, NU)
            err = _triad_err(du, ref, (oz, oy, ox))
            print(f"{name} variant {v}: {err:.3e}")
            assert err < 1e-5, (name, v, err)
    # the three sweeps with TMA-fed variants on one configuration at once, with
    # no bounded wait run out
    for v in (4, 5, 6):
        A.set_variants(g, {"z_inverse": 0, "y_inverse": v, "x_sweep": 0, "y_forward": v, "z_forward": v})
        S.convectiondiffusion_(du, uin, g, NU)
        err = _triad_err(du, ref, (oz, oy, ox))
        print(f"TMA-fed column sweeps, variant {v}: {err:.3e}")
        assert err < 1e-5
    assert S.plan_status(g) == 0
    g.close()


def test_tma_sweep_wait_limit_reports_timeout_and_recovers():
    """SC_OPT_WAIT_LIMIT = 0 makes the first mbarrier wait of every CTA of the
    TMA-fed column sweeps give up at once: the CTA records the timeout, waits
    (with the default bound) for its copies in flight and returns, nothing
    hangs or faults, sc_plan_status reports SC_ERR_TIMEOUT once, and the next
    evaluation with the default bound is exact again."""
    from symcode import autotune as A
    from symcode._lib import SC_ERR_TIMEOUT, SC_OPT_WAIT_LIMIT
    k, u = T.random_sparse_field(N, 60, 29, extra=EDGES)
    kout, du_ref = T.convectiondiffusion(k, u, N, NU)
    g = S.Grid(3, N, dtype=torch.float32, device=DEV)
    kf, uf = T.full_modes(k, u)
    m = kf[:, 0] >= 0
    iz, iy, ix = (torch.from_numpy(a).to(DEV) for a in T.to_rfft_index(kf[m], N))
    uin = []
    for c in range(3):
        t = torch.zeros(g.spec_shape, dtype=g.cdtype, device=DEV)
        t[iz, iy, ix] = torch.from_numpy(uf[m][:, c]).to(g.cdtype).to(DEV)
        uin.append(t)
    oz, oy, ox = (torch.from_numpy(a).to(DEV) for a in T.to_rfft_index(kout, N))
    ref = [torch.from_numpy(du_ref[:, c]).to(DEV) for c in range(3)]
    A.set_variants(g, {"y_inverse": 4, "y_forward": 4, "z_forward": 4})
    good = S.vectorfield(g)
    S.convectiondiffusion_(good, uin, g, NU)
    # the FP32 floor at 810 (about 1e-5, growing like n; the bench field's bar)
    assert _triad_err(good, ref, (oz, oy, ox)) < 1.2e-5
    assert S.plan_status(g) == 0
    du = S.vectorfield(g)
    S.set_option(g, SC_OPT_WAIT_LIMIT, 0)
    S.convectiondiffusion_(du, uin, g, NU)
    torch.cuda.synchronize()
    assert S.plan_status(g) == SC_ERR_TIMEOUT
    assert S.plan_status(g) == 0  # reading cleared the record
    S.set_option(g, SC_OPT_WAIT_LIMIT, -1)
    S.convectiondiffusion_(du, uin, g, NU)
    assert S.plan_status(g) == 0
    for a, b in zip(du, good):  # the same deterministic launches as before the timeout
        assert torch.equal(a, b)
    g.close()


def test_autotune_picks_the_fastest_measured_variant(tmp_path):
    from symcode import autotune as A
    g = S.Grid(3, N, dtype=torch.float32, device=DEV)
    st = S.State(g)
    # any state: the timing does not depend on the field
    st.load([torch.zeros(g.spec_shape, dtype=g.cdtype, device=DEV) for _ in range(3)])
    cache = str(tmp_path / "tune.json")
    rep = A.tune(g, visc=NU, reps=2, cache=cache)
    assert rep["source"] == "timed"
    counts = A.num_variants(g)
    timings = {int(v): t for v, t in rep["ms"].items()}
    for s, name in enumerate(A.SWEEPS):
        best = min(range(counts[s]), key=lambda v: (timings[v][name], v))
        assert rep["variants"][name] == best
    # a second plan of the same shape takes the cached choice without timing
    rep2 = A.tune(g, visc=NU, cache=cache)
    assert rep2["source"] == "cache" and rep2["variants"] == rep["variants"]
    g.close()

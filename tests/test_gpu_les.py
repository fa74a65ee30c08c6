"""LES closures and les! through the C ABI against the FP64 oracle."""

import math

import numpy as np
import pytest
import torch

import oracle as O
import symcode as S
from _util import rel_l2, to_dev, to_np

pytestmark = pytest.mark.gpu

TOL64 = 1e-12

KINDS = ["clark", "smagorinsky", "verstappen", "dynsmag", "bardina"]


def _models(kind, delta, g, D):
    """(CUDA closure, oracle model(u, G) -> packed tau)."""
    if kind == "clark":
        return S.create_clark(delta, g), lambda u, G, go: O.clark(G, delta, D)
    if kind == "smagorinsky":
        return S.create_smagorinsky(0.17, delta, g), lambda u, G, go: O.smagorinsky(G, 0.17, delta, D)
    if kind == "verstappen":
        return S.create_verstappen(0.3, delta, g), lambda u, G, go: O.verstappen(G, 0.3, delta, D)
    if kind == "dynsmag":
        return S.create_dynamic_smagorinsky(delta, g), lambda u, G, go: O.dynamic_smagorinsky(u, delta, go)
    return S.create_bardina(2.0, delta, g), lambda u, G, go: O.bardina(u, 2.0, delta, go)


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("D,n", [(3, 24), (2, 48)])
def test_les_rhs_matches_oracle(kind, D, n):
    if kind == "verstappen" and D == 2:
        pytest.skip("Q-R model is only defined in 3D")
    g = S.Grid(D, n, dtype=torch.float64, device="cuda:0")
    go = O.Grid(D, n)
    u = O.random_field(go, seed=21, kpeak=3)
    delta = 2 * go.l / n
    cl, ref_model = _models(kind, delta, g, D)
    ref = [O.twothirds(c, go) for c in O.les_rhs(u, go, lambda uu, GG: ref_model(uu, GG, go), 1e-3)]
    du = S.vectorfield(g)
    S.les_(du, [to_dev(c, g) for c in u], g, cl, 1e-3)
    assert rel_l2([to_np(c) for c in du], ref) < TOL64
    # the closure protocol model(u, G) itself
    GG = O.physical_gradient(u, go)
    tau_ref = ref_model(u, GG, go)
    names = "xyz"[:D]
    order = [names[a] + names[b] for b in range(D) for a in range(D)]  # G[a + D b]
    Gt = [to_dev(GG[k], g) for k in order]
    tau = cl([to_dev(c, g) for c in u], Gt)
    assert rel_l2(to_np(tau), tau_ref) < 1e-11


def test_les_rhs_no_closure_is_convectiondiffusion():
    g = S.Grid(3, 16, dtype=torch.float64, device="cuda:0")
    go = O.Grid(3, 16)
    u = O.random_field(go, seed=2, kpeak=3)
    du = S.vectorfield(g)
    S.les_(du, [to_dev(c, g) for c in u], g, None, 1e-2)
    ref = [O.twothirds(c, go) for c in O.convectiondiffusion(u, go, 1e-2)]
    assert rel_l2([to_np(c) for c in du], ref) < TOL64


@pytest.mark.parametrize("kind", ["clark", "dynsmag"])
def test_les_wray3_matches_oracle(kind):
    g = S.Grid(3, 24, dtype=torch.float64, device="cuda:0")
    go = O.Grid(3, 24)
    u = O.random_field(go, seed=5, kpeak=3)
    delta = 4 * go.l / 24
    cl, ref_model = _models(kind, delta, g, 3)
    f = lambda uu, gg, visc: O.les_rhs(uu, gg, lambda a, b: ref_model(a, b, gg), visc)  # noqa: E731
    ref = [O.twothirds(c, go) for c in O.wray3(f, u, 0.01, go, visc=2e-3)]
    ut = [to_dev(c, g) for c in u]
    S.les_wray3_(ut, 0.01, g, cl, 2e-3)
    assert rel_l2([to_np(c) for c in ut], ref) < TOL64


def test_les_rk4_fp32_dynsmag():
    g = S.Grid(3, 32, dtype=torch.float32, device="cuda:0")
    go = O.Grid(3, 32)
    u = O.random_field(go, seed=6, kpeak=3)
    delta = 2 * go.l / 32
    cl = S.create_dynamic_smagorinsky(delta, g)
    model = lambda uu, gg: O.dynamic_smagorinsky(uu, delta, go)  # noqa: E731
    ref = u
    for _ in range(2):
        def rhs(v):
            d = O.les_rhs(v, go, model, 1e-3)
            return O.project([O.twothirds(c, go) for c in d], go)
        k1 = rhs(ref)
        k2 = rhs([a + 0.005 * b for a, b in zip(ref, k1)])
        k3 = rhs([a + 0.005 * b for a, b in zip(ref, k2)])
        k4 = rhs([a + 0.01 * b for a, b in zip(ref, k3)])
        ref = [a + 0.01 / 6 * (b + 2 * c + 2 * d + e) for a, b, c, d, e in zip(ref, k1, k2, k3, k4)]
    ut = [to_dev(c, g) for c in u]
    S.les_rk4_(ut, 0.01, g, cl, 1e-3, nsteps=2)
    assert rel_l2([to_np(c) for c in ut], ref) < 2e-5


def test_closure_rejects_bad_arguments():
    g2 = S.Grid(2, 16, dtype=torch.float64, device="cuda:0")
    with pytest.raises(S.SymcodeError):
        S.create_verstappen(0.3, 0.1, g2)  # test/test_closures.jl:56-59
    with pytest.raises(S.SymcodeError):
        S.create_clark(-1.0, g2)


def test_les_batch_matches_single_instances_and_guard():
    """Three heterogeneous instances in one graph equal the same instances run one
    by one; a blown-up instance is flagged and frozen without stopping the others."""
    n = 32
    go = O.Grid(3, n)
    specs = [(1e-3, "dynsmag", 2, 0.1), (6e-4, "clark", 4, None), (3e-4, "smagorinsky", 2, 0.1),
             (1e-3, "clark", 2, None)]
    fields = [O.random_field(go, seed=30 + i, kpeak=3) for i in range(len(specs))]
    fields[3] = [c * 2e3 for c in fields[3]]  # energy far above the 1e5 blow-up limit
    ref = []
    for (nu, kind, dh, eps), u in zip(specs, fields):
        g = S.Grid(3, n, dtype=torch.float32, device="cuda:0")
        cl, _ = _models(kind, dh * go.l / n, g, 3)
        st = S.State(g)
        st.load([to_dev(c, g) for c in u])
        st.les_rk4(cl, 2e-3, nu, nsteps=3, eps=eps)
        out = S.vectorfield(g)
        st.store(out)
        ref.append([to_np(c) for c in out])
    grids, insts = [], []
    for (nu, kind, dh, eps), u in zip(specs, fields):
        g = S.Grid(3, n, dtype=torch.float32, device="cuda:0")
        cl, _ = _models(kind, dh * go.l / n, g, 3)
        S.State(g).load([to_dev(c, g) for c in u])
        grids.append((g, cl))
        insts.append(dict(grid=g, closure=cl, visc=nu, dt=2e-3, eps=eps))
    b = S.LesBatch(insts)
    b.run(3)
    status, energy = b.status(freeze=True)
    assert status[:3] == [0, 0, 0] and status[3] != 0
    for i in range(3):
        g = grids[i][0]
        out = S.vectorfield(g)
        S.State(g).store(out)
        assert rel_l2([to_np(c) for c in out], ref[i]) < 1e-6
    b.run(2)  # the frozen instance no longer advances; the others keep going
    status2, _ = b.status()
    assert status2[:3] == [0, 0, 0]


@pytest.mark.parametrize("kind", [None, "clark", "smagorinsky", "dynsmag"])
def test_les_diagnostics_match_oracle(kind):
    """reduce! of solve_les! (src/les.jl:94-148): e_post, ke, eps_visc, spectrum,
    eps_sfs and the shell transfer, against the physical-space oracle."""
    D, n, visc = 3, 32, 1e-3
    g, go = S.Grid(D, n, dtype=torch.float64, device="cuda:0"), O.Grid(D, n)
    u = [O.twothirds(c, go) for c in O.random_field(go, seed=31, kpeak=3)]
    uref = O.random_field(go, seed=32, kpeak=3)
    delta = 2 * go.l / n
    if kind is None:
        cl, model = None, None
    else:
        cl, m = _models(kind, delta, g, D)
        model = lambda uu, GG: m(uu, GG, go)  # noqa: E731
    ref = O.les_aposteriori(u, uref, go, model, visc)
    got = S.les_diagnostics([to_dev(c, g) for c in u], g, cl, [to_dev(c, g) for c in uref], visc)
    for k in ("e_post", "ke", "eps_visc"):
        assert math.isclose(got[k], ref[k], rel_tol=1e-11), k
    assert np.allclose(got["spectrum"], ref["spectrum"], rtol=1e-11, atol=1e-300)
    if kind is None:
        assert got["eps_sfs"] == 0 and not any(got["transfer"])
    else:
        assert math.isclose(got["eps_sfs"], ref["eps_sfs"], rel_tol=1e-9), (got["eps_sfs"], ref["eps_sfs"])
        t, tr = np.array(got["transfer"]), np.array(ref["transfer"])
        assert np.linalg.norm(t - tr) <= 1e-9 * np.linalg.norm(tr)


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-11), (torch.float32, 2e-5)])
@pytest.mark.parametrize("widths,redelta", [([9, 16, 12, 6], False), ([10, 8, 6], True)])
def test_mlp_closure_matches_oracle(dtype, tol, widths, redelta):
    """fullchain(mlp) (src/nets.jl:311-331): model(u, G) and les! against the oracle."""
    D, n, visc = 3, 32, 1e-3
    g, go = S.Grid(D, n, dtype=dtype, device="cuda:0"), O.Grid(D, n)
    u = O.random_field(go, seed=33, kpeak=3)
    delta = 2 * go.l / n
    rng = np.random.default_rng(34)
    ws = [rng.standard_normal((widths[l + 1], widths[l])) / np.sqrt(widths[l]) for l in range(len(widths) - 1)]
    bs = [0.1 * rng.standard_normal(widths[l + 1]) for l in range(len(widths) - 2)] + [None]
    cl = S.create_mlp_closure(delta, visc, g, ws, bs, use_redelta=redelta, mu=2.0, sigma=1.5)
    eps = np.finfo(np.float32 if dtype == torch.float32 else np.float64).eps
    model = lambda uu, GG: O.mlp_fullchain(GG, delta, visc, ws, bs, D, redelta, 2.0, 1.5, eps)  # noqa: E731
    GG = O.physical_gradient(u, go)
    names = "xyz"[:D]
    Gt = [to_dev(GG[names[a] + names[b]], g) for b in range(D) for a in range(D)]
    tau = cl([to_dev(c, g) for c in u], Gt)
    assert rel_l2(to_np(tau), model(u, GG)) < tol
    ref = [O.twothirds(c, go) for c in O.les_rhs(u, go, model, visc)]
    du = S.vectorfield(g)
    S.les_(du, [to_dev(c, g) for c in u], g, cl, visc)
    assert rel_l2([to_np(c) for c in du], ref) < tol
    assert S.closure_num_params(cl) == sum(w.size for w in ws) + sum(b.size for b in bs if b is not None)


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-11), (torch.float32, 5e-5)])
@pytest.mark.parametrize("D,redelta", [(3, False), (3, True), (2, False)])
def test_tbnn_closure_matches_oracle(dtype, tol, D, redelta):
    """tbnn (src/nets.jl:560-588) with the tensor basis of tb_kernel!: model(u, G) and les!."""
    n, visc = (32 if D == 3 else 64), 1e-3
    g, go = S.Grid(D, n, dtype=dtype, device="cuda:0"), O.Grid(D, n)
    u = O.random_field(go, seed=35, kpeak=3)
    delta = 2 * go.l / n
    nin, nb = (5, 7) if D == 3 else (2, 2)
    widths = [nin + int(redelta), 12, 10, nb]
    rng = np.random.default_rng(36)
    ws = [rng.standard_normal((widths[l + 1], widths[l])) / np.sqrt(widths[l]) for l in range(len(widths) - 1)]
    bs = [0.1 * rng.standard_normal(widths[l + 1]) for l in range(len(widths) - 2)] + [None]
    cl = S.create_tbnn_closure(delta, visc, g, ws, bs, use_redelta=redelta, mu=2.0, sigma=1.5)
    eps = np.finfo(np.float32 if dtype == torch.float32 else np.float64).eps
    model = lambda uu, GG: O.tbnn(GG, delta, visc, ws, bs, D, redelta, 2.0, 1.5, eps)  # noqa: E731
    GG = O.physical_gradient(u, go)
    names = "xyz"[:D]
    Gt = [to_dev(GG[names[a] + names[b]], g) for b in range(D) for a in range(D)]
    tau = cl([to_dev(c, g) for c in u], Gt)
    assert rel_l2(to_np(tau), model(u, GG)) < tol
    ref = [O.twothirds(c, go) for c in O.les_rhs(u, go, model, visc)]
    du = S.vectorfield(g)
    S.les_(du, [to_dev(c, g) for c in u], g, cl, visc)
    assert rel_l2([to_np(c) for c in du], ref) < tol


def test_les_batch_snapshot_reductions_match_per_snapshot_diagnostics():
    """reduce! fused into the batched stepper (src/les.jl:94-148): the device
    record of every second step equals sc_les_diagnostics called on the same
    states between the steps (FP64, several closure kinds and none)."""
    n, dt, nshell, every, nsnap = 32, 2e-3, 10, 2, 3
    go = O.Grid(3, n)
    specs = [(1e-3, "dynsmag", 2), (6e-4, "clark", 4), (1e-3, None, 2), (3e-4, "smagorinsky", 2)]
    fields = [O.random_field(go, seed=50 + i, kpeak=3) for i in range(len(specs))]

    def make():
        out = []
        for (nu, kind, dh), u in zip(specs, fields):
            g = S.Grid(3, n, dtype=torch.float64, device="cuda:0")
            cl = _models(kind, dh * go.l / n, g, 3)[0] if kind else None
            S.State(g).load([to_dev(c, g) for c in u])
            out.append(dict(grid=g, closure=cl, visc=nu, dt=dt, eps=None))
        return out

    insts = make()
    b = S.LesBatch(insts)
    b.set_snapshots(every, nshell, nsnap)
    b.run(every * nsnap + 1)  # one step past the last snapshot: no fourth record
    rec = b.snapshots()
    assert len(rec) == nsnap and len(rec[0]) == len(specs)

    singles = make()
    for s in range(nsnap):
        for i, d in enumerate(singles):
            st = S.State(d["grid"])
            st.les_rk4(d["closure"], dt, d["visc"], nsteps=every)
            u = S.vectorfield(d["grid"])
            st.store(u)
            ref = S.les_diagnostics(u, d["grid"], d["closure"], None, d["visc"], nshell)
            got = rec[s][i]
            for k in ("ke", "eps_visc"):
                assert math.isclose(got[k], ref[k], rel_tol=1e-10), (s, i, k, got[k], ref[k])
            assert np.allclose(got["spectrum"], ref["spectrum"], rtol=1e-10, atol=1e-300)
            if d["closure"] is None:
                assert got["eps_sfs"] == 0 and not np.any(got["transfer"])
            else:
                assert math.isclose(got["eps_sfs"], ref["eps_sfs"], rel_tol=1e-9), (s, i)
                t, tr = got["transfer"], np.array(ref["transfer"])
                assert np.linalg.norm(t - tr) <= 1e-9 * np.linalg.norm(tr)
    b.set_snapshots(0, 0, 0)  # off again
    b.close()


def test_les_batch_with_cnn_matches_oracle():
    """The batch of the 12-instance LES configuration in miniature: a tensor-core
    CNN instance and a dynamic Smagorinsky instance at 64^3 (FP32) advance in one
    graph; after one RK4 step each state is compared with the FP64 oracle's RK4
    step of les! with the same closure (the CNN with BF16 rounding emulated)."""
    n, dt = 64, 5e-3
    go = O.Grid(3, n)
    ws, bs = S.kaiming_cnn_weights(3)
    specs = [(6e-4, "cnn", 4), (1e-3, "dynsmag", 2)]
    fields = [O.random_field(go, seed=70 + i, kpeak=4) for i in range(len(specs))]
    insts, oracles = [], []
    for (nu, kind, dh), u in zip(specs, fields):
        g = S.Grid(3, n, dtype=torch.float32, device="cuda:0")
        delta = dh * go.l / n
        if kind == "cnn":
            cl = S.create_cnn_closure(delta, nu, g, ws, bs, mu=5.0, sigma=2.0)

            def model(uu, GG, delta=delta, nu=nu):
                uphys = np.stack([O.to_phys(O.twothirds(c, go), go) for c in uu], 0)
                z = O.cnn_redelta_channel(uu, go, delta, nu, mu=5.0, sigma=2.0)
                return O.cnn_field(uphys, z, ws, bs)
        else:
            cl = S.create_dynamic_smagorinsky(delta, g)

            def model(uu, GG, delta=delta):
                return O.dynamic_smagorinsky(uu, delta, go)
        S.State(g).load([to_dev(c, g) for c in u])
        insts.append(dict(grid=g, closure=cl, visc=nu, dt=dt, eps=None))
        oracles.append((model, nu))
    b = S.LesBatch(insts)
    b.run(1)
    status, _ = b.status()
    assert status == [0, 0]
    for d, (model, nu), u, spec in zip(insts, oracles, fields, specs):
        def rhs(v):
            return O.project([O.twothirds(c, go) for c in O.les_rhs(v, go, model, nu)], go)
        k1 = rhs(u)
        k2 = rhs([a + 0.5 * dt * c for a, c in zip(u, k1)])
        k3 = rhs([a + 0.5 * dt * c for a, c in zip(u, k2)])
        k4 = rhs([a + dt * c for a, c in zip(u, k3)])
        ref = [a + dt / 6 * (p + 2 * q + 2 * r + s) for a, p, q, r, s in zip(u, k1, k2, k3, k4)]
        out = S.vectorfield(d["grid"])
        S.State(d["grid"]).store(out)
        got = [to_np(c) for c in out]
        e_state = rel_l2(got, ref)
        e_inc = rel_l2([a - c for a, c in zip(got, u)], [a - c for a, c in zip(ref, u)])
        print(f"{spec[1]}: state {e_state:.2e}, increment {e_inc:.2e}")
        if spec[1] == "cnn":
            # BF16 weights and activations and the hardware tanh of the tensor-core
            # closure (its own output matches the BF16 oracle within 5e-3)
            assert e_state < 2e-4 and e_inc < 1e-2
        else:
            assert e_state < 2e-5 and e_inc < 2e-3
    b.close()

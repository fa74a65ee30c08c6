"""The CNN oracle's windowed evaluation equals a full periodic evaluation (CPU)."""

import numpy as np

import oracle as O


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, -2.5, 3.14159])
    r = O.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -7 and r[3] == -2.5
    assert abs(r[4] - 3.140625) < 1e-12


def test_cnn_rows_window_matches_full_grid():
    n = 12
    rng = np.random.default_rng(0)
    u = rng.standard_normal((3, n, n, n)) * 0.5
    layers = ((4, 5), (5, 5), (5, 5), (5, 6))
    ws = [rng.standard_normal((co, ci, 3, 3, 3)) * 0.2 for ci, co in layers]
    bs = [rng.standard_normal(co) * 0.1 for ci, co in layers]
    rows = [(3, 7), (0, 0), (11, 5)]
    got = O.cnn_rows(u, 0.3, ws, bs, rows)
    # full-grid evaluation with np.roll in every direction
    act = np.concatenate([O.bf16(u), np.full((1, n, n, n), O.bf16(np.array([0.3]))[0])], 0)
    for li, (w, b) in enumerate(zip(ws, bs)):
        wb = O.bf16(w)
        out = np.zeros((w.shape[0], n, n, n))
        for kz in range(3):
            for ky in range(3):
                for kx in range(3):
                    sh = np.roll(act, (-(kz - 1), -(ky - 1), -(kx - 1)), axis=(1, 2, 3))
                    out += np.einsum("oc,czyx->ozyx", wb[:, :, kz, ky, kx], sh)
        act = out + b[:, None, None, None]
        if li < 3:
            act = O.bf16(0.5 * act * (1 + np.tanh(np.sqrt(2 / np.pi) * (act + 0.044715 * act ** 3))))
    ref = np.stack([act[:, z, y, :] for (y, z) in rows], 1)
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12)


def test_cnn_field_equals_cnn_rows():
    """The whole-grid CNN oracle gives the row oracle's values on its rows."""
    import symcode as S
    n = 16
    rng = np.random.default_rng(0)
    uphys = rng.standard_normal((3, n, n, n))
    ws, bs = S.kaiming_cnn_weights(7)
    f = O.cnn_field(uphys, 0.3, ws, bs)
    rows = [(0, 0), (5, 7), (15, 3)]
    r = O.cnn_rows(uphys, 0.3, ws, bs, rows)
    assert np.array_equal(np.stack([f[:, z, y, :] for (y, z) in rows], 1), r)


def test_split_parts_carry_22_bits():
    """x = hi + lo with FP16 parts: |x - hi - lo| <= 2^-22 |x| while lo is a
    normal FP16 number (|x| >= 2^-3), else at most half the subnormal spacing
    2^-24.  The weights are stored x 64 to stay in the first range."""
    rng = np.random.default_rng(3)
    x = rng.standard_normal(10000) * 10.0 ** rng.uniform(-4, 3, 10000)
    hi, lo = O.split_parts(x)
    assert np.all(O.f16(hi) == hi) and np.all(O.f16(lo) == lo)
    assert np.all(np.abs(x - hi - lo) <= np.maximum(2.0 ** -22 * np.abs(x), 2.0 ** -25))
    big = np.abs(x) >= 2.0 ** -3
    assert np.max(np.abs(x - hi - lo)[big] / np.abs(x[big])) <= 2.0 ** -22


def test_split_network_sits_at_the_fp32_floor():
    """The split precision's roundings alone move tau by 1.5e-7 here, against
    4.6e-3 for one BF16 pass; the GPU's 2-3e-6 against FP64 is set by its FP32
    accumulation, not by the parts."""
    n = 16
    rng = np.random.default_rng(11)
    uphys = rng.standard_normal((3, n, n, n))
    ws, bs = [], []
    for cin, cout in ((4, 32), (32, 32), (32, 32), (32, 6)):
        ws.append(rng.standard_normal((cout, cin, 3, 3, 3)) * (2.0 / (27 * cin)) ** 0.5)
        bs.append(0.05 * np.arange(cout, dtype=np.float64))
    rows = [(0, 0), (5, 9), (15, 15)]
    ref = O.cnn_rows(uphys, 0.7, ws, bs, rows, round_bf16=False)
    split = O.cnn_rows_split(uphys, 0.7, ws, bs, rows)
    bf = O.cnn_rows(uphys, 0.7, ws, bs, rows)
    e_split = np.linalg.norm(split - ref) / np.linalg.norm(ref)
    e_bf = np.linalg.norm(bf - ref) / np.linalg.norm(ref)
    assert e_split < 1e-6
    assert e_bf > 1e-3 * 0.5 and e_split < 1e-3 * e_bf

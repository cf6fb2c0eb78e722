"""The oracle's restatement of the learned correction: its analytic gradient
against central finite differences (exact FP64 mode), and its feature rows
against an independent NumPy construction."""
from __future__ import annotations

import numpy as np

import oracle


def _net(seed):
    rng = np.random.default_rng(seed)
    w = (rng.standard_normal(oracle.lib().oracle_mlp_nparam()) * 0.3).astype(np.float32)
    w[:1024].reshape(32, 32)[:, 26:] = 0
    X = oracle.to_bf16(rng.uniform(-1, 1, (37, 32)).astype(np.float32))
    X[:, 26:] = 0
    t = rng.standard_normal(37).astype(np.float32)
    return w, X, t


def test_mlp_gradient_matches_finite_differences():
    w, X, t = _net(0)
    _, g = oracle.mlp_grad(w, X, t, round_bf16=False)
    rng = np.random.default_rng(1)
    idx = rng.choice(np.flatnonzero(np.abs(g) > 1e-4), 60, replace=False)
    for i in idx:
        h = 1e-4 * max(1.0, abs(float(w[i])))
        wp, wm = w.copy(), w.copy()
        wp[i] = np.float32(w[i] + h)
        wm[i] = np.float32(w[i] - h)
        lp, _ = oracle.mlp_grad(wp, X, t, False)
        lm, _ = oracle.mlp_grad(wm, X, t, False)
        fd = (lp - lm) / (float(wp[i]) - float(wm[i]))
        assert abs(fd - g[i]) <= 1e-6 * max(abs(g[i]), 1e-3), i


def test_mlp_loss_is_mean_square_error():
    w, X, t = _net(2)
    y = oracle.mlp_forward(w, X, round_bf16=True)
    loss, _ = oracle.mlp_grad(w, X, t, round_bf16=True)
    assert np.isclose(loss, np.mean((y - t) ** 2), rtol=1e-12)


def test_mlp_features_match_numpy():
    rng = np.random.default_rng(3)
    p = rng.standard_normal((20, 18, 16)).astype(np.float32)
    v2 = rng.uniform(1500, 4500, p.shape).astype(np.float32) ** 2
    z, y, x = 9, 8, 7
    c = (z * 18 + y) * 16 + x
    row, s = oracle.mlp_features(p, v2, c, np.float32(1e-3 / 10.0))
    star = [p[z, y, x]] + [p[z, y, x + r] for r in range(-4, 5) if r] + \
           [p[z, y + r, x] for r in range(-4, 5) if r] + [p[z + r, y, x] for r in range(-4, 5) if r]
    star = np.array(star, np.float32)
    m = np.abs(star).max()
    # s: the smallest power of two above max |star|
    assert s == 2.0 ** (np.floor(np.log2(m)) + 1) and s > m >= s / 2
    inv = np.float32(1.0) / np.float32(s)
    c0 = star[0]
    f = []
    axes = [star[1:9], star[9:17], star[17:25]]  # offsets -4..-1, 1..4
    for ax in axes:  # per axis and radius: difference, second difference
        for r in range(1, 5):
            f.append((ax[3 + r] - ax[4 - r]) * inv)
            f.append(((ax[3 + r] + ax[4 - r]) - np.float32(2) * c0) * inv)
    f.append(c0 * inv)
    assert np.array_equal(row[:25], oracle.to_bf16(np.array(f, np.float32)))
    assert row[25] == oracle.to_bf16(np.sqrt(v2[z, y, x]) * np.float32(1e-3 / 10.0))
    assert not row[26:].any()

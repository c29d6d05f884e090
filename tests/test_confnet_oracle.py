"""The confidence-net oracle's backward pass against central finite
differences of its own float64 forward (no bf16 rounding), and its AUC
helper against hand-computed cases. CPU only."""
import numpy as np

import confnet as cn


def test_oracle_gradient_matches_finite_differences():
    r = np.random.default_rng(0)
    x = r.integers(0, 256, (6, 128)).astype(np.uint8)
    y = r.integers(0, 2, 6)
    p = cn.init_params(1).astype(np.float64) + r.normal(0, 0.05, cn.N_PARAMS)
    _, g = cn.loss_and_grad(x, y, p, emulate=False)
    eps = 1e-6
    # every bias and conv1 weight, plus a sample of the rest
    idx = np.r_[np.arange(0, 192), np.arange(5312, 5344), np.arange(10464, 10496), np.arange(12544, 12673),
                r.choice(cn.N_PARAMS, 200, replace=False)]
    num = np.empty(idx.size)
    for k, i in enumerate(idx):
        q = p.copy()
        q[i] += eps
        lp, _ = cn.loss_and_grad(x, y, q, emulate=False)
        q[i] -= 2 * eps
        lm, _ = cn.loss_and_grad(x, y, q, emulate=False)
        num[k] = (lp - lm) / (2 * eps)
    assert np.abs(num - g[idx]).max() <= 1e-6 * max(1.0, np.abs(g[idx]).max())


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -3.0e-3, 0.0], np.float32)
    got = cn.bf16(v)
    # 1 + 2^-8 is a tie -> even (1.0); 1 + 1.5 * 2^-8 -> 1 + 2^-7
    np.testing.assert_array_equal(got[:4], [1.0, 1.0, 1.0078125, 1.0078125])
    assert got[5] == 0.0 and abs(got[4] + 3.0e-3) < 2e-5


def test_auc_hand_cases():
    assert cn.auc([0.1, 0.4, 0.35, 0.8], [1, 1, 0, 0]) == 0.75
    assert cn.auc([0, 0, 1, 1], [1, 1, 0, 0]) == 1.0
    assert cn.auc([1, 1, 1, 1], [1, 1, 0, 0]) == 0.5   # all ties
    assert cn.auc([0, 1, 0, 1], [1, 0, 0, 1]) == 0.5


def test_recenter_places_the_winner_at_64():
    c = np.arange(128, dtype=np.uint8)[None, :].repeat(3, 0)
    r = cn.recenter(c, np.array([0, 64, 127]))
    assert r[0, 64] == 0 and (r[0, :64] == 255).all() and r[0, 127] == 63
    np.testing.assert_array_equal(r[1], np.arange(128))
    assert r[2, 64] == 127 and (r[2, 65:] == 255).all() and r[2, 0] == 63

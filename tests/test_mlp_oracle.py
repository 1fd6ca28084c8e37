"""The CPU restatement of the level network (oracle/mlp_ref.py): its gradient
against central finite differences, and its BF16 rounding."""
import numpy as np

from oracle import mlp_ref as M


def _case(seed=0, n=40):
    rng = np.random.default_rng(seed)
    w = rng.normal(0, 0.3, M.N_PARAMS)
    feat = rng.normal(0, 1, (n, M.N_IN))
    lab = rng.integers(0, M.N_OUT, n)
    return w, np.zeros(M.N_IN), np.ones(M.N_IN), feat, lab


def test_gradient_matches_finite_differences():
    w, mu, sig, feat, lab = _case()
    _, g = M.loss_and_grad(w, mu, sig, feat, lab, round_bf16=False)
    rng = np.random.default_rng(1)
    for q in rng.choice(M.N_PARAMS, 60, replace=False):
        h = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[q] += h
        wm[q] -= h
        fd = (M.loss_and_grad(wp, mu, sig, feat, lab, round_bf16=False)[0] -
              M.loss_and_grad(wm, mu, sig, feat, lab, round_bf16=False)[0]) / (2 * h)
        assert abs(fd - g[q]) <= 1e-6 + 1e-5 * abs(g[q])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.001953125, 1.005859375, -3.14159265, 0.0], np.float32)
    r = M.bf16(x)
    # 1 + 2^-8 is halfway between 1 and 1 + 2^-7: ties to even -> 1
    assert r[0] == 1.0 and r[2] == 1.0
    assert r[1] == np.float32(1.0078125) or r[1] == 1.0
    assert abs(r[4] - (-3.140625)) < 1e-6
    assert np.all(M.bf16(r) == r)

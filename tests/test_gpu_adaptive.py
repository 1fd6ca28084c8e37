"""Adaptive IPM and its level network on the GPU.

* level 1 everywhere is the plain FP32 map, bit for bit (same corners, same
  triangles, fixed-point deposition);
* uniform refinement converges towards the level-16 (uniform-fine) map;
* the audit sends exactly the tiles whose level exceeds the tolerance to 16;
* the device gradients of the network match the FP64 CPU restatement
  (oracle/mlp_ref.py) with the same BF16 weights, within FP32 summation error;
* training learns a separable labelling;
* the trained network buys its accuracy with fewer cells than the uniform
  level that meets the same tolerance on every tile (the method without it).
"""
import numpy as np
import pytest

import irs_b200
from irs_b200.adaptive import LevelNet
from oracle import mlp_ref

pytestmark = pytest.mark.gpu

ADA = dict(kappa_tot=0.45, shear=0.4, smooth_fraction=0.5, mass_function="salpeter", m_lower=0.08, m_upper=1.0,
           theta_star=1.0, half_length_y1=4.0, half_length_y2=4.0, num_pixels_y1=128, num_pixels_y2=128,
           random_seed=4, write_histograms=0)
EPS = 1e-4


def _ada(**kw):
    a = irs_b200.AdaptiveIPM(**{**ADA, **kw})
    a.run()
    return a


def test_level1_equals_plain_map(gpu):
    a = _ada(policy="uniform", level=1, audit_fraction=0.0)
    p = irs_b200.IPM(**ADA)
    p.run()
    np.testing.assert_array_equal(a.magnifications, p.magnifications)
    assert a.value("cells_evaluated") == a.value("cells_base")


def test_tiled_and_pointwise_refinement_agree(gpu):
    # the tiled lens kernel over the level-s lattice and the point-by-point
    # evaluation compute each refined corner with the same arithmetic
    rng = np.random.default_rng(5)
    n = len(_ada(policy="uniform", level=1, audit_fraction=0.0).levels())
    lv = rng.choice([1, 2, 4, 8], n).astype(np.int32)
    a = _ada(policy="given", levels=lv, audit_fraction=0.0, tiled_min=1)
    b = _ada(policy="given", levels=lv, audit_fraction=0.0, tiled_min=1 << 30)
    mu_a, mu_b = a.magnifications.astype(np.float64), b.magnifications.astype(np.float64)
    assert np.abs(mu_a - mu_b).max() <= 1e-6 * mu_b.max()
    assert a.value("cells_evaluated") == b.value("cells_evaluated")


def test_uniform_refinement_converges(gpu):
    ref = _ada(policy="uniform", level=16, audit_fraction=0.0).magnifications.astype(np.float64)
    errs = []
    for lv in (1, 2, 4):
        mu = _ada(policy="uniform", level=lv, audit_fraction=0.0).magnifications.astype(np.float64)
        errs.append(np.abs(mu - ref).mean())
    assert errs[0] > errs[1] > errs[2]


def test_mixed_levels_between_their_uniform_bounds(gpu):
    a0 = _ada(policy="uniform", level=1, audit_fraction=0.0)
    n = len(a0.levels())
    rng = np.random.default_rng(3)
    lv = rng.choice([2, 4, 8], n).astype(np.int32)
    ref = _ada(policy="uniform", level=16, audit_fraction=0.0).magnifications.astype(np.float64)
    mixed = _ada(policy="given", levels=lv, audit_fraction=0.0)
    e_mixed = np.abs(mixed.magnifications - ref).mean()
    e2 = np.abs(_ada(policy="uniform", level=2, audit_fraction=0.0).magnifications - ref).mean()
    assert e_mixed < e2
    assert mixed.value("cells_evaluated") > 4 * mixed.value("cells_base")
    np.testing.assert_array_equal(mixed.levels(), lv)


def test_audit_sends_failing_tiles_to_level_16(gpu):
    a = _ada(policy="uniform", level=1, audit_fraction=1.0, tolerance=EPS)
    n = len(a.levels())
    lab, err = a.labels(np.arange(n))
    assert a.value("audited") == n
    assert a.value("audit_failures") == int(np.sum(lab > 0))
    np.testing.assert_array_equal(a.levels(), np.where(lab > 0, 16, 1))
    # interpolation errors shrink with the level
    assert np.mean(err[:, 3] <= err[:, 0] + 1e-6) > 0.95


def test_network_gradients_match_oracle(gpu):
    rng = np.random.default_rng(0)
    n = 300
    feat = rng.normal(0, 1, (n, 8)).astype(np.float32)
    lab = rng.integers(0, 5, n).astype(np.int32)
    net = LevelNet(rng.normal(0, 0.3, mlp_ref.N_PARAMS), rng.normal(0, 0.1, 8), rng.uniform(0.5, 2, 8))
    g, loss = net.gradients(feat, lab)
    loss_ref, g_ref = mlp_ref.loss_and_grad(net.w, net.mu, net.sig, feat, lab)
    assert abs(loss - loss_ref) <= 1e-5 * max(1.0, abs(loss_ref))
    np.testing.assert_allclose(g, g_ref, rtol=1e-3, atol=1e-5 * np.abs(g_ref).max())
    cls = net.predict(feat)
    np.testing.assert_array_equal(cls, mlp_ref.predict(net.w, net.mu, net.sig, feat))


def test_network_training_learns(gpu):
    rng = np.random.default_rng(1)
    feat = rng.normal(0, 1, (4000, 8)).astype(np.float32)
    lab = np.digitize(feat[:, 3] + 0.5 * feat[:, 6], [-1.0, -0.2, 0.4, 1.2]).astype(np.int32)
    net, loss = LevelNet.train(feat, lab, epochs=25, batch=256, lr=3e-3, seed=0)
    assert loss[-1] < 0.5 * loss[0]
    assert np.mean(net.predict(feat) == lab) > 0.9


# the learned-adaptive lens (Salpeter, kappa 0.6, shear 0.3, smooth 0.3) on a
# small map: much of its lattice lands off the source region
ADA_C5 = dict(kappa_tot=0.6, shear=0.3, smooth_fraction=0.3, mass_function="salpeter", m_lower=0.08, m_upper=1.0,
              theta_star=1.0, half_length_y1=6.0, half_length_y2=6.0, num_pixels_y1=128, num_pixels_y2=128,
              write_histograms=0)


def _training_set(seeds):
    F, Y = [], []
    for s in seeds:
        a = irs_b200.AdaptiveIPM(**{**ADA_C5, "random_seed": s}, policy="uniform", level=1, audit_fraction=0.0,
                                 tolerance=EPS)
        a.run()
        n = len(a.levels())
        lab, _ = a.labels(np.arange(n))
        F.append(a.features)
        Y.append(lab)
        a.close()
    return np.concatenate(F), np.concatenate(Y)


def test_network_gain_over_uniform_subdivision(gpu):
    """Cells the network's map needs against the uniform subdivision that
    reaches the same map error (both measured against the uniform-fine map of
    a star field the network has not seen)."""
    feat, lab = _training_set(range(11, 17))
    net, _ = LevelNet.train(feat, lab, epochs=40, batch=256, lr=3e-3, seed=0)
    held = {**ADA_C5, "random_seed": 21}

    def run(**kw):
        a = irs_b200.AdaptiveIPM(**held, tolerance=EPS, **kw)
        a.run()
        return a

    ref = run(policy="uniform", level=16, audit_fraction=0.0).magnifications.astype(np.float64)
    ok = ref > 0

    def med(mu):
        return np.median(np.abs(mu[ok] - ref[ok]) / ref[ok])

    a = run(policy="network", network=net, audit_fraction=0.05, audit_bound=1.0)  # the network's own choice
    e_net = med(a.magnifications)
    base = a.value("cells_base")
    match = 16
    for L in (1, 2, 4, 8):
        if med(run(policy="uniform", level=L, audit_fraction=0.0).magnifications) <= e_net:
            match = L
            break
    gain = base * match * match / a.value("cells_evaluated")
    print(f"network error {e_net:.2e}, matching uniform level {match}, gain {gain:.2f}, "
          f"audit {a.value('audit_failures'):.0f}/{a.value('audited'):.0f}")
    assert e_net < 1e-3
    assert gain > 1.2


def test_audit_escalates_above_the_bound(gpu):
    """When more of the audited tiles miss the tolerance than the bound allows,
    the level choice escalates (network quantile, then every tile finer): the
    final miss share is not above the network's and levels only grow; with a
    bound of 1 nothing escalates."""
    net = LevelNet.load()
    kw = dict(policy="network", network=net, audit_fraction=0.2, tolerance=EPS)
    a = _ada(**kw, audit_bound=1.0)
    b = _ada(**kw, audit_bound=0.0)
    assert a.value("escalation") == 0 and a.value("fail_rate") == a.value("fail_rate_initial")
    assert b.value("fail_rate_initial") == a.value("fail_rate_initial")
    if a.value("fail_rate_initial") > 0:
        assert b.value("escalation") > 0
        assert b.value("fail_rate") <= b.value("fail_rate_initial")
        assert np.all(b.levels() >= a.levels(predicted=True))

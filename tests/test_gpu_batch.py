"""Batches of realizations through the graph-captured pipeline.

Each realization's map must equal, bit for bit, a single run of the same
inputs at the same expansion order (FP32 form): the batch shares launches,
not arithmetic, and the deposition is fixed point. The cases vary the star
count, convergence, shear, smooth fraction and mass function, and force the
corner buffer to split realizations over several passes.
"""
import numpy as np
import pytest

import irs_b200

pytestmark = pytest.mark.gpu

BASE = dict(half_length_y1=2.5, half_length_y2=2.5, num_pixels_y1=72, num_pixels_y2=72, theta_star=1.0,
            light_loss=0.01, write_histograms=0)
REALIZATIONS = [
    dict(kappa_tot=0.3, shear=0.2, smooth_fraction=0.0, mass_function="equal", random_seed=1001),
    dict(kappa_tot=0.55, shear=0.35, smooth_fraction=0.5, mass_function="salpeter", m_lower=0.08, m_upper=1.0,
         random_seed=1002),
    dict(kappa_tot=0.8, shear=0.1, smooth_fraction=0.2, mass_function="kroupa", m_lower=0.01, m_upper=1.5,
         random_seed=1003),
    dict(kappa_tot=0.2, shear=0.6, smooth_fraction=0.8, mass_function="equal", random_seed=1004),
    dict(kappa_tot=0.45, shear=0.4, smooth_fraction=0.3, mass_function="salpeter", m_lower=0.08, m_upper=1.0,
         random_seed=1005),
]
ORDER = 10


def _cases():
    return [{**BASE, **r} for r in REALIZATIONS]


def _single(kw, dbl):
    extra = dict(precision=2) if dbl else {}
    m = irs_b200.IPM(**kw, is_double=dbl, expansion_order=ORDER, **extra)
    m.run()
    return m


@pytest.mark.parametrize("dbl", [False, True])
@pytest.mark.parametrize("corner_capacity", [0, 6000])
def test_batch_maps_equal_single_runs(gpu, dbl, corner_capacity):
    cases = _cases()
    b = irs_b200.BatchIPM(cases, is_double=dbl, expansion_order=ORDER, corner_capacity=corner_capacity)
    b.run()
    if corner_capacity:
        assert b.value("passes") > len(cases)
    maps = b.maps
    assert maps.shape == (len(cases), 72, 72)
    for r, kw in enumerate(cases):
        s = _single(kw, dbl)
        assert int(b.value("num_stars", r)) == s.value("num_stars")
        np.testing.assert_array_equal(b.stars(r), s.stars)
        np.testing.assert_array_equal(maps[r], s.magnifications)
        assert int(b.value("tree_levels", r)) == int(s.value("tree_levels"))
    # a replay of the captured graph reproduces the maps
    b.rerun(2)
    np.testing.assert_array_equal(b.maps, maps)


def test_batch_default_order_and_values(gpu):
    cases = _cases()[:3]
    b = irs_b200.BatchIPM(cases)
    b.run()
    assert 3 <= b.value("expansion_order") <= 31
    assert b.value("graph_nodes") > 10
    assert b.value("total_cells") == sum(b.value("num_cells", r) for r in range(3))
    mu = b.maps
    assert np.all(np.isfinite(mu)) and mu.mean() > 0

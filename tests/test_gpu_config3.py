"""The rectangular Kroupa configuration (8192^2 map, ~6.5e5 / 4.3e5 stars,
expansion order 16): kappa 0.7, shear 0.2, smooth fraction 0.1, Kroupa
0.01-1.5, theta_star 1, source half length 50, approximate smooth sheet (the
Taylor series of degree 39, alpha_smooth.cuh:62-127), IPM at one cell per
pixel (2.5e9 cells) and IRS at 64 rays per pixel (1.1e11 rays).

Whole maps of this size are timed by bench.py; here bands of the lattice
through its centre are checked:
  * IPM FP32 corner positions against the FP64 direct sum over all stars
    (oracle), on a seeded sample of 4000 corners of two cell rows: median
    within 1e-3 pixel, all within 0.05 pixel (pixels are 1/82 of the source
    unit; the FP32 form evaluates the leaf-relative near field, the far field
    and the folded smooth sheet in FP32);
  * the same corners from the FP64 plain form against the oracle: within the
    expansion error (median 1e-4 pixel);
  * IRS FP32 against the FP64 plain form (the float library's two forms, one
    star field) on four ray rows (5.1e5 rays received): at most 1e-3 of the
    rays land in another pixel.
"""
import numpy as np
import pytest

import irs_b200
from oracle import pyoracle as po
from tests.cases import lattice, oracle_lens, to_pixels

pytestmark = pytest.mark.gpu

C3 = dict(kappa_tot=0.7, shear=0.2, smooth_fraction=0.1, theta_star=1.0, mass_function="kroupa", m_lower=0.01,
          m_upper=1.5, rectangular=True, approx=True, half_length_y1=50.0, half_length_y2=50.0, num_pixels_y1=8192,
          num_pixels_y2=8192, random_seed=3, expansion_order=16, write_histograms=0)


def _band_vertices(dbl, rows=2):
    m = irs_b200.IPM(**C3, num_rays_y=1, is_double=dbl)
    m.derive()
    ny = int(m.value("num_ray_threads_2"))
    j0 = ny // 2
    m.lib.set_band(m.obj, j0, j0 + rows)
    m.run()
    return m, j0, m.vertices()


def _oracle(m, j0, jj, ii):
    x, _ = lattice(m, vertices=True)
    oy = m.value("center_x2") - m.value("half_length_x2")
    y = oy + 2.0 * (m.value("ray_half_sep_2") * (j0 + jj).astype(np.float64))
    wx, wy = po.shoot_direct(m.stars.astype(np.float64), oracle_lens(m), x[ii], y)
    return to_pixels(m, wx, wy)


def _corner_errors(dbl):
    m, j0, v = _band_vertices(dbl)
    try:
        rng = np.random.default_rng(0)
        jj = rng.integers(0, v.shape[0], 4000)
        ii = rng.integers(0, v.shape[1], 4000)
        px, py = _oracle(m, j0, jj, ii)
        got = v[jj, ii]
        return np.hypot(got[:, 0] - px, got[:, 1] - py)
    finally:
        m.close()


def test_config3_ipm_fp32_corners_vs_fp64_direct_sum(gpu):
    err = _corner_errors(False)
    print(f"config 3 FP32 corners vs FP64 direct sum: median {np.median(err):.2e} px, max {err.max():.2e} px")
    assert np.median(err) <= 1e-3
    assert err.max() <= 0.05


def test_config3_ipm_fp64_plain_corners_vs_fp64_direct_sum(gpu):
    err = _corner_errors(True)
    print(f"config 3 FP64 plain corners vs FP64 direct sum: median {np.median(err):.2e} px, max {err.max():.2e} px")
    assert np.median(err) <= 1e-4


def test_config3_irs_fp32_vs_fp64_plain_band(gpu):
    maps = []
    for prec in (1, 2):  # the FP64 plain and the FP32 form of the float library: the same star field
        r = irs_b200.IRS(**C3, num_rays_y=64, is_double=False, precision=prec)
        r.derive()
        ny = int(r.value("num_ray_threads_2"))
        r.lib.set_band(r.obj, ny // 2, ny // 2 + 4)
        r.run()
        maps.append(r.magnifications.astype(np.int64))
        r.close()
    moved = np.abs(maps[0] - maps[1]).sum() // 2
    print(f"config 3 IRS FP32 vs FP64 plain: {moved} of {maps[0].sum()} rays moved")
    assert maps[0].sum() > 0
    assert moved <= 1e-3 * maps[0].sum()

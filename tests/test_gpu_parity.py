"""GPU parity: the CUDA path through the C ABI against the CPU oracle on the
same star field.

Tolerances:
  * tree structure: exact (levels, centres, star sets, neighbour sets);
  * FMM coefficients (FP64 both sides): relative 1e-9 of the largest coefficient;
  * FP64 plain form: source positions within 1e-9 pixel of the oracle's FMM form
    (same expansion), IRS maps identical up to rays within rounding of a pixel
    edge (<= 2 rays);
  * smooth sheets: the approximate (default) and the exact forms, circular and
    rectangular fields, under the same bars;
  * FP32 form: source positions within 2e-3 pixel at the 99.9th percentile of
    the oracle's FMM form; IRS rays moved between pixels <= 1e-4 of those
    received; median relative magnification error vs the FP64 direct-sum
    oracle <= 1e-3;
  * IPM deposition: bit-exact fixed-point maps against the oracle's fixed-point
    deposition of the GPU's own vertex positions; within 1e-9 (FP64) of the
    reference polygon algorithm on the same vertices.
"""
import numpy as np
import pytest

import irs_b200
from oracle import pyoracle as po
from tests.cases import IPM_RECT, IPM_SMALL, IRS_SMALL, lattice, oracle_lens, to_pixels

pytestmark = pytest.mark.gpu


def _run(cls, cfg, dbl, **kw):
    m = cls(is_double=dbl, **cfg, **kw)
    m.run()
    return m


def _oracle_tree(m):
    return po.Tree(m.stars.astype(np.float64), m.value("root_half_length"), order=m.expansion_order)


@pytest.mark.parametrize("dbl", [True, False])
def test_tree_structure_and_coefficients(gpu, dbl):
    m = _run(irs_b200.IRS, IRS_SMALL, dbl, expansion_order=10)
    t = _oracle_tree(m)
    gi, gg, gn, gs, gd = m.tree_arrays()
    oi, og, on, os_, od = t.arrays()
    assert m.value("tree_levels") == t.levels
    assert gi.shape == oi.shape
    np.testing.assert_array_equal(gi, oi)
    if dbl:
        np.testing.assert_array_equal(gg, og)
    else:  # float objects build the tree in float, as lib_ipm.so does (centres differ by float rounding)
        np.testing.assert_allclose(gg, og, rtol=2e-7, atol=1e-6)
    for k in range(gi.shape[0]):
        assert list(gn[k, :gi[k, 5]]) == list(on[k, :oi[k, 5]])
        assert list(gs[k, :gi[k, 6]]) == list(os_[k, :oi[k, 6]])
        assert list(gd[k, :gi[k, 7]]) == list(od[k, :oi[k, 7]])
    np.testing.assert_array_equal(t.stars(), m.stars.astype(np.float64))
    gm, gl = m.coeffs()
    om, ol = t.coeffs()
    scale_m = np.abs(om).max()
    scale_l = np.abs(ol).max()
    tol = 1e-9 if dbl else 1e-6  # float objects carry float node centres into the FP64 expansions
    assert np.abs(gm - om).max() <= tol * scale_m
    assert np.abs(gl - ol).max() <= tol * scale_l


def test_tree_rebuild_after_node_overflow(gpu):
    """Four clusters of stars 1e-6 of the field radius across need about 3300
    tree nodes, more than the build reserves at first (1.5 per star + 1024):
    the build restores the star order, reserves twice as many and builds again.
    The tree must equal the oracle's exactly."""
    a = irs_b200.IRS(**IRS_SMALL, is_double=True)
    a.derive()
    n = int(a.value("num_stars"))
    R = float(np.hypot(a.value("corner_x1"), a.value("corner_x2")))
    rng = np.random.default_rng(5)
    ang = 2 * np.pi * rng.random(4)
    cen = R * 0.6 * np.sqrt(rng.random(4))[:, None] * np.stack([np.cos(ang), np.sin(ang)], 1)
    per = n // 4
    pts = np.concatenate([cen[i] + 1e-6 * R * rng.standard_normal((per, 2)) for i in range(4)] +
                         [R * 0.5 * (rng.random((n - 4 * per, 2)) - 0.5)])
    stars = np.concatenate([pts, np.ones((n, 1))], 1)
    b = irs_b200.IRS(**IRS_SMALL, is_double=True, safety_scale=1.3)
    b.set_stars(stars, rectangular=False, corner=(R, 0.0), theta_star=1.0)
    b.run()
    t = _oracle_tree(b)
    assert t.overflow == 0
    gi, gg, gn, gs, gd = b.tree_arrays()
    oi, og, on, os_, od = t.arrays()
    assert gi.shape[0] > 1.5 * n + 1024  # the first reservation was too small
    assert b.value("tree_levels") == t.levels
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(gg, og)
    for k in range(gi.shape[0]):
        assert list(gn[k, :gi[k, 5]]) == list(on[k, :oi[k, 5]])
        assert list(gs[k, :gi[k, 6]]) == list(os_[k, :oi[k, 6]])
        assert list(gd[k, :gi[k, 7]]) == list(od[k, :oi[k, 7]])
    np.testing.assert_array_equal(t.stars(), b.stars.astype(np.float64))
    assert np.isfinite(b.magnifications).all()


def _vertex_positions_oracle(m, t):
    x, y = lattice(m, vertices=True)
    X, Y = np.meshgrid(x, y)
    wx, wy = t.shoot(oracle_lens(m), X, Y)
    px, py = to_pixels(m, wx, wy)
    return np.stack([px, py], -1).reshape(len(y), len(x), 2)


EXACT = [dict(IPM_SMALL, approx=False), dict(IPM_RECT, approx=False)]  # exact smooth sheets (alpha_smooth.cuh:62-127)


@pytest.mark.parametrize("cfg", [IPM_SMALL, IPM_RECT] + EXACT, ids=["circle", "rect", "circle_exact", "rect_exact"])
def test_ipm_fp64_vertices_match_oracle(gpu, cfg):
    m = _run(irs_b200.IPM, cfg, True, expansion_order=12)
    t = _oracle_tree(m)
    v = m.vertices()
    o = _vertex_positions_oracle(m, t)
    assert v.shape == o.shape
    err = np.abs(v - o)
    assert np.nanmax(err) < 1e-8


@pytest.mark.parametrize("cfg", [IPM_SMALL, IPM_RECT] + EXACT, ids=["circle", "rect", "circle_exact", "rect_exact"])
def test_ipm_fp32_vertices_close_to_oracle(gpu, cfg):
    m = _run(irs_b200.IPM, cfg, False, expansion_order=12)
    t = _oracle_tree(m)
    v = m.vertices()
    o = _vertex_positions_oracle(m, t)
    err = np.hypot(*(v - o).transpose(2, 0, 1)).ravel()
    assert np.quantile(err, 0.999) < 2e-3
    assert np.median(err) < 1e-4


@pytest.mark.parametrize("dbl", [True, False])
@pytest.mark.parametrize("parities", [False, True])
def test_ipm_deposit_bit_exact(gpu, dbl, parities):
    m = _run(irs_b200.IPM, IPM_SMALL, dbl, expansion_order=12, write_parities=parities)
    v = m.vertices()
    rhs1, rhs2 = m.value("ray_half_sep_1"), m.value("ray_half_sep_2")
    npx, npy = m.num_pixels
    hx, hy = m.half_length
    if dbl:
        factor = 2 * rhs1 * rhs2 * npx * npy / (2 * hx * 2 * hy)
    else:
        f32 = np.float32
        factor = float(f32(f32(f32(f32(f32(2) * f32(rhs1)) * f32(rhs2)) * f32(npx)) * f32(npy))
                       / f32(f32(f32(f32(2) * f32(hx)) * f32(2)) * f32(hy)))
    got = m.fixed_maps()
    ref = po.ipm_deposit_fixed(v, factor, (npx, npy), parities=parities, single=not dbl)
    if parities:
        np.testing.assert_array_equal(got[0], ref[0])
        np.testing.assert_array_equal(got[1], ref[1])
        tot = po.fix_to_float(got[0] + got[1])
        np.testing.assert_allclose(m.magnifications, tot.astype(m.magnifications.dtype), rtol=0, atol=0)
    else:
        np.testing.assert_array_equal(got, ref)


def test_ipm_deposit_matches_reference_polygon_algorithm(gpu):
    m = _run(irs_b200.IPM, IPM_SMALL, True, expansion_order=12)
    v = m.vertices()
    rhs1, rhs2 = m.value("ray_half_sep_1"), m.value("ray_half_sep_2")
    npx, npy = m.num_pixels
    hx, hy = m.half_length
    factor = 2 * rhs1 * rhs2 * npx * npy / (2 * hx * 2 * hy)
    ref = po.ipm_deposit_ref(v, factor, (npx, npy))
    got = m.magnifications
    assert np.abs(got - ref).max() <= 1e-8 * max(1.0, np.abs(ref).max())


def test_ipm_deterministic(gpu):
    a = _run(irs_b200.IPM, IPM_SMALL, False, expansion_order=12)
    b = _run(irs_b200.IPM, IPM_SMALL, False, expansion_order=12)
    np.testing.assert_array_equal(a.magnifications, b.magnifications)
    np.testing.assert_array_equal(a.stars, b.stars)


def _irs_oracle_map(m, t, want_mu=False):
    x, y = lattice(m, vertices=False)
    X, Y = np.meshgrid(x, y)
    L = oracle_lens(m)
    if want_mu:
        wx, wy, mu = t.shoot(L, X, Y, want_mu=True)
    else:
        (wx, wy), mu = t.shoot(L, X, Y), None
    return po.irs_bin(wx, wy, m.center, m.half_length, m.num_pixels, mu=mu)


@pytest.mark.parametrize("approx", [True, False], ids=["approx_sheet", "exact_sheet"])
def test_irs_fp64_matches_oracle(gpu, approx):
    m = _run(irs_b200.IRS, dict(IRS_SMALL, approx=approx), True, expansion_order=10)
    t = _oracle_tree(m)
    ref = _irs_oracle_map(m, t)
    got = m.magnifications
    assert got.sum() == m.num_rays_received
    assert np.abs(got.astype(np.int64) - ref).sum() <= 2
    assert m.num_rays_shot == m.value("num_ray_threads_1") * m.value("num_ray_threads_2")


def test_irs_fp64_parities_match_oracle(gpu):
    m = _run(irs_b200.IRS, IRS_SMALL, True, expansion_order=10, write_parities=True)
    t = _oracle_tree(m)
    pix, pmin, psad = _irs_oracle_map(m, t, want_mu=True)
    assert np.abs(m.magnifications.astype(np.int64) - pix).sum() <= 2
    assert np.abs(m.magnifications_minima.astype(np.int64) - pmin).sum() <= 4
    assert np.abs(m.magnifications_saddles.astype(np.int64) - psad).sum() <= 4
    np.testing.assert_array_equal(m.magnifications, m.magnifications_minima + m.magnifications_saddles)


def test_irs_fp32_matches_fp64_same_expansion(gpu):
    a = _run(irs_b200.IRS, IRS_SMALL, False, expansion_order=10)
    b = _run(irs_b200.IRS, IRS_SMALL, True, expansion_order=10)
    moved = np.abs(a.magnifications.astype(np.int64) - b.magnifications).sum() / 2
    assert moved <= 2e-4 * b.num_rays_received  # ~2 x FP32 position error / pixel size


def test_irs_fp32_accuracy_vs_fp64_direct(gpu):
    m = _run(irs_b200.IRS, IRS_SMALL, False, expansion_order=16)
    x, y = lattice(m, vertices=False)
    X, Y = np.meshgrid(x, y)
    wx, wy = po.shoot_direct(m.stars.astype(np.float64), oracle_lens(m), X, Y)
    ref = po.irs_bin(wx, wy, m.center, m.half_length, m.num_pixels)
    got = m.magnifications.astype(np.int64)
    moved = np.abs(got - ref).sum() / 2
    assert moved <= 1e-4 * ref.sum()
    rel = np.abs(got - ref) / np.maximum(ref, 1)
    assert np.median(rel) <= 1e-3


def test_irs_deterministic_and_conserving(gpu):
    a = _run(irs_b200.IRS, IRS_SMALL, False, expansion_order=10)
    b = _run(irs_b200.IRS, IRS_SMALL, False, expansion_order=10)
    np.testing.assert_array_equal(a.magnifications, b.magnifications)
    assert a.num_rays_received == a.magnifications.sum()
    assert 0 < a.num_rays_received < a.num_rays_shot

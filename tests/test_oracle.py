"""The CPU oracle (a C restatement of the reference algorithm) pinned against
golden vectors produced by the reference's own code compiled for the host
(tests/golden/make_golden.py), and its internal consistency checks."""
import os

import numpy as np
import pytest

from oracle import pyoracle as po

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_small.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.fixture(scope="module")
def tree(gold):
    return po.Tree(gold["stars"], float(gold["root_hl"]), order=int(gold["order"]))


def lens_of(gold):
    k, g, ks, th = gold["lens"]
    return po.lens(k, g, ks, th)


def test_tree_matches_reference(gold, tree):
    assert tree.levels == int(gold["levels"])
    assert tree.n == int(gold["num_nodes"])
    ints, geom, *_ = tree.arrays()
    key = {(int(ints[k, 0]), geom[k, 0], geom[k, 1]): k for k in range(tree.n)}
    for lvl, (cx, cy, hl), ns, nch in zip(gold["node_level"], gold["node_geom"], gold["node_numstars"],
                                         gold["node_children"]):
        k = key[(int(lvl), cx, cy)]
        assert geom[k, 2] == hl
        assert ints[k, 4] == ns
        assert (ints[k, 2] >= 0) == (nch > 0)


def test_source_positions_match_reference(gold, tree):
    wx, wy = tree.shoot(lens_of(gold), gold["pts"][:, 0], gold["pts"][:, 1])
    assert np.abs(wx - gold["wx"]).max() < 1e-11
    assert np.abs(wy - gold["wy"]).max() < 1e-11


def _lattice(rhs, nrt, hlx, vertices):
    if vertices:
        x = -hlx[0] + 2.0 * (rhs * np.arange(nrt[0] + 1))
        y = -hlx[1] + 2.0 * (rhs * np.arange(nrt[1] + 1))
    else:
        x = (-hlx[0] + rhs) + 2.0 * (rhs * np.arange(nrt[0]))
        y = (-hlx[1] + rhs) + 2.0 * (rhs * np.arange(nrt[1]))
    return np.meshgrid(x, y)


def test_irs_map_matches_reference(gold, tree):
    X, Y = _lattice(float(gold["irs_rhs"]), gold["irs_nrt"], gold["irs_hlx"], False)
    wx, wy = tree.shoot(lens_of(gold), X, Y)
    h, n = float(gold["ipm_hly"]), int(gold["ipm_npix"])
    pix = po.irs_bin(wx, wy, (0.0, 0.0), (h, h), (n, n))
    assert np.abs(pix.astype(np.int64) - gold["irs_map"]).sum() <= 1


def test_ipm_map_matches_reference(gold, tree):
    rhs = float(gold["ipm_rhs"])
    X, Y = _lattice(rhs, gold["ipm_nrt"], gold["ipm_hlx"], True)
    wx, wy = tree.shoot(lens_of(gold), X, Y)
    wx, wy = wx.reshape(X.shape), wy.reshape(X.shape)
    h, n = float(gold["ipm_hly"]), int(gold["ipm_npix"])
    px = (wx + h) * n / (2 * h)
    py = n - (wy + h) * n / (2 * h)
    v = np.stack([px, py], -1)
    factor = 2 * rhs * rhs * n * n / (2 * h * 2 * h)
    mu = po.ipm_deposit_ref(v, factor, (n, n))
    ref = gold["ipm_map"]
    # The reference evaluates each cell's four corners on its own (z +- rhs),
    # the oracle evaluates the shared corner lattice: the corner positions
    # differ in the last bits, which cells next to a star amplify.
    rel = np.abs(mu - ref) / ref
    assert np.median(rel) < 1e-7
    assert np.quantile(rel, 0.99) < 2e-5
    assert rel.max() < 1e-3


def test_polygon_deposition_matches_reference(gold):
    mu = po.ipm_deposit_ref(gold["dep_verts"], float(gold["dep_factor"]), (24, 20))
    np.testing.assert_array_equal(mu, gold["dep_map"])


@pytest.mark.parametrize("single", [False, True])
def test_fixed_point_sweep_close_to_reference_deposition(gold, single):
    v = gold["dep_verts"]
    f = np.float32(gold["dep_factor"]) if single else float(gold["dep_factor"])
    q = po.fix_to_float(po.ipm_deposit_fixed(v, f, (24, 20), single=single))
    ref = gold["dep_map"]
    tol = 1e-4 if single else 1e-8
    assert np.abs(q - ref).max() <= tol * max(1.0, ref.max())


def test_fixed_point_conserves_area():
    # a lattice of cells entirely inside the map deposits exactly its area
    rng = np.random.default_rng(1)
    v = np.stack(np.meshgrid(np.linspace(5, 25, 21), np.linspace(4, 30, 27)), -1) + rng.normal(0, 0.2, (27, 21, 2))
    q = po.fix_to_float(po.ipm_deposit_fixed(v, 1.0, (40, 40), single=False))
    assert abs(q.sum() - 2 * 20 * 26) < 1e-6


@pytest.mark.parametrize("step", [1.0, 0.5, 2.0])
@pytest.mark.parametrize("single", [False, True])
def test_fixed_point_pixel_aligned_cells(step, single):
    # cell edges exactly on pixel lines (no deflection): an edge on the line
    # between two rows must be counted once
    v = np.stack(np.meshgrid(np.arange(5, 26, step), np.arange(4, 31, step)), -1)
    q = po.fix_to_float(po.ipm_deposit_fixed(v, 1.0, (40, 40), single=single))
    ref = po.ipm_deposit_ref(v, 1.0, (40, 40))
    np.testing.assert_array_equal(q, ref)


@pytest.mark.parametrize("order,tol", [(8, 5e-3), (16, 5e-6), (24, 5e-9)])
def test_expansion_converges_to_direct_sum(order, tol):
    rng = np.random.default_rng(0)
    n = 1500
    r = np.sqrt(rng.random(n)) * 30
    a = rng.random(n) * 2 * np.pi
    st = np.stack([r * np.cos(a), r * np.sin(a), rng.uniform(0.1, 1, n)], 1)
    L = po.lens(0.4, 0.3, 0.4, 1.0)
    zx, zy = rng.uniform(-15, 15, 5000), rng.uniform(-15, 15, 5000)
    d = po.shoot_direct(st, L, zx, zy)
    t = po.Tree(st, 33.0, order=order)
    f = t.shoot(L, zx, zy)
    assert np.hypot(f[0] - d[0], f[1] - d[1]).max() < tol


def test_irs_binning_edges():
    # clamp at the right / top edge and row flip (irs_functions.cuh:167-184)
    wx = np.array([-1.0, 1.0, 0.0, -1.0, 1.0000001])
    wy = np.array([-1.0, 1.0, 0.0, 0.999, 0.0])
    pix = po.irs_bin(wx, wy, (0.0, 0.0), (1.0, 1.0), (4, 4))
    assert pix.sum() == 4  # the last ray is outside
    assert pix[3, 0] == 1  # (-1, -1): bottom-left -> last row, first column
    assert pix[0, 3] == 1  # (1, 1) clamps into the top-right pixel
    assert pix[1, 2] == 1  # (0, 0)
    assert pix[0, 0] == 1  # (-1, 0.999)


@pytest.mark.skipif(not po.ref_available(), reason="reference host build not present")
def test_ref_host_build_matches_oracle_on_random_field():
    rng = np.random.default_rng(7)
    n = 900
    r = np.sqrt(rng.random(n)) * 25
    a = rng.random(n) * 2 * np.pi
    st = np.stack([r * np.cos(a), r * np.sin(a), rng.uniform(0.05, 2, n)], 1)
    L = po.lens(0.6, 0.2, 0.4, 1.2, rect=0, approx=0)
    t = po.Tree(st, 28.0, order=10)
    rt = po.RefTree(st, 28.0, order=10)
    assert (t.levels, t.n) == (rt.levels, rt.n)
    zx, zy = rng.uniform(-10, 10, 3000), rng.uniform(-10, 10, 3000)
    a1 = t.shoot(L, zx, zy)
    a2 = rt.points(L, zx, zy)
    assert np.abs(a1[0] - a2[0]).max() < 1e-11 and np.abs(a1[1] - a2[1]).max() < 1e-11

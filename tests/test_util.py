"""File helpers (irs_b200.util) against the layouts the map makers write and,
where the reference's own helper module has been built into oracle/_ref, against
that module on the same files (microlensing/Util/util.py:5-125)."""
import importlib.util
import os

import numpy as np
import pytest

from irs_b200 import util

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_UTIL = os.path.join(ROOT, "oracle", "_ref", "gpu", "microlensing", "Util", "util.py")


def _ref_util():
    if not os.path.exists(REF_UTIL):
        pytest.skip("the reference's helper module is not built (make -C oracle ref)")
    spec = importlib.util.spec_from_file_location("ref_util", REF_UTIL)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _field(dtype, rect, n=37, seed=4):
    rng = np.random.default_rng(seed)
    stars = np.column_stack([rng.uniform(-9, 9, n), rng.uniform(-9, 9, n), rng.uniform(0.08, 1, n)]).astype(dtype)
    corner = np.array([9.0, 7.5] if rect else [12.5, 0.0], dtype=dtype)
    return stars, corner


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("rect", [False, True])
def test_star_file_round_trip(tmp_path, dtype, rect):
    stars, corner = _field(dtype, rect)
    f = str(tmp_path / "s.bin")
    util.write_stars(f, len(stars), rect, corner, 1.5, stars, dtype=dtype)
    assert os.path.getsize(f) == 8 + np.dtype(dtype).itemsize * (3 + stars.size)
    s, r, c, t = util.read_stars(f, dtype=dtype)
    np.testing.assert_array_equal(s, stars)
    np.testing.assert_array_equal(c, corner)
    assert r == rect and t == dtype(1.5) and s.dtype == dtype


def test_star_file_rejections(tmp_path):
    stars, corner = _field(np.float32, False)
    with pytest.raises(ValueError):
        util.write_stars(str(tmp_path / "s.txt"), len(stars), False, corner, 1.0, stars)
    with pytest.raises(ValueError):
        util.write_stars(str(tmp_path / "s.bin"), len(stars), False, corner, 1.0, stars, dtype=np.int32)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("rect", [False, True])
def test_star_files_interchange_with_reference(tmp_path, dtype, rect):
    ref = _ref_util()
    stars, corner = _field(dtype, rect)
    mine, theirs = str(tmp_path / "mine.bin"), str(tmp_path / "ref.bin")
    util.write_stars(mine, len(stars), rect, corner, 1.0, stars, dtype=dtype)
    ref.write_stars(theirs, len(stars), rect, corner, 1.0, stars, dtype=dtype)
    assert open(mine, "rb").read() == open(theirs, "rb").read()
    a, b = util.read_stars(theirs, dtype=dtype), ref.read_stars(mine, dtype=dtype)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[2], b[2])
    assert a[1] == b[1] and a[3] == b[3]


def test_params(tmp_path):
    f = tmp_path / "p.txt"
    f.write_text("num_stars 1234\nkappa_tot 0.45\nmass_function salpeter\n\nhalf_length 2.5e+01\nbig 1e20\n")
    p = util.read_params(str(f))
    assert p == {"num_stars": 1234, "kappa_tot": 0.45, "mass_function": "salpeter", "half_length": 25,
                 "big": 10**20}
    assert isinstance(p["num_stars"], int) and isinstance(p["kappa_tot"], float)
    assert isinstance(p["half_length"], int)
    f.write_text("a 1\nb 2 3\n")
    with pytest.raises(ValueError):
        util.read_params(str(f))


def test_params_match_reference(tmp_path):
    ref = _ref_util()
    f = tmp_path / "p.txt"
    f.write_text("num_stars 1234\nkappa_tot 0.45\nmass_function kroupa\nshear -0.2\nlight_loss 1e-3\nseed 7\n")
    assert util.read_params(str(f)) == ref.read_params(str(f))


@pytest.mark.parametrize("dtype,cplx", [(np.float32, False), (np.float64, False), (np.int32, False),
                                        (np.float64, True)])
def test_array_file(tmp_path, dtype, cplx):
    rng = np.random.default_rng(2)
    shape = (5, 7, 2) if cplx else (5, 7)
    a = (rng.normal(size=shape) * 100).astype(dtype)
    f = str(tmp_path / "a.bin")
    with open(f, "wb") as fh:
        fh.write(np.array([5, 7], np.int32).tobytes())
        fh.write(a.tobytes())
    got = util.read_array(f, dtype, is_complex=cplx)
    np.testing.assert_array_equal(got, a)
    assert got.dtype == dtype and got.shape == shape
    ref = _ref_util() if os.path.exists(REF_UTIL) else None
    if ref is not None:
        np.testing.assert_array_equal(ref.read_array(f, dtype, is_complex=cplx), got)


def test_hist_file(tmp_path):
    f = tmp_path / "h.txt"
    f.write_text("0 12\n1000 40\n2250 3\n")
    h = util.read_hist(str(f))
    assert h.dtype == np.int32
    np.testing.assert_array_equal(h, [[0, 12], [1000, 40], [2250, 3]])

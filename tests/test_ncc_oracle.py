"""NCC (caustic-crossing maps): the C restatement (oracle.c orc_ncc) pinned
against the reference's own kernels run on the host
(oracle/_ref/libref_ncc.so), on caustics of the CCF oracle; and the C ABI of
lib_ncc.so (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

from oracle import ccf_ref
from oracle import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def caustics(n=30, seed=5, nphi=200):
    rng = np.random.default_rng(seed)
    rad = np.sqrt(n / 0.27)
    r = rad * np.sqrt(rng.random(n))
    a = 2 * np.pi * rng.random(n)
    stars = np.stack([r * np.cos(a), r * np.sin(a), np.ones(n)], 1)
    L = ccf_ref.Lens(stars, 0.3, 0.3, 0.27, 1.0, 1, rad)
    z = ccf_ref.critical_curves(L, ccf_ref.initial_roots(stars, 2 * n, nphi, 1, rad), nphi, 1)
    return ccf_ref.outputs(L, z, 1)[1]


@pytest.mark.skipif(not po.ref_ncc_available(), reason="reference NCC library not built (oracle/Makefile ref)")
@pytest.mark.parametrize("center,hl,npix,os_", [((0.3, -0.2), (4, 4), (100, 100), 2), ((0, 0), (6, 3), (120, 60), 1),
                                                ((1, 1), (3, 3), (64, 64), 0), ((0, 0), (10, 10), (200, 200), 3)])
def test_oracle_matches_reference(center, hl, npix, os_):
    c = caustics()
    ours, err = po.ncc(c, center, hl, npix, os_)
    ref = po.ref_ncc(c, center, hl, npix, os_)
    assert err == 0
    assert ours.max() > 0
    assert np.array_equal(ours, ref)


def test_oracle_counts_nested_caustics():
    """A clockwise circle adds one inside it; two nested circles two."""
    t = -np.linspace(0, 2 * np.pi, 401)
    circ = lambda r, x0: x0 + r * np.cos(t) + 1j * r * np.sin(t)
    c = np.stack([circ(1.0, 0), circ(2.0, 0)])
    m, err = po.ncc(c, (0, 0), (3, 3), (60, 60), 0)
    assert err == 0
    y, x = np.mgrid[0:60, 0:60]
    px, py = -3 + (x + 0.5) * 0.1, 3 - (y + 0.5) * 0.1
    rr = np.hypot(px, py)
    assert np.all(m[rr < 0.95] == 2) and np.all(m[(rr > 1.05) & (rr < 1.95)] == 1) and np.all(m[rr > 2.05] == 0)


def declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", txt)) - {"if", "while", "for", "return"})


def test_ncc_library_exports():
    from irs_b200 import ncc
    from irs_b200._lib import LIBDIR
    lib = ctypes.CDLL(os.path.join(LIBDIR, "lib_ncc.so"))
    names = declared("lib_ncc.h")
    assert len(names) >= 29
    assert not [n for n in names if not hasattr(lib, n)]
    assert len(ncc.REFERENCE_NCC_SYMBOLS) == 26  # src/lib_ncc.cu:15-44
    assert not [n for n in ncc.REFERENCE_NCC_SYMBOLS if not hasattr(lib, n)]


def test_ncc_wrapper_setters():
    from irs_b200 import NCC
    n = NCC(infile_prefix="./Some/", center_y1=0.5, half_length_y1=2.0, half_length_y2=3.0, num_pixels_y1=50,
            num_pixels_y2=40, over_sample=1)
    assert n.infile_prefix == "./Some/" and n.num_pixels == (50, 40) and n.over_sample == 1
    assert n.pixel_scales == (0.08, 0.15)
    with pytest.raises(ValueError):
        n.half_length_y1 = 0
    with pytest.raises(ValueError):
        n.over_sample = -1
    n.close()

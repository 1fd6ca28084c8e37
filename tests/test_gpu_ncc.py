"""NCC on the GPU (lib_ncc.so) against the C restatement (oracle.c orc_ncc,
pinned against the reference's own kernels in tests/test_ncc_oracle.py):
integer maps, bit for bit; and the chain CCF -> ccf_caustics.bin -> NCC."""
import os
import struct

import numpy as np
import pytest

from oracle import ccf_ref
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def oracle_caustics(n, seed, nphi=200):
    rng = np.random.default_rng(seed)
    rad = np.sqrt(n / 0.27)
    r = rad * np.sqrt(rng.random(n))
    a = 2 * np.pi * rng.random(n)
    stars = np.stack([r * np.cos(a), r * np.sin(a), np.ones(n)], 1)
    L = ccf_ref.Lens(stars, 0.3, 0.3, 0.27, 1.0, 1, rad)
    z = ccf_ref.critical_curves(L, ccf_ref.initial_roots(stars, 2 * n, nphi, 1, rad), nphi, 1)
    return ccf_ref.outputs(L, z, 1)[1]


@pytest.mark.parametrize("center,hl,npix,os_", [((0.3, -0.2), (4, 4), (100, 100), 2), ((0, 0), (6, 3), (120, 60), 1),
                                                ((1, 1), (3, 3), (64, 64), 0), ((0, 0), (10, 10), (200, 200), 3)])
def test_ncc_matches_oracle(center, hl, npix, os_):
    from irs_b200 import NCC
    c = oracle_caustics(30, 5)
    n = NCC(center_y1=center[0], center_y2=center[1], half_length_y1=hl[0], half_length_y2=hl[1],
            num_pixels_y1=npix[0], num_pixels_y2=npix[1], over_sample=os_)
    n.set_caustics(c)
    n.run()
    ref, err = po.ncc(c, center, hl, npix, os_)
    assert err == 0 and n.value("errors") == 0
    assert n.num_caustic_crossings.shape == (npix[1], npix[0])
    assert np.array_equal(n.num_caustic_crossings, ref)
    assert n.value("max_num") == ref.max() > 0
    n.close()


def test_ccf_to_ncc_through_files(tmp_path):
    """A CCF run writes ccf_caustics.bin; NCC reads it (the reference's
    workflow) and its map equals the oracle's on the same caustics; save()
    writes the reference's files."""
    from irs_b200 import CCF, NCC
    pre = str(tmp_path) + "/"
    c = CCF(kappa_tot=0.3, shear=0.3, kappa_star=0.27, num_stars=60, random_seed=11, num_phi=200,
            write_caustics=True, outfile_prefix=pre)
    c.run()
    c.save()
    caus = c.caustics[..., 0] + 1j * c.caustics[..., 1]
    n = NCC(infile_prefix=pre, half_length_y1=5, half_length_y2=5, num_pixels_y1=256, num_pixels_y2=256,
            over_sample=2, outfile_prefix=pre)
    n.run()
    ref, _ = po.ncc(caus, (0, 0), (5, 5), (256, 256), 2)
    assert np.array_equal(n.num_caustic_crossings, ref)
    n.save()
    with open(tmp_path / "ncc_ncc.bin", "rb") as f:
        nr, nc = struct.unpack("ii", f.read(8))
        m = np.frombuffer(f.read(), np.int32).reshape(nr, nc)
    assert np.array_equal(m, ref)
    hist = np.loadtxt(tmp_path / "ncc_ncc_numpixels.txt", dtype=np.int64, ndmin=2)
    vals, counts = np.unique(ref, return_counts=True)
    assert np.array_equal(hist[:, 0], vals) and np.array_equal(hist[:, 1], counts)
    assert "over_sample 2" in open(tmp_path / "ncc_parameter_info.txt").read()
    c.close()
    n.close()


def test_ncc_missing_file_fails(tmp_path):
    from irs_b200 import NCC
    n = NCC(infile_prefix=str(tmp_path) + "/nothing_")
    with pytest.raises(Exception, match="Error running NCC"):
        n.run()
    n.close()

"""CCF on the GPU (lib_ccf.so) against the numpy restatement
oracle/ccf_ref.py (itself pinned against the reference's own root finding in
tests/test_ccf_oracle.py).

Both move every root of a chain at once from the previous iterate, so they
label the roots alike; the GPU takes the stars' near field and local
expansion from its tree (expansion error 1e-7 theta_star) where the oracle
sums every star, so positions agree to about that precision. The curves are
compared after matching labels at each branch centre (identical labels
expected), positions and caustics to 1e-7 theta_star, length scales to 1e-5
relative, and the error bound in 1/mu to the reference's 1e-9 precision."""
import os
import struct

import numpy as np
import pytest
from scipy.optimize import linear_sum_assignment

from oracle import ccf_ref
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def write_stars(path, stars, rad, theta=1.0):
    with open(path, "wb") as f:
        f.write(struct.pack("ii", len(stars), 0))
        f.write(struct.pack("ddd", rad, 0.0, theta))
        f.write(np.ascontiguousarray(stars, np.float64).tobytes())


def star_field(n, kstar, seed):
    rng = np.random.default_rng(seed)
    rad = np.sqrt(n / kstar)
    r = rad * np.sqrt(rng.random(n))
    a = 2 * np.pi * rng.random(n)
    m = rng.uniform(0.2, 1.0, n)
    return np.stack([r * np.cos(a), r * np.sin(a), m], 1), rad


def labels(ref, ours, nb):
    centre = (ref.shape[1] - 1) // 2
    perm = np.empty(ref.shape[0], int)
    for c in range(nb):
        rows = np.arange(c, ref.shape[0], nb)
        d = np.abs(ref[rows, centre][:, None] - ours[rows, centre][None, :])
        i, j = linear_sum_assignment(d)
        perm[rows[i]] = rows[j]
    return perm


def as_complex(a):
    return a[..., 0] + 1j * a[..., 1]


@pytest.mark.parametrize("n,approx,nphi,nb", [(20, 1, 24, 1), (20, 0, 24, 1), (30, 1, 40, 2), (200, 1, 20, 1)])
def test_ccf_matches_oracle(tmp_path, n, approx, nphi, nb):
    from irs_b200 import CCF
    kappa, gamma = 0.45, 0.25
    stars, rad = star_field(n, kstar=0.3, seed=n + approx)
    sf = str(tmp_path / "stars.bin")
    write_stars(sf, stars, rad)
    c = CCF(kappa_tot=kappa, shear=gamma, starfile=sf, approx=bool(approx), num_phi=nphi, num_branches=nb,
            write_caustics=True, write_length_scales=True, outfile_prefix=str(tmp_path) + "/")
    c.run()
    kstar = c.kappa_star
    assert c.num_roots == ccf_ref.num_roots(n, 0, approx)
    assert c.value("max_error") < 1e-8
    L = ccf_ref.Lens(stars, kappa, gamma, kstar, 1.0, approx, rad)
    init = ccf_ref.initial_roots(stars, c.num_roots, nphi, nb, rad)
    z = ccf_ref.critical_curves(L, init, nphi, nb)
    occs, ocaus, omu = ccf_ref.outputs(L, z, nb)
    gccs, gcaus = as_complex(c.critical_curves), as_complex(c.caustics)
    perm = labels(occs, gccs, nb)
    assert np.mean(perm == np.arange(len(perm))) > 0.95  # the same update scheme labels the roots alike
    assert np.abs(gccs[perm] - occs).max() < 1e-7
    assert np.abs(gcaus[perm] - ocaus).max() < 1e-7
    assert np.max(np.abs(c.mu_length_scales[perm] - omu) / np.abs(omu)) < 1e-5
    # stars come back in tree order: the same set
    assert np.allclose(np.sort(c.stars[:, 0]), np.sort(stars[:, 0]))
    c.close()


def test_ccf_generated_field_and_files(tmp_path):
    """The reference's default configuration (137 equal-mass stars, 100 phi
    steps): every root is critical to 1e-9 in 1/mu, two runs are identical,
    the caustics are the lens equation at the roots, and save() writes the
    reference's files."""
    from irs_b200 import CCF
    kw = dict(kappa_tot=0.3, shear=0.3, kappa_star=0.27, num_stars=137, random_seed=7, num_phi=100,
              write_caustics=True, write_length_scales=True, outfile_prefix=str(tmp_path) + "/")
    a = CCF(**kw)
    a.run()
    b = CCF(**kw)
    b.run()
    assert a.value("max_error") < 1e-8
    assert np.array_equal(a.critical_curves, b.critical_curves)
    assert np.array_equal(a.caustics, b.caustics)
    z = as_complex(a.critical_curves).ravel()
    L = ccf_ref.Lens(a.stars, a.kappa_tot, a.shear, a.kappa_star, 1.0, 1, a.corner[0])
    s1, dwdz, dwdzb, _ = L.fields(z)
    assert np.abs(dwdz ** 2 - np.abs(dwdzb) ** 2).max() < 1e-6  # det J = 0 on the critical curves
    w = (1 - L.kappa) * z + L.gamma * np.conj(z) - np.conj(s1) - L.alpha_smooth(z)
    assert np.abs(as_complex(a.caustics).ravel() - w).max() < 1e-6
    a.save()
    for name in ("ccf_parameter_info.txt", "ccf_stars.bin", "ccf_ccs.bin", "ccf_caustics.bin",
                 "ccf_mu_length_scales.bin"):
        assert os.path.exists(tmp_path / name)
    with open(tmp_path / "ccf_ccs.bin", "rb") as f:
        nr, nc = struct.unpack("ii", f.read(8))
        data = np.frombuffer(f.read(), np.float64).reshape(nr, nc, 2)
    assert (nr, nc) == (a.num_roots, 101)
    assert np.array_equal(data, a.critical_curves)
    info = open(tmp_path / "ccf_parameter_info.txt").read()
    assert "num_roots 274" in info and "max_error_1/mu" in info
    a.close()
    b.close()


def test_ccf_rejects_bad_input():
    from irs_b200 import CCF
    c = CCF(kappa_tot=0.3, shear=0.3, num_stars=10, num_phi=20)
    c.lib.set_num_branches(c.obj, 3)  # num_phi is not a multiple of 2 * num_branches
    with pytest.raises(Exception, match="Error running CCF"):
        c.run()
    c.close()


@pytest.mark.skipif(not po.ref_ccf_available(),
                    reason="reference CCF library not built (oracle/Makefile ref)")
@pytest.mark.parametrize("approx", [1, 0])
def test_ccf_rectangular_matches_reference(tmp_path, approx):
    """Rectangular fields (the smooth sheet's derivatives of
    alpha_smooth.cuh:141-300, and for approx the extra roots of its Taylor
    series) against the reference's own CCF kernels run on the host: at every
    phi the two sets of critical-curve points (and their caustics) agree.
    Sets, not labels: the two update schemes may follow a curve through a
    near-degenerate point on different roots."""
    from irs_b200 import CCF
    n = 24
    rng = np.random.default_rng(21 + approx)
    cx, cy = 8.0, 6.0  # kappa_star about 0.29
    stars = np.stack([rng.uniform(-cx, cx, n), rng.uniform(-cy, cy, n), rng.uniform(0.5, 1.0, n)], 1)
    sf = str(tmp_path / "rect.bin")
    with open(sf, "wb") as f:
        f.write(struct.pack("ii", n, 1))
        f.write(struct.pack("ddd", cx, cy, 1.0))
        f.write(np.ascontiguousarray(stars, np.float64).tobytes())
    nphi = 20
    c = CCF(kappa_tot=0.5, shear=0.2, starfile=sf, approx=bool(approx), num_phi=nphi, write_caustics=True)
    c.run()
    assert c.value("max_error") < 1e-8
    ts = int(c.value("taylor_smooth"))
    lens = po.lens(0.5, 0.2, c.kappa_star, 1.0, 1, approx, ts, (cx, cy))
    init = ccf_ref.initial_roots(stars, c.num_roots, nphi, 1, np.hypot(cx, cy))
    rc, rw, _, rme, _ = po.ref_ccf(stars, lens, max(cx, cy) * 1.1, init, nphi, 1)
    assert 0 <= rme < 1e-8
    g, gw = as_complex(c.critical_curves), as_complex(c.caustics)
    for k in range(g.shape[1]):
        d = np.abs(rc[:, k][:, None] - g[:, k][None, :])
        i, j = linear_sum_assignment(d)
        assert d[i, j].max() < 1e-6
        assert np.abs(rw[i, k] - gw[j, k]).max() < 1e-6
    c.close()

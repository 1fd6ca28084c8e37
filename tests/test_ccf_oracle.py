"""CCF (critical curves): the numpy restatement oracle/ccf_ref.py pinned
against the reference's own root finding run on the host
(oracle/_ref/libref_ccf.so), and the C ABI of lib_ccf.so (no GPU needed).

The two update schemes (the reference moves roots in place, the restatement
and the GPU move all roots of a chain at once) can send a starting point to a
different root at the branch centre; the curves then agree up to one
relabelling of the roots, the same for every phi row."""
import ctypes
import os
import re

import numpy as np
import pytest
from scipy.optimize import linear_sum_assignment

from oracle import ccf_ref
from oracle import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def star_field(n, kstar, seed, theta=1.0):
    rng = np.random.default_rng(seed)
    rad = np.sqrt(theta ** 2 * n * 1.0 / kstar)
    r = rad * np.sqrt(rng.random(n))
    a = 2 * np.pi * rng.random(n)
    return np.stack([r * np.cos(a), r * np.sin(a), np.ones(n)], 1), rad


def relabel(ref, ours, nb):
    """Permutation of our rows (root a of branch c is row a * nb + c) that
    matches the reference's roots at each branch's centre column; the labels
    of a branch are set where its roots are first found."""
    centre = (ref.shape[1] - 1) // 2
    perm = np.empty(ref.shape[0], int)
    for c in range(nb):
        rows = np.arange(c, ref.shape[0], nb)
        d = np.abs(ref[rows, centre][:, None] - ours[rows, centre][None, :])
        i, j = linear_sum_assignment(d)
        perm[rows[i]] = rows[j]
    return perm


@pytest.mark.skipif(not po.ref_ccf_available(), reason="reference CCF library not built (oracle/Makefile ref)")
@pytest.mark.parametrize("approx,nphi,nb", [(1, 20, 1), (0, 20, 1), (1, 24, 2), (0, 24, 2)])
def test_oracle_matches_reference(approx, nphi, nb):
    # With the exact circular sheet, d alpha_smooth / dz jumps at |z| = |corner|
    # and a root close to that circle can exist on either side; the update
    # schemes may then find different ones. The seeds keep the roots clear.
    kappa, gamma, kstar = 0.3, 0.3, 0.27
    stars, rad = star_field(12, kstar, seed=5 + nb if approx else 7 + nb)
    nroots = ccf_ref.num_roots(len(stars), 0, approx)
    init = ccf_ref.initial_roots(stars, nroots, nphi, nb, rad)
    L = ccf_ref.Lens(stars, kappa, gamma, kstar, 1.0, approx, rad)
    z = ccf_ref.critical_curves(L, init, nphi, nb)
    ccs, caus, mu = ccf_ref.outputs(L, z, nb)
    lens = po.lens(kappa, gamma, kstar, 1.0, 0, approx, 1, (rad, 0.0))
    rc, rw, rmu, rme, _ = po.ref_ccf(stars, lens, rad * 1.1, init, nphi, nb)
    assert 0 <= rme < 1e-8
    assert ccf_ref.max_error(L, z, nphi, nb) < 1e-8
    perm = relabel(rc, ccs, nb)
    assert np.abs(rc - ccs[perm]).max() < 1e-8
    assert np.abs(rw - caus[perm]).max() < 1e-8
    assert np.max(np.abs(rmu - mu[perm]) / np.abs(rmu)) < 1e-5


def test_oracle_roots_are_critical_points():
    """Every root of every row satisfies the critical-curve equation: the
    Jacobian determinant (1/mu) vanishes there."""
    kappa, gamma, kstar = 0.4, 0.2, 0.3
    stars, rad = star_field(8, kstar, seed=11)
    nphi, nb = 16, 1
    nroots = ccf_ref.num_roots(len(stars), 0, 1)
    L = ccf_ref.Lens(stars, kappa, gamma, kstar, 1.0, 1, rad)
    z = ccf_ref.critical_curves(L, ccf_ref.initial_roots(stars, nroots, nphi, nb, rad), nphi, nb)
    _, dwdz, dwdzb, _ = L.fields(z.ravel())
    inv_mu = dwdz ** 2 - np.abs(dwdzb) ** 2
    assert np.abs(inv_mu).max() < 1e-8


def declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", txt)) - {"if", "while", "for", "return"})


def test_ccf_library_exports():
    from irs_b200 import ccf
    from irs_b200._lib import LIBDIR
    lib = ctypes.CDLL(os.path.join(LIBDIR, "lib_ccf.so"))
    names = declared("lib_ccf.h")
    assert len(names) >= 56
    assert not [n for n in names if not hasattr(lib, n)]
    assert len(ccf.REFERENCE_CCF_SYMBOLS) == 53  # src/lib_ccf.cu:15-71
    assert not [n for n in ccf.REFERENCE_CCF_SYMBOLS if not hasattr(lib, n)]


def test_ccf_wrapper_setters():
    from irs_b200 import CCF
    c = CCF(kappa_tot=0.5, shear=0.2, smooth_fraction=0.2, mass_function="Kroupa", m_lower=0.1, m_upper=1.0,
            num_stars=50, num_phi=40, num_branches=2, random_seed=3)
    assert abs(c.kappa_star - 0.4) < 1e-12
    assert c.mass_function == "kroupa" and c.num_branches == 2 and c.num_phi == 40
    with pytest.raises(ValueError):
        c.safety_scale = 1.0
    with pytest.raises(ValueError):
        CCF(kappa_tot=0.5, shear=0.2, num_phi=30, num_branches=2)
    c.close()

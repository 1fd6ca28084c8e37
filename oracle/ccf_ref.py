"""Test infrastructure: CPU restatement (numpy, FP64) of the critical-curve
finder of the reference (include/ccf.cuh, include/ccf_functions.cuh) for
circular star fields, the check of irs_b200's CCF kernels.

It follows the reference's algorithm with the deflection of the stars summed
directly over every star (no tree expansion) and the simultaneous root update
applied as a Jacobi step (all roots of a chain move from the previous
iterate), as the GPU kernels apply it:
  * initial roots star +/- 1 and, beyond 2 N, on the circle |z| = |corner|
    (ccf.cuh:706-726), at the centre row of each branch (ccf_functions.cuh:355);
  * f0 = conj(dw/dzbar) - dw/dz e^{-i phi}, f1 = conj(d2w/dzbar2)
    (ccf_functions.cuh:69-124); update z - f0 / (f1 + f0 (p_sum - root_sum))
    with p_sum = 2 (sum 1/(z - z_i) [+ 1/z for the exact circular sheet])
    (ccf_functions.cuh:196-253); a root is final once its 1/mu bound is below
    1e-9 or a step moves it by less than 1e-9 theta (:205-210, :367-372);
  * steps j = 1 .. nphi / (2 nb) start from step j - 1 (:268-301);
  * caustics w(z) (:33-46) and magnification length scales (:145-166).
Its own results are pinned against the reference run on the host
(oracle/_ref/libref_ccf.so, built from the reference's sources by
oracle/Makefile) in tests/test_ccf_oracle.py.
"""
from __future__ import annotations

import numpy as np


def num_roots(n, rect=0, approx=1, taylor_smooth=1):
    """include/ccf.cuh:470-494"""
    if rect:
        return 2 * n + taylor_smooth - 1 if approx else 2 * n
    return 2 * n if approx else 2 * n + 2


def row(nphi, nb, c, j):
    return nphi // (2 * nb) + c * (nphi // nb) + c + j


def phi_of(nphi, nb, c, j):
    return np.pi / nb + c * 2 * np.pi / nb + 2 * np.pi / nphi * j


def initial_roots(stars, nroots, nphi, nb, corner_abs):
    """(nphi + nb, nroots) complex array with the branch-centre rows set."""
    s = np.asarray(stars, np.float64)
    n = s.shape[0]
    z = np.zeros((nphi + nb, nroots), np.complex128)
    pos = s[:, 0] + 1j * s[:, 1]
    extra = nroots - 2 * n
    for c in range(nb):
        r = row(nphi, nb, c, 0)
        z[r, :n] = pos + 1
        z[r, n:2 * n] = pos - 1
        if extra > 0:
            ang = 2 * np.pi / extra * np.arange(extra)
            z[r, 2 * n:] = corner_abs * (np.cos(ang) + 1j * np.sin(ang))
    return z


class Lens:
    """Circular field: kappa, gamma, kappa_star, theta, approx, |corner|."""

    def __init__(self, stars, kappa, gamma, kstar, theta=1.0, approx=1, corner_abs=None):
        self.s = np.asarray(stars, np.float64)
        self.pos = self.s[:, 0] + 1j * self.s[:, 1]
        self.m = self.s[:, 2]
        self.kappa, self.gamma, self.kstar, self.theta, self.approx = kappa, gamma, kstar, theta, approx
        self.ca = corner_abs

    def fields(self, z):
        """s1, dw/dz, dw/dzbar, d2w/dzbar2 at the points z (1-d)."""
        d = z[:, None] - self.pos[None, :]
        r = 1.0 / d
        t2 = self.theta ** 2
        s1 = (self.m * r).sum(1)
        s2 = (self.m * r * r).sum(1)
        s3 = (self.m * r * r * r).sum(1)
        das = np.conj(-t2 * s2)
        d2as = np.conj(2 * t2 * s3)
        if self.approx:
            dsz = np.full(z.shape, -self.kstar)
            dszb = np.zeros_like(z)
            d2szb = np.zeros_like(z)
        else:
            ca2 = self.ca ** 2
            dsz = -self.kstar * (self.ca - np.abs(z) >= 0)
            dszb = self.kstar * ca2 / np.conj(z) ** 2
            d2szb = -2 * self.kstar * ca2 / np.conj(z) ** 3
        dwdz = 1 - self.kappa - dsz
        dwdzb = self.gamma - das - dszb
        d2wdzb2 = -(d2as + d2szb)
        return s1, dwdz, dwdzb, d2wdzb2

    def alpha_smooth(self, z):
        if self.approx:
            return -self.kstar * z
        inside = np.abs(z) <= self.ca
        return np.where(inside, -self.kstar * z, -self.kstar * self.ca ** 2 / np.conj(np.where(inside, 1, z)))


def _bound(af0, dwdz):
    return np.maximum(np.abs(af0 * (af0 + 2 * dwdz)), np.abs(af0 * (af0 - 2 * dwdz)))


def jacobi_step(L: Lens, z, phi, fin):
    """One simultaneous update of the roots z of one chain; fin is updated."""
    _, dwdz, dwdzb, d2 = L.fields(z)
    f0 = np.conj(dwdzb) - dwdz * np.exp(-1j * phi)
    act = ~fin
    done = _bound(np.abs(f0), dwdz) < 1e-9
    fin |= act & done
    act &= ~done
    f1 = np.conj(d2)
    ps = (1.0 / (z[:, None] - L.pos[None, :])).sum(1)
    if not L.approx:
        ps = ps + 1.0 / z
    ps = 2 * ps
    dz = z[:, None] - z[None, :]
    np.fill_diagonal(dz, 1.0)
    rr = 1.0 / dz
    np.fill_diagonal(rr, 0.0)
    rs = rr.sum(1)
    zn = z - f0 / (f1 + f0 * (ps - rs))
    out = np.where(act, zn, z)
    fin |= act & (np.abs(zn - z) / L.theta < 1e-9)
    return out


def critical_curves(L: Lens, init, nphi, nb, iters=(30, 20)):
    """Roots of every row, (nphi + nb, nroots), from `init` (initial_roots)."""
    z = np.array(init, np.complex128)
    nroots = z.shape[1]
    it0 = iters[0] + (iters[0] & 1)
    it1 = iters[1] + (iters[1] & 1)
    for c in range(nb):
        r = row(nphi, nb, c, 0)
        fin = np.zeros(nroots, bool)
        for _ in range(it0):
            z[r] = jacobi_step(L, z[r], phi_of(nphi, nb, c, 0), fin)
    for j in range(1, nphi // (2 * nb) + 1):
        for c in range(nb):
            for sgn in (-1, 1):
                r, rp = row(nphi, nb, c, sgn * j), row(nphi, nb, c, sgn * (j - 1))
                z[r] = z[rp]
                fin = np.zeros(nroots, bool)
                for _ in range(it1):
                    z[r] = jacobi_step(L, z[r], phi_of(nphi, nb, c, sgn * j), fin)
    return z


def max_error(L: Lens, z, nphi, nb):
    """Largest error bound in 1/mu over every root of every row (:420-463)."""
    rows, _ = z.shape
    per = nphi // nb + 1
    half = nphi // (2 * nb)
    e = 0.0
    for r in range(rows):
        c, sj = r // per, r % per - half
        _, dwdz, dwdzb, _ = L.fields(z[r])
        f0 = np.conj(dwdzb) - dwdz * np.exp(-1j * phi_of(nphi, nb, c, sj))
        e = max(e, float(_bound(np.abs(f0), dwdz).max()))
    return e


def outputs(L: Lens, z, nb):
    """Critical curves, caustics and length scales, each (nroots * nb, rows / nb)."""
    rows, nroots = z.shape
    zz = z.T.reshape(-1)  # [root][row]
    s1, dwdz, dwdzb, d2 = L.fields(zz)
    t2 = L.theta ** 2
    w = (1 - L.kappa) * zz + L.gamma * np.conj(zz) - np.conj(t2 * s1) - L.alpha_smooth(zz)
    cct = -2j * np.conj(dwdzb) * d2
    ct = dwdz * cct + dwdzb * np.conj(cct)
    mu = 1.0 / (2 * np.abs(ct))
    shape = (nroots * nb, rows // nb)
    return zz.reshape(shape), w.reshape(shape), mu.reshape(shape)

"""ctypes wrapper of oracle/liboracle.so -- test infrastructure only.

The CPU oracle restates the reference algorithm in FP64 (see oracle.c). Only
tests, the smoke check and the benchmark's CPU-baseline leg use it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


class OrcLens(C.Structure):
    _fields_ = [("kappa", C.c_double), ("gamma", C.c_double), ("kstar", C.c_double), ("theta", C.c_double),
                ("rect", C.c_int), ("approx", C.c_int), ("taylor_smooth", C.c_int),
                ("corner_re", C.c_double), ("corner_im", C.c_double)]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        vp, d, i, ll = C.c_void_p, C.c_double, C.c_int, C.c_longlong
        L.orc_tree_build.argtypes = [i, vp, d, i, d, d]
        L.orc_tree_build.restype = vp
        L.orc_tree_free.argtypes = [vp]
        for f in ["orc_tree_num_nodes", "orc_tree_levels", "orc_tree_order", "orc_tree_overflow"]:
            getattr(L, f).argtypes = [vp]
            getattr(L, f).restype = i
        L.orc_tree_stars.argtypes = [vp, vp]
        L.orc_tree_nodes.argtypes = [vp, vp, vp, vp, vp, vp]
        L.orc_tree_coeffs.argtypes = [vp, vp, vp]
        L.orc_shoot_fmm.argtypes = [vp, C.POINTER(OrcLens), ll, vp, vp, vp, vp, vp]
        L.orc_shoot_direct.argtypes = [i, vp, C.POINTER(OrcLens), ll, vp, vp, vp, vp, i]
        L.orc_shoot_direct_lattice.argtypes = [i, vp, C.POINTER(OrcLens), d, d, d, d, ll, ll, ll, ll, vp, vp, i]
        L.orc_irs_bin.argtypes = [ll, vp, vp, vp, d, d, d, d, i, i, vp, vp, vp]
        L.orc_ipm_deposit_ref.argtypes = [ll, ll, vp, vp, d, i, i, vp, vp, vp, i]
        L.orc_ipm_deposit_fix_f32.argtypes = [ll, ll, vp, C.c_float, i, i, vp, vp, vp, i]
        L.orc_ipm_deposit_fix_f64.argtypes = [ll, ll, vp, d, i, i, vp, vp, vp, i]
        L.orc_derive.argtypes = [d, d, d, d, d, d, d, i, d, d, d, d, d, i, i, i, vp]
        L.orc_ncc.argtypes = [vp, i, i, d, d, d, d, i, i, i, vp]
        L.orc_ncc.restype = i
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data


def lens(kappa, gamma, kstar, theta, rect=0, approx=1, taylor_smooth=1, corner=(0.0, 0.0)):
    return OrcLens(float(kappa), float(gamma), float(kstar), float(theta), int(rect), int(approx),
                   int(taylor_smooth), float(corner[0]), float(corner[1]))


class Tree:
    """Quadtree + expansions of the reference algorithm (FP64)."""

    def __init__(self, stars, root_hl, order=0, theta=1.0, alpha_error=1e-3):
        s = np.ascontiguousarray(np.asarray(stars, np.float64).reshape(-1, 3))
        self.h = lib().orc_tree_build(int(s.shape[0]), _p(s), float(root_hl), int(order), float(theta),
                                      float(alpha_error))
        self.n = lib().orc_tree_num_nodes(self.h)
        self.levels = lib().orc_tree_levels(self.h)
        self.order = lib().orc_tree_order(self.h)
        self.overflow = lib().orc_tree_overflow(self.h)
        self.nstars = s.shape[0]

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_tree_free(self.h)
            self.h = None

    def stars(self):
        out = np.zeros((self.nstars, 3))
        lib().orc_tree_stars(self.h, _p(out))
        return out

    def arrays(self):
        ints = np.zeros((self.n, 8), np.int32)
        geom = np.zeros((self.n, 3))
        nbr = np.zeros((self.n, 8), np.int32)
        sil = np.zeros((self.n, 27), np.int32)
        dil = np.zeros((self.n, 5), np.int32)
        lib().orc_tree_nodes(self.h, _p(ints), _p(geom), _p(nbr), _p(sil), _p(dil))
        return ints, geom, nbr, sil, dil

    def coeffs(self):
        m = np.zeros((self.n, self.order + 1, 2))
        l = np.zeros((self.n, self.order + 1, 2))
        lib().orc_tree_coeffs(self.h, _p(m), _p(l))
        return m[..., 0] + 1j * m[..., 1], l[..., 0] + 1j * l[..., 1]

    def shoot(self, lens_, zx, zy, want_mu=False):
        zx = np.ascontiguousarray(zx, np.float64).ravel()
        zy = np.ascontiguousarray(zy, np.float64).ravel()
        wx = np.zeros_like(zx)
        wy = np.zeros_like(zy)
        mu = np.zeros_like(zx) if want_mu else None
        lib().orc_shoot_fmm(self.h, C.byref(lens_), zx.size, _p(zx), _p(zy), _p(wx), _p(wy),
                            _p(mu) if want_mu else None)
        return (wx, wy, mu) if want_mu else (wx, wy)


def shoot_direct(stars, lens_, zx, zy, threads=0):
    s = np.ascontiguousarray(np.asarray(stars, np.float64).reshape(-1, 3))
    zx = np.ascontiguousarray(zx, np.float64).ravel()
    zy = np.ascontiguousarray(zy, np.float64).ravel()
    wx = np.zeros_like(zx)
    wy = np.zeros_like(zy)
    lib().orc_shoot_direct(s.shape[0], _p(s), C.byref(lens_), zx.size, _p(zx), _p(zy), _p(wx), _p(wy), threads)
    return wx, wy


def shoot_direct_lattice(stars, lens_, bx, by, rx, ry, i0, ni, j0, nj, threads=0):
    s = np.ascontiguousarray(np.asarray(stars, np.float64).reshape(-1, 3))
    wx = np.zeros((nj, ni))
    wy = np.zeros((nj, ni))
    lib().orc_shoot_direct_lattice(s.shape[0], _p(s), C.byref(lens_), bx, by, rx, ry, i0, ni, j0, nj, _p(wx),
                                   _p(wy), threads)
    return wx, wy


def irs_bin(wx, wy, center, hly, npix, mu=None):
    wx = np.ascontiguousarray(wx, np.float64).ravel()
    wy = np.ascontiguousarray(wy, np.float64).ravel()
    pix = np.zeros((npix[1], npix[0]), np.int32)
    pmin = np.zeros_like(pix)
    psad = np.zeros_like(pix)
    m = None if mu is None else np.ascontiguousarray(mu, np.float64).ravel()
    lib().orc_irs_bin(wx.size, _p(wx), _p(wy), _p(m) if m is not None else None, center[0], center[1], hly[0],
                      hly[1], npix[0], npix[1], _p(pix), _p(pmin), _p(psad))
    return (pix, pmin, psad) if mu is not None else pix


def ipm_deposit_ref(verts, factor, npix, parities=False):
    """verts: (ny+1, nx+1, 2) vertex pixel positions (row axis flipped)."""
    v = np.ascontiguousarray(verts, np.float64)
    assert v.ndim == 3 and v.shape[2] == 2, "verts must be (ny+1, nx+1, 2)"
    ncy, ncx = v.shape[0] - 1, v.shape[1] - 1
    vx = np.ascontiguousarray(v[..., 0])
    vy = np.ascontiguousarray(v[..., 1])
    pix = np.zeros((npix[1], npix[0]))
    pmin = np.zeros_like(pix)
    psad = np.zeros_like(pix)
    lib().orc_ipm_deposit_ref(ncx, ncy, _p(vx), _p(vy), float(factor), npix[0], npix[1], _p(pix), _p(pmin),
                              _p(psad), int(parities))
    return (pix, pmin, psad) if parities else pix


def ipm_deposit_fixed(verts, factor, npix, parities=False, single=True):
    v = np.ascontiguousarray(verts, np.float64)
    assert v.ndim == 3 and v.shape[2] == 2, "verts must be (ny+1, nx+1, 2)"
    ncy, ncx = v.shape[0] - 1, v.shape[1] - 1
    mt = np.zeros((npix[1], npix[0]), np.uint64)
    mn = np.zeros_like(mt)
    ms = np.zeros_like(mt)
    f = lib().orc_ipm_deposit_fix_f32 if single else lib().orc_ipm_deposit_fix_f64
    f(ncx, ncy, _p(v), factor, npix[0], npix[1], _p(mt), _p(mn), _p(ms), int(parities))
    return (mn, ms) if parities else mt


def fix_to_float(a):
    """Fixed-point map (uint64, 2^32 per unit, modulo 2^64) -> float64: read
    as signed, a few units below zero (rounding where the coverage is zero or
    nearly so) read as 0, as the GPU's conversion does."""
    return np.maximum(np.asarray(a).view(np.int64), 0).astype(np.float64) / 2.0 ** 32


def derive(kappa, gamma, kstar, theta, mean_mass, mean_mass2, light_loss, rect, safety, center, hly, npix, nry):
    out = np.zeros(14)
    lib().orc_derive(kappa, gamma, kstar, theta, mean_mass, mean_mass2, light_loss, int(rect), safety, center[0],
                     center[1], hly[0], hly[1], npix[0], npix[1], nry, _p(out))
    keys = ["mu_ave", "num_rays_x", "ray_half_sep_1", "ray_half_sep_2", "half_length_x1", "half_length_x2",
            "num_ray_threads_1", "num_ray_threads_2", "center_x1", "center_x2", "num_stars", "corner_x1",
            "corner_x2", "alpha_error"]
    return dict(zip(keys, out))


# ---------------------------------------------------------------- reference code on the host
REFDIR = os.path.join(HERE, "_ref")


class RefLens(C.Structure):
    _fields_ = OrcLens._fields_


_ref = {}


def ref_available() -> bool:
    return all(os.path.exists(os.path.join(REFDIR, f)) for f in ("libref_ipm.so", "libref_irs.so"))


def build_ref():
    """Compile the reference's headers for the host (needs the reference sources)."""
    subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def ref_lib(kind="ipm"):
    if kind not in _ref:
        L = C.CDLL(os.path.join(REFDIR, f"libref_{kind}.so"))
        vp, d, i, ll = C.c_void_p, C.c_double, C.c_int, C.c_longlong
        if kind == "ncc":
            L.ref_ncc_run.argtypes = [vp, i, i, d, d, d, d, i, i, i, vp]
            _ref[kind] = L
            return L
        L.ref_tree_build.argtypes = [i, vp, d, i, d, d]
        L.ref_tree_build.restype = vp
        L.ref_tree_free.argtypes = [vp]
        for f in ["ref_tree_levels", "ref_tree_order", "ref_tree_num_nodes"]:
            getattr(L, f).argtypes = [vp]
            getattr(L, f).restype = i
        L.ref_tree_nodes.argtypes = [vp] + [vp] * 7
        L.ref_points.argtypes = [vp, C.POINTER(RefLens), ll, vp, vp, vp, vp, i]
        if kind == "ccf":
            L.ref_ccf_run.argtypes = [vp, C.POINTER(RefLens), i, i, i, vp, i, i, vp, vp, vp, vp]
        elif kind == "ipm":
            L.ref_shoot_cells.argtypes = [vp, C.POINTER(RefLens), d, d, i, i, d, d, d, d, d, d, d, d, i, i, vp, vp,
                                          vp, i]
            L.ref_deposit_cells.argtypes = [ll, ll, vp, d, i, i, vp, vp, vp, i]
        else:
            L.ref_shoot_rays.argtypes = [vp, C.POINTER(RefLens), d, d, i, i, d, d, d, d, d, d, d, d, i, i, vp, vp,
                                         vp, i]
        _ref[kind] = L
    return _ref[kind]


def ref_lens(l: OrcLens) -> RefLens:
    return RefLens(*[getattr(l, f[0]) for f in OrcLens._fields_])


class RefTree:
    """Tree and expansions built by the reference's own kernels on the host."""

    def __init__(self, stars, root_hl, order=0, theta=1.0, alpha_error=1e-3, kind="ipm"):
        self.L = ref_lib(kind)
        s = np.ascontiguousarray(np.asarray(stars, np.float64).reshape(-1, 3))
        self.h = self.L.ref_tree_build(s.shape[0], _p(s), float(root_hl), int(order), float(theta),
                                       float(alpha_error))
        self.levels = self.L.ref_tree_levels(self.h)
        self.order = self.L.ref_tree_order(self.h)
        self.n = self.L.ref_tree_num_nodes(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_tree_free(self.h)
            self.h = None

    def nodes(self):
        n, P = self.n, self.order
        ints = np.zeros((n, 8), np.int32)
        geom = np.zeros((n, 3))
        nbr = np.zeros((n, 8), np.int32)
        sil = np.zeros((n, 27), np.int32)
        dil = np.zeros((n, 5), np.int32)
        mult = np.zeros((n, P + 1, 2))
        loc = np.zeros((n, P + 1, 2))
        self.L.ref_tree_nodes(self.h, _p(ints), _p(geom), _p(nbr), _p(sil), _p(dil), _p(mult), _p(loc))
        return ints, geom, nbr, sil, dil, mult[..., 0] + 1j * mult[..., 1], loc[..., 0] + 1j * loc[..., 1]

    def points(self, lens_, zx, zy, threads=0):
        zx = np.ascontiguousarray(zx, np.float64).ravel()
        zy = np.ascontiguousarray(zy, np.float64).ravel()
        wx, wy = np.zeros_like(zx), np.zeros_like(zy)
        self.L.ref_points(self.h, C.byref(ref_lens(lens_)), zx.size, _p(zx), _p(zy), _p(wx), _p(wy), threads)
        return wx, wy

    def shoot(self, lens_, rhs, nrt, center_x, hlx, center_y, hly, npix, threads=0, parities=False, ints=False):
        T = np.int32 if ints else np.float64
        pix = np.zeros((npix[1], npix[0]), T)
        pmin = np.zeros_like(pix) if parities else None
        psad = np.zeros_like(pix) if parities else None
        f = self.L.ref_shoot_rays if ints else self.L.ref_shoot_cells
        f(self.h, C.byref(ref_lens(lens_)), rhs[0], rhs[1], int(nrt[0]), int(nrt[1]), center_x[0], center_x[1],
          hlx[0], hlx[1], center_y[0], center_y[1], hly[0], hly[1], int(npix[0]), int(npix[1]), _p(pix),
          _p(pmin) if parities else None, _p(psad) if parities else None, threads)
        if parities and not ints:
            pix = pmin + psad  # add_arrays_kernel (ipm.cuh:937-945)
        return (pix, pmin, psad) if parities else pix


def ref_deposit_cells(verts, factor, npix, parities=False):
    L = ref_lib("ipm")
    v = np.ascontiguousarray(verts, np.float64)
    assert v.ndim == 3 and v.shape[2] == 2, "verts must be (ny+1, nx+1, 2)"
    ncy, ncx = v.shape[0] - 1, v.shape[1] - 1
    pix = np.zeros((npix[1], npix[0]))
    pmin, psad = np.zeros_like(pix), np.zeros_like(pix)
    L.ref_deposit_cells(ncx, ncy, _p(v), float(factor), npix[0], npix[1], _p(pix), _p(pmin), _p(psad),
                        int(parities))
    return (pmin + psad, pmin, psad) if parities else pix


def ref_ccf_available() -> bool:
    return os.path.exists(os.path.join(REFDIR, "libref_ccf.so"))


def ref_ccf(stars, lens_, root_hl, init_roots, nphi, nb, iters=(30, 20), alpha_error=1e-7):
    """The reference's own critical-curve pipeline (include/ccf.cuh) on the
    host: tree and expansions of `stars` (x, y, m rows, in the given order),
    then the root finding from `init_roots` ((nphi + nb, nroots) complex, the
    branch-centre rows filled). Returns (ccs, caustics, mu_length_scales,
    max_error) with ccs / caustics of shape (nroots * nb, nphi / nb + 1)."""
    tree = RefTree(stars, root_hl, 0, lens_.theta, alpha_error * lens_.theta, kind="ccf")
    z = np.ascontiguousarray(np.asarray(init_roots, np.complex128))
    rows, nroots = z.shape
    ccs = np.zeros(rows * nroots, np.complex128)
    caus = np.zeros_like(ccs)
    mu = np.zeros(rows * nroots)
    me = C.c_double(0)
    tree.L.ref_ccf_run(tree.h, C.byref(ref_lens(lens_)), nroots, int(nphi), int(nb), _p(z), int(iters[0]),
                       int(iters[1]), _p(ccs), _p(caus), _p(mu), C.byref(me))
    shape = (nroots * nb, nphi // nb + 1)
    return ccs.reshape(shape), caus.reshape(shape), mu.reshape(shape), me.value, tree


def ncc(caustics, center, half_length, npix, over_sample=2):
    """Number-of-caustic-crossings map (oracle restatement, oracle.c orc_ncc):
    caustics (rows, cols) complex; returns (npy, npx) int32 and the number of
    crossings that fell outside the map."""
    c = np.ascontiguousarray(np.asarray(caustics, np.complex128))
    out = np.zeros((npix[1], npix[0]), np.int32)
    err = lib().orc_ncc(_p(c), c.shape[0], c.shape[1], float(center[0]), float(center[1]), float(half_length[0]),
                        float(half_length[1]), int(npix[0]), int(npix[1]), int(over_sample), _p(out))
    return out, err


def ref_ncc_available() -> bool:
    return os.path.exists(os.path.join(REFDIR, "libref_ncc.so"))


def ref_ncc(caustics, center, half_length, npix, over_sample=2):
    """The reference's own NCC kernels on the host (oracle/_ref/libref_ncc.so)."""
    c = np.ascontiguousarray(np.asarray(caustics, np.complex128))
    out = np.zeros((npix[1], npix[0]), np.int32)
    ref_lib("ncc").ref_ncc_run(_p(c), c.shape[0], c.shape[1], float(center[0]), float(center[1]),
                               float(half_length[0]), float(half_length[1]), int(npix[0]), int(npix[1]),
                               int(over_sample), _p(out))
    return out

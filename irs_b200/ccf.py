"""Critical curves and caustics of a star field (CCF) on the GPU.

`CCF` mirrors the reference wrapper microlensing/CCF/ccf.py (class CCF): the
same constructor keywords, validated property setters that raise ValueError,
run() raising Exception("Error running CCF") on failure, numpy copies of the
critical curves, caustics, magnification length scales and stars, t_ccs and
save(). The library is irs_b200/lib/lib_ccf.so (double), whose symbols are
those of the reference's src/lib_ccf.cu.

Extensions beyond the reference: num_iters (iterations of the simultaneous
root update at the branch centres and per phi step), value(name) for derived
values and timings, and close().
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import LIBDIR

_MASS_FUNCTIONS = ["equal", "uniform", "salpeter", "kroupa", "optical_depth"]
_FLOAT_FIELDS = ["kappa_tot", "shear", "kappa_star", "theta_star", "m_solar", "m_lower", "m_upper", "safety_scale"]
_INT_FIELDS = ["rectangular", "approx", "num_stars", "num_phi", "num_branches", "random_seed", "write_stars",
               "write_critical_curves", "write_caustics", "write_mu_length_scales"]
_STR_FIELDS = ["mass_function", "starfile", "outfile_prefix"]
_lib_cache = []
# the exports of the reference's src/lib_ccf.cu (lines 15-71)
REFERENCE_CCF_SYMBOLS = (["init", "run", "save", "get_num_roots", "get_corner_x1", "get_corner_x2", "get_stars",
                          "get_critical_curves", "get_caustics", "get_mu_length_scales", "get_t_ccs"] +
                         [f"{a}_{f}" for f in _FLOAT_FIELDS + _INT_FIELDS + _STR_FIELDS for a in ("set", "get")])


def load():
    """Load (once) and bind lib_ccf.so; raises if it is missing."""
    if _lib_cache:
        return _lib_cache[0]
    path = os.path.join(LIBDIR, "lib_ccf.so")
    if not os.path.exists(path):
        raise RuntimeError(f"irs_b200: CUDA library {path} is missing; build it with `python -m irs_b200.build` "
                           "(there is no CPU fallback)")
    lib = C.CDLL(path)
    vp, D, I, S = C.c_void_p, C.c_double, C.c_int, C.c_char_p
    lib.init.argtypes, lib.init.restype = [], vp
    for group, T in ((_FLOAT_FIELDS, D), (_INT_FIELDS, I), (_STR_FIELDS, S)):
        for f in group:
            getattr(lib, f"set_{f}").argtypes, getattr(lib, f"set_{f}").restype = [vp, T], None
            getattr(lib, f"get_{f}").argtypes, getattr(lib, f"get_{f}").restype = [vp], T
    for name, res in (("get_num_roots", I), ("get_corner_x1", D), ("get_corner_x2", D), ("get_t_ccs", D)):
        getattr(lib, name).argtypes, getattr(lib, name).restype = [vp], res
    for name in ("get_stars", "get_critical_curves", "get_caustics", "get_mu_length_scales"):
        getattr(lib, name).argtypes, getattr(lib, name).restype = [vp], C.POINTER(D)
    for name in ("run", "save"):
        getattr(lib, name).argtypes, getattr(lib, name).restype = [vp, I], C.c_bool
    lib.destroy.argtypes, lib.destroy.restype = [vp], None
    lib.set_num_iters.argtypes, lib.set_num_iters.restype = [vp, I, I], None
    lib.get_value.argtypes, lib.get_value.restype = [vp, S], D
    _lib_cache.append(lib)
    return lib


class CCF:
    def __init__(self, kappa_tot: float = None, shear: float = None, smooth_fraction: float = None,
                 kappa_star: float = None, theta_star: float = None, mass_function: str = None,
                 m_solar: float = None, m_lower: float = None, m_upper: float = None, rectangular: bool = None,
                 approx: bool = None, safety_scale: float = None, num_stars: int = None, starfile: str = None,
                 num_phi: int = None, num_branches: int = None, random_seed: int = None, write_stars: bool = None,
                 write_critical_curves: bool = None, write_caustics: bool = None, write_length_scales: bool = None,
                 outfile_prefix: str = None, verbose: int = 0, num_iters: tuple = None):
        self.lib = load()
        self.obj = self.lib.init()
        self.verbose = verbose
        self.kappa_tot = kappa_tot
        self.shear = shear
        if starfile is None:
            if smooth_fraction is not None and kappa_star is None:
                kappa_star = (1 - smooth_fraction) * self.kappa_tot
            self.kappa_star = kappa_star
            self.theta_star = theta_star
            self.mass_function = mass_function
            self.m_solar = m_solar
            self.m_lower = m_lower
            self.m_upper = m_upper
            if self.m_lower > self.m_upper:
                raise ValueError("m_lower must be <= m_upper")
            self.num_stars = num_stars
            self.random_seed = random_seed
        self.rectangular = rectangular
        self.approx = approx
        self.safety_scale = safety_scale
        self.starfile = starfile
        self.num_phi = num_phi
        if self.num_phi % 2 != 0:
            raise ValueError("num_phi must be an even number")
        self.num_branches = num_branches
        if self.num_phi % (2 * self.num_branches) != 0:
            raise ValueError("num_phi must be a multiple of 2 * num_branches")
        self.write_stars = write_stars
        self.write_critical_curves = write_critical_curves
        self.write_caustics = write_caustics
        self.write_mu_length_scales = write_length_scales
        self.outfile_prefix = outfile_prefix
        if num_iters is not None:
            self.lib.set_num_iters(self.obj, int(num_iters[0]), int(num_iters[1]))
        self.critical_curves = self.caustics = self.mu_length_scales = self.stars = None

    # ---- validated inputs (microlensing/CCF/ccf.py property setters)
    def _set(self, name, value, check=None, conv=float):
        if value is None:
            return
        if check is not None:
            msg = check(value)
            if msg:
                raise ValueError(msg)
        getattr(self.lib, f"set_{name}")(self.obj, conv(value))

    kappa_tot = property(lambda s: s.lib.get_kappa_tot(s.obj),
                         lambda s, v: s._set("kappa_tot", v, lambda v: "kappa_tot must be >= 0" if v < 0 else None))
    shear = property(lambda s: s.lib.get_shear(s.obj), lambda s, v: s._set("shear", v))

    @property
    def kappa_star(self):
        return self.lib.get_kappa_star(self.obj)

    @kappa_star.setter
    def kappa_star(self, value):
        if value is None:
            return
        if value < 0:
            raise ValueError("kappa_star must be >= 0")
        if value > self.kappa_tot:
            raise ValueError("kappa_star must be <= kappa_tot")
        self.lib.set_kappa_star(self.obj, float(value))

    theta_star = property(lambda s: s.lib.get_theta_star(s.obj),
                          lambda s, v: s._set("theta_star", v, lambda v: "theta_star must be >= 0" if v < 0 else None))

    @property
    def mass_function(self):
        return self.lib.get_mass_function(self.obj).decode("utf-8")

    @mass_function.setter
    def mass_function(self, value):
        if value is None:
            return
        if value.lower() not in _MASS_FUNCTIONS:
            raise ValueError("mass_function must be equal, uniform, Salpeter, Kroupa, or optical_depth")
        self.lib.set_mass_function(self.obj, value.lower().encode("utf-8"))

    m_solar = property(lambda s: s.lib.get_m_solar(s.obj),
                       lambda s, v: s._set("m_solar", v, lambda v: "m_solar must be >= 0" if v < 0 else None))
    m_lower = property(lambda s: s.lib.get_m_lower(s.obj),
                       lambda s, v: s._set("m_lower", v, lambda v: "m_lower must be >= 0" if v < 0 else None))
    m_upper = property(lambda s: s.lib.get_m_upper(s.obj),
                       lambda s, v: s._set("m_upper", v, lambda v: "m_upper must be >= 0" if v < 0 else None))
    rectangular = property(lambda s: bool(s.lib.get_rectangular(s.obj)),
                           lambda s, v: s._set("rectangular", v, conv=int))
    approx = property(lambda s: bool(s.lib.get_approx(s.obj)), lambda s, v: s._set("approx", v, conv=int))
    safety_scale = property(lambda s: s.lib.get_safety_scale(s.obj),
                            lambda s, v: s._set("safety_scale", v,
                                                lambda v: "safety_scale must be >= 1.1" if v < 1.1 else None))
    num_stars = property(lambda s: s.lib.get_num_stars(s.obj),
                         lambda s, v: s._set("num_stars", v, lambda v: "num_stars must be >= 1" if v < 1 else None,
                                             int))

    @property
    def starfile(self):
        return self.lib.get_starfile(self.obj).decode("utf-8")

    @starfile.setter
    def starfile(self, value):
        if value is not None:
            self.lib.set_starfile(self.obj, value.encode("utf-8"))

    num_phi = property(lambda s: s.lib.get_num_phi(s.obj),
                       lambda s, v: s._set("num_phi", v, lambda v: "num_phi must be >= 1" if v < 1 else None, int))
    num_branches = property(lambda s: s.lib.get_num_branches(s.obj),
                            lambda s, v: s._set("num_branches", v,
                                                lambda v: "num_branches must be >= 1" if v < 1 else None, int))
    random_seed = property(lambda s: s.lib.get_random_seed(s.obj), lambda s, v: s._set("random_seed", v, conv=int))
    write_stars = property(lambda s: bool(s.lib.get_write_stars(s.obj)),
                           lambda s, v: s._set("write_stars", v, conv=int))
    write_critical_curves = property(lambda s: bool(s.lib.get_write_critical_curves(s.obj)),
                                     lambda s, v: s._set("write_critical_curves", v, conv=int))
    write_caustics = property(lambda s: bool(s.lib.get_write_caustics(s.obj)),
                              lambda s, v: s._set("write_caustics", v, conv=int))
    write_mu_length_scales = property(lambda s: bool(s.lib.get_write_mu_length_scales(s.obj)),
                                      lambda s, v: s._set("write_mu_length_scales", v, conv=int))

    @property
    def outfile_prefix(self):
        return self.lib.get_outfile_prefix(self.obj).decode("utf-8")

    @outfile_prefix.setter
    def outfile_prefix(self, value):
        if value is not None:
            self.lib.set_outfile_prefix(self.obj, value.encode("utf-8"))

    # ---- derived values
    @property
    def mu_ave(self):
        return 1 / ((1 - self.kappa_tot) ** 2 - self.shear ** 2)

    @property
    def stellar_fraction(self):
        return self.kappa_star / self.kappa_tot

    @property
    def smooth_fraction(self):
        return 1 - self.kappa_star / self.kappa_tot

    @property
    def corner(self):
        return (self.lib.get_corner_x1(self.obj), self.lib.get_corner_x2(self.obj))

    @property
    def num_roots(self):
        return self.lib.get_num_roots(self.obj)

    @property
    def t_ccs(self):
        return self.lib.get_t_ccs(self.obj)

    def value(self, name: str) -> float:
        return float(self.lib.get_value(self.obj, name.encode()))

    # ---- run / save
    def run(self):
        if not self.lib.run(self.obj, self.verbose):
            raise Exception("Error running CCF")
        rows, cols = self.num_roots * self.num_branches, self.num_phi // self.num_branches + 1
        self.critical_curves = np.ctypeslib.as_array(self.lib.get_critical_curves(self.obj),
                                                     shape=(rows, cols, 2)).copy()
        self.caustics = (np.ctypeslib.as_array(self.lib.get_caustics(self.obj), shape=(rows, cols, 2)).copy()
                         if self.write_caustics else None)
        self.mu_length_scales = (np.ctypeslib.as_array(self.lib.get_mu_length_scales(self.obj),
                                                       shape=(rows, cols)).copy()
                                 if self.write_mu_length_scales else None)
        self.stars = np.ctypeslib.as_array(self.lib.get_stars(self.obj), shape=(self.num_stars, 3)).copy()

    def save(self):
        if not self.lib.save(self.obj, self.verbose):
            raise Exception("Error saving CCF")

    def close(self):
        if getattr(self, "obj", None):
            self.lib.destroy(self.obj)
            self.obj = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

"""Python interface of the irs_b200 map engine.

`IPM` mirrors the reference wrapper microlensing/IPM/ipm.py (class IPM,
lines 7-473): the same constructor keywords, validated property setters that
raise ValueError, run() raising Exception("Error running IPM") on failure,
numpy copies of the maps and stars, t_shoot_cells, magnitudes and save().
`IRS` offers the same interface for inverse ray shooting (the reference has no
IRS wrapper; its IRS class is include/irs.cuh), with integer ray-count maps.

Extensions beyond the reference: expansion_order (0 = the reference's
formula), precision (0 = default form of the library, 1 = FP64 plain,
2 = FP32), set_stars() for a star field in memory, and close().
"""
from __future__ import annotations

import ctypes as C
import sys

import numpy as np

from . import _lib

_MASS_FUNCTIONS = ["equal", "uniform", "salpeter", "kroupa", "optical_depth"]


class _MapMaker:
    _kind = "ipm"
    _label = "IPM"

    def __init__(self, kappa_tot: float = None, shear: float = None, smooth_fraction: float = None,
                 kappa_star: float = None, theta_star: float = None, mass_function: str = None,
                 m_solar: float = None, m_lower: float = None, m_upper: float = None,
                 light_loss: float = None, rectangular: bool = None, approx: bool = None,
                 safety_scale: float = None, starfile: str = None, center_y1: float = None,
                 center_y2: float = None, half_length_y1: float = None, half_length_y2: float = None,
                 num_pixels_y1: int = None, num_pixels_y2: int = None, num_rays_y: int = None,
                 random_seed: int = None, write_stars: bool = None, write_maps: bool = None,
                 write_parities: bool = None, write_histograms: bool = None, outfile_prefix: str = None,
                 verbose: int = 0, is_double: bool = False, expansion_order: int = None,
                 precision: int = None, _handle=None):
        self.is_double = bool(is_double)
        self.lib = _lib.load(self._kind, self.is_double)
        self._T = C.c_double if self.is_double else C.c_float
        self._np_T = np.float64 if self.is_double else np.float32
        # _handle: an object owned elsewhere (the base map of an adaptive run)
        self._owned = _handle is None
        self.obj = self.lib.init() if _handle is None else _handle
        self.verbose = verbose
        self._host_stars = None

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
            self.random_seed = random_seed
        self.light_loss = light_loss
        self.rectangular = rectangular
        self.approx = approx
        self.safety_scale = safety_scale
        self.starfile = starfile
        self.center_y1 = center_y1
        self.center_y2 = center_y2
        self.half_length_y1 = half_length_y1
        self.half_length_y2 = half_length_y2
        self.num_pixels_y1 = num_pixels_y1
        self.num_pixels_y2 = num_pixels_y2
        self.num_rays_y = num_rays_y
        self.write_stars = write_stars
        self.write_maps = write_maps
        self.write_parities = write_parities
        self.write_histograms = write_histograms
        self.outfile_prefix = outfile_prefix
        if expansion_order is not None:
            self.expansion_order = expansion_order
        if precision is not None:
            self.precision = precision

    # ------------------------------------------------------------ lifetime
    def close(self):
        if getattr(self, "obj", None):
            if getattr(self, "_owned", True):
                self.lib.destroy(self.obj)
            self.obj = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ helpers
    def _get(self, name):
        return getattr(self.lib, f"get_{name}")(self.obj)

    def _set(self, name, value):
        getattr(self.lib, f"set_{name}")(self.obj, value)

    # ------------------------------------------------------------ parameters
    @property
    def kappa_tot(self):
        return self._get("kappa_tot")

    @kappa_tot.setter
    def kappa_tot(self, value):
        if value is not None:
            if value < 0:
                raise ValueError("kappa_tot must be >= 0")
            self._set("kappa_tot", value)

    @property
    def shear(self):
        return self._get("shear")

    @shear.setter
    def shear(self, value):
        if value is not None:
            self._set("shear", value)

    @property
    def mu_ave(self):
        return 1 / ((1 - self.kappa_tot) ** 2 - self.shear ** 2)

    @property
    def kappa_star(self):
        return self._get("kappa_star")

    @kappa_star.setter
    def kappa_star(self, value):
        if value is not None:
            if value < 0:
                raise ValueError("kappa_star must be >= 0")
            elif value > self.kappa_tot:
                raise ValueError("kappa_star must be <= kappa_tot")
            self._set("kappa_star", value)

    @property
    def stellar_fraction(self):
        return self.kappa_star / self.kappa_tot

    @property
    def smooth_fraction(self):
        return 1 - self.kappa_star / self.kappa_tot

    @property
    def theta_star(self):
        return self._get("theta_star")

    @theta_star.setter
    def theta_star(self, value):
        if value is not None:
            if value < 0:
                raise ValueError("theta_star must be >= 0")
            self._set("theta_star", value)

    @property
    def mass_function(self):
        return self._get("mass_function").decode("utf-8")

    @mass_function.setter
    def mass_function(self, value):
        if value is not None:
            if value.lower() not in _MASS_FUNCTIONS:
                raise ValueError("mass_function must be equal, uniform, Salpeter, Kroupa, or optical_depth")
            self._set("mass_function", value.lower().encode("utf-8"))

    @property
    def m_solar(self):
        return self._get("m_solar")

    @m_solar.setter
    def m_solar(self, value):
        if value is not None:
            if value < 0:
                raise ValueError("m_solar must be >= 0")
            self._set("m_solar", value)

    @property
    def m_lower(self):
        return self._get("m_lower")

    @m_lower.setter
    def m_lower(self, value):
        if value is not None:
            if value < 0:
                raise ValueError("m_lower must be >= 0")
            self._set("m_lower", value)

    @property
    def m_upper(self):
        return self._get("m_upper")

    @m_upper.setter
    def m_upper(self, value):
        if value is not None:
            if value < 0:
                raise ValueError("m_upper must be >= 0")
            self._set("m_upper", value)

    @property
    def light_loss(self):
        return self._get("light_loss")

    @light_loss.setter
    def light_loss(self, value):
        if value is not None:
            if value < 0:
                raise ValueError("light_loss must be > 0")
            elif value > 0.01:
                raise ValueError("light_loss must be <= 0.01")
            self._set("light_loss", value)

    @property
    def rectangular(self):
        return bool(self._get("rectangular"))

    @rectangular.setter
    def rectangular(self, value):
        if value is not None:
            self._set("rectangular", int(value))

    @property
    def approx(self):
        return bool(self._get("approx"))

    @approx.setter
    def approx(self, value):
        if value is not None:
            self._set("approx", int(value))

    @property
    def safety_scale(self):
        return self._get("safety_scale")

    @safety_scale.setter
    def safety_scale(self, value):
        if value is not None:
            if value < 1.1:
                raise ValueError("safety_scale must be >= 1.1")
            self._set("safety_scale", value)

    @property
    def starfile(self):
        return self._get("starfile").decode("utf-8")

    @starfile.setter
    def starfile(self, value):
        if value is not None:
            self._set("starfile", value.encode("utf-8"))

    @property
    def center_y1(self):
        return self._get("center_y1")

    @center_y1.setter
    def center_y1(self, value):
        if value is not None:
            self._set("center_y1", value)

    @property
    def center_y2(self):
        return self._get("center_y2")

    @center_y2.setter
    def center_y2(self, value):
        if value is not None:
            self._set("center_y2", value)

    @property
    def center(self):
        return (self.center_y1, self.center_y2)

    @property
    def half_length_y1(self):
        return self._get("half_length_y1")

    @half_length_y1.setter
    def half_length_y1(self, value):
        if value is not None:
            if value < 0:
                raise ValueError("half_length_y1 must be > 0")
            self._set("half_length_y1", value)

    @property
    def half_length_y2(self):
        return self._get("half_length_y2")

    @half_length_y2.setter
    def half_length_y2(self, value):
        if value is not None:
            if value < 0:
                raise ValueError("half_length_y2 must be > 0")
            self._set("half_length_y2", value)

    @property
    def half_length(self):
        return (self.half_length_y1, self.half_length_y2)

    @property
    def num_pixels_y1(self):
        return self._get("num_pixels_y1")

    @num_pixels_y1.setter
    def num_pixels_y1(self, value):
        if value is not None:
            if value < 1:
                raise ValueError("num_pixels_y1 must be >= 1")
            self._set("num_pixels_y1", value)

    @property
    def num_pixels_y2(self):
        return self._get("num_pixels_y2")

    @num_pixels_y2.setter
    def num_pixels_y2(self, value):
        if value is not None:
            if value < 1:
                raise ValueError("num_pixels_y2 must be >= 1")
            self._set("num_pixels_y2", value)

    @property
    def num_pixels(self):
        return (self.num_pixels_y1, self.num_pixels_y2)

    @property
    def pixel_scales(self):
        return (2 * self.half_length[0] / self.num_pixels[0], 2 * self.half_length[1] / self.num_pixels[1])

    @property
    def num_rays_y(self):
        return self._get("num_rays_y")

    @num_rays_y.setter
    def num_rays_y(self, value):
        if value is not None:
            if value < 1:
                raise ValueError("num_rays_y must be >= 1")
            self._set("num_rays_y", value)

    @property
    def random_seed(self):
        return self._get("random_seed")

    @random_seed.setter
    def random_seed(self, value):
        if value is not None:
            self._set("random_seed", value)

    @property
    def write_stars(self):
        return bool(self._get("write_stars"))

    @write_stars.setter
    def write_stars(self, value):
        if value is not None:
            self._set("write_stars", int(value))

    @property
    def write_maps(self):
        return bool(self._get("write_maps"))

    @write_maps.setter
    def write_maps(self, value):
        if value is not None:
            self._set("write_maps", int(value))

    @property
    def write_parities(self):
        return bool(self._get("write_parities"))

    @write_parities.setter
    def write_parities(self, value):
        if value is not None:
            self._set("write_parities", int(value))

    @property
    def write_histograms(self):
        return bool(self._get("write_histograms"))

    @write_histograms.setter
    def write_histograms(self, value):
        if value is not None:
            self._set("write_histograms", int(value))

    @property
    def outfile_prefix(self):
        return self._get("outfile_prefix").decode("utf-8")

    @outfile_prefix.setter
    def outfile_prefix(self, value):
        if value is not None:
            self._set("outfile_prefix", value.encode("utf-8"))

    # ------------------------------------------------------------ extensions
    @property
    def expansion_order(self):
        return self.lib.get_expansion_order(self.obj)

    @expansion_order.setter
    def expansion_order(self, value):
        if value is not None:
            if value != 0 and not (3 <= value <= 31):
                raise ValueError("expansion_order must be 0 (derived) or in [3, 31]")
            self.lib.set_expansion_order(self.obj, int(value))

    @property
    def precision(self):
        return self.lib.get_precision(self.obj)

    @precision.setter
    def precision(self, value):
        if value not in (0, 1, 2):
            raise ValueError("precision must be 0 (default), 1 (FP64) or 2 (FP32)")
        self.lib.set_precision(self.obj, int(value))

    def set_stars(self, stars, rectangular: bool, corner, theta_star: float = 1.0):
        """Use a star field held in memory: stars is (N, 3) with x1, x2, mass.

        corner is (corner_x1, corner_x2) for a rectangular field, or (radius, 0)
        for a circular one, as in a star file. stars=None reverts to generation.
        """
        if stars is None:
            self.lib.set_stars(self.obj, None, 0, 0, 0.0, 0.0, 1.0)
            self._host_stars = None
            return
        a = np.ascontiguousarray(np.asarray(stars, dtype=self._np_T).reshape(-1, 3))
        self._host_stars = a
        self.lib.set_stars(self.obj, a.ctypes.data_as(C.POINTER(self._T)), int(a.shape[0]), int(bool(rectangular)),
                           float(corner[0]), float(corner[1]), float(theta_star))

    def value(self, name: str) -> float:
        """A derived or run-time quantity by name (see get_value in the C ABI)."""
        return self.lib.get_value(self.obj, name.encode("utf-8"))

    def derive(self):
        """Validate inputs and compute derived parameters without GPU work."""
        if not self.lib.derive(self.obj):
            raise ValueError(f"Invalid {self._label} parameters")

    @property
    def t_pipeline(self):
        return self.lib.get_t_pipeline(self.obj)

    def rerun(self, repeats: int = 1) -> float:
        """Re-run tree, expansions and shoot on the device-resident star field of
        the last run(); returns the summed device seconds."""
        t = C.c_double(0.0)
        if not self.lib.rerun(self.obj, int(repeats), C.byref(t)):
            raise Exception(f"Error re-running {self._label}")
        return t.value

    # ------------------------------------------------------------ results
    @property
    def num_stars(self):
        return self.lib.get_num_stars(self.obj)

    @property
    def corner(self):
        return (self.lib.get_corner_x1(self.obj), self.lib.get_corner_x2(self.obj))

    def _map(self, which):
        """A numpy copy of the last run's map (0 total, 1 minima, 2 saddles),
        filled by the library's multi-threaded copy; None if it does not exist."""
        ptr = getattr(self.lib, ("get_pixels", "get_pixels_minima", "get_pixels_saddles")[which])(self.obj)
        if not ptr:
            return None
        out = np.empty((self.num_pixels_y2, self.num_pixels_y1), dtype=ptr._type_)
        if not self.lib.copy_pixels(self.obj, which, out.ctypes.data_as(C.POINTER(ptr._type_))):
            raise Exception(f"Error copying the {self._label} map")
        return out

    def run(self):
        # the map lands in a fresh numpy array during run(), chunk by chunk as
        # it arrives from the device
        pix_t = self.lib.get_pixels.restype._type_
        shape = (self.num_pixels_y2, self.num_pixels_y1)
        out = getattr(self, "magnifications", None)
        # the previous map's memory is reused when nothing outside this object
        # refers to it (no caller variable or view: references here are the
        # attribute, `out` and getrefcount's argument), so that a loop of runs
        # does not fault fresh pages in for every map
        if not (isinstance(out, np.ndarray) and out.shape == shape and out.dtype == np.dtype(pix_t)
                and out.base is None and out.flags.c_contiguous and out.flags.writeable
                and sys.getrefcount(out) <= 3):
            out = np.empty(shape, dtype=pix_t)
        self.magnifications = None
        self.lib.set_pixels_out(self.obj, out.ctypes.data_as(C.POINTER(pix_t)))
        ok = self.lib.run(self.obj, self.verbose)
        self.lib.set_pixels_out(self.obj, None)
        if not ok:
            raise Exception(f"Error running {self._label}")
        self.magnifications = out
        if self.write_parities:
            self.magnifications_minima = self._map(1)
            self.magnifications_saddles = self._map(2)
        else:
            self.magnifications_minima = None
            self.magnifications_saddles = None
        self.stars = np.ctypeslib.as_array(self.lib.get_stars(self.obj), shape=(self.num_stars, 3)).copy()

    def save(self):
        if not self.lib.save(self.obj, self.verbose):
            raise Exception(f"Error saving {self._label}")

    def _magnitudes(self, m):
        if m is None:
            raise ValueError("map is None")
        return -2.5 * np.log10(m / np.abs(self.mu_ave))

    @property
    def magnitudes(self):
        return self._magnitudes(self._mu(self.magnifications))

    @property
    def magnitudes_minima(self):
        return self._magnitudes(self._mu(self.magnifications_minima))

    @property
    def magnitudes_saddles(self):
        return self._magnitudes(self._mu(self.magnifications_saddles))

    def _mu(self, m):
        return m

    def plot_map(self, fig, ax, **kwargs):
        kwargs.setdefault("vmin", np.percentile(self.magnitudes.ravel(), 2.5))
        kwargs.setdefault("vmax", np.percentile(self.magnitudes.ravel(), 97.5))
        kwargs.setdefault("cmap", "viridis_r")
        extent = [(self.center[0] - self.half_length[0]) / self.theta_star,
                  (self.center[0] + self.half_length[0]) / self.theta_star,
                  (self.center[1] - self.half_length[1]) / self.theta_star,
                  (self.center[1] + self.half_length[1]) / self.theta_star]
        img = ax.imshow(self.magnitudes, extent=extent, **kwargs)
        cbar = fig.colorbar(img, label="microlensing $\\Delta m$ (magnitudes)")
        cbar.ax.invert_yaxis()
        ax.set_xlabel("$y_1 / \\theta_★$")
        ax.set_ylabel("$y_2 / \\theta_★$")
        ax.set_aspect(self.half_length[0] / self.half_length[1])

    def plot_hist(self, fig, ax, bins=None, **kwargs):
        if bins is None:
            vmin, vmax = (np.min(self.magnitudes), np.max(self.magnitudes))
            bins = np.arange(vmin - 0.01, vmax + 0.01, 0.01)
        ax.hist(self.magnitudes.ravel(), bins=bins, density=True, **kwargs)
        ax.set_xlabel("microlensing $\\Delta m$ (magnitudes)")
        ax.set_ylabel("p($\\Delta m$)")
        ax.invert_xaxis()

    # ------------------------------------------------------------ diagnostics
    def tree_arrays(self):
        """(ints[n,8], geom[n,3], nbr[n,8], sil[n,27], dil[n,5]) of the last run's tree."""
        n = self.lib.get_tree_num_nodes(self.obj)
        ints = np.zeros((n, 8), np.int32)
        geom = np.zeros((n, 3), np.float64)
        nbr = np.zeros((n, 8), np.int32)
        sil = np.zeros((n, 27), np.int32)
        dil = np.zeros((n, 5), np.int32)
        ok = self.lib.copy_tree(self.obj, ints.ctypes.data, geom.ctypes.data, nbr.ctypes.data, sil.ctypes.data,
                                dil.ctypes.data)
        if not ok:
            raise RuntimeError("copy_tree failed")
        return ints, geom, nbr, sil, dil

    def coeffs(self):
        n = self.lib.get_tree_num_nodes(self.obj)
        p = self.expansion_order
        mult = np.zeros((n, p + 1, 2), np.float64)
        loc = np.zeros((n, p + 1, 2), np.float64)
        if not self.lib.copy_coeffs(self.obj, mult.ctypes.data, loc.ctypes.data):
            raise RuntimeError("copy_coeffs failed")
        return mult[..., 0] + 1j * mult[..., 1], loc[..., 0] + 1j * loc[..., 1]


class IPM(_MapMaker):
    """Inverse polygon mapping (interface of microlensing.IPM.IPM)."""
    _kind = "ipm"
    _label = "IPM"

    @property
    def t_shoot_cells(self):
        return self.lib.get_t_shoot_cells(self.obj)

    def vertices(self):
        """Source positions of the cell-corner lattice, shape (ny+1, nx+1, 2), pixel units, row axis flipped."""
        n = self.lib.get_num_vertices(self.obj)
        v = np.zeros((n, 2), np.float64)
        if n and not self.lib.copy_vertices(self.obj, v.ctypes.data):
            raise RuntimeError("copy_vertices failed")
        nx = int(self.value("num_ray_threads_1")) + 1
        return v.reshape(-1, nx, 2)

    def fixed_maps(self):
        """Fixed-point accumulators (uint64, 2^32 per unit): total, or (minima, saddles) with parities."""
        shape = (self.num_pixels_y2, self.num_pixels_y1)
        a = np.zeros(shape, np.uint64)
        b = np.zeros(shape, np.uint64)
        c = np.zeros(shape, np.uint64)
        if not self.lib.copy_fixed_maps(self.obj, a.ctypes.data, b.ctypes.data, c.ctypes.data):
            raise RuntimeError("copy_fixed_maps failed")
        return (b, c) if self.write_parities else a


class IRS(_MapMaker):
    """Inverse ray shooting with integer ray-count maps (include/irs.cuh of the reference)."""
    _kind = "irs"
    _label = "IRS"

    @property
    def t_shoot_rays(self):
        return self.lib.get_t_shoot_rays(self.obj)

    @property
    def num_rays_shot(self):
        return self.lib.get_num_rays_shot(self.obj)

    @property
    def num_rays_received(self):
        return self.lib.get_num_rays_received(self.obj)

    def _mu(self, m):
        return None if m is None else m / self.num_rays_y

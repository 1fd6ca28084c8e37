"""Number-of-caustic-crossings maps (NCC) on the GPU.

`NCC` mirrors the reference wrapper microlensing/NCC/ncc.py (class NCC): the
same constructor keywords, validated property setters that raise ValueError,
run() raising Exception("Error running NCC") on failure, a numpy copy of the
map (num_caustic_crossings) and save(). The library is
irs_b200/lib/lib_ncc.so (double), whose symbols are those of the reference's
src/lib_ncc.cu. The input is <infile_prefix>ccf_caustics.bin, as a CCF run
writes it, or caustics given in memory (set_caustics, e.g. CCF.caustics).
Unlike the reference wrapper the infile prefix is not lower-cased.

Extensions: set_caustics(), value(name) and close().
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import LIBDIR

_lib_cache = []
_FLOAT = ["center_y1", "center_y2", "half_length_y1", "half_length_y2"]
_INT = ["num_pixels_y1", "num_pixels_y2", "over_sample", "write_maps", "write_histograms"]
_STR = ["infile_prefix", "outfile_prefix"]
# the exports of the reference's src/lib_ncc.cu (lines 15-44)
REFERENCE_NCC_SYMBOLS = (["init", "run", "save", "get_num_crossings"] +
                         [f"{a}_{f}" for f in _FLOAT + _INT + _STR for a in ("set", "get")])


def load():
    """Load (once) and bind lib_ncc.so; raises if it is missing."""
    if _lib_cache:
        return _lib_cache[0]
    path = os.path.join(LIBDIR, "lib_ncc.so")
    if not os.path.exists(path):
        raise RuntimeError(f"irs_b200: CUDA library {path} is missing; build it with `python -m irs_b200.build` "
                           "(there is no CPU fallback)")
    lib = C.CDLL(path)
    vp, D, I, S = C.c_void_p, C.c_double, C.c_int, C.c_char_p
    lib.init.argtypes, lib.init.restype = [], vp
    for group, T in ((_FLOAT, D), (_INT, I), (_STR, S)):
        for f in group:
            getattr(lib, f"set_{f}").argtypes, getattr(lib, f"set_{f}").restype = [vp, T], None
            getattr(lib, f"get_{f}").argtypes, getattr(lib, f"get_{f}").restype = [vp], T
    lib.get_num_crossings.argtypes, lib.get_num_crossings.restype = [vp], C.POINTER(C.c_int)
    for name in ("run", "save"):
        getattr(lib, name).argtypes, getattr(lib, name).restype = [vp, I], C.c_bool
    lib.destroy.argtypes, lib.destroy.restype = [vp], None
    lib.set_caustics.argtypes, lib.set_caustics.restype = [vp, vp, I, I], None
    lib.get_value.argtypes, lib.get_value.restype = [vp, S], D
    _lib_cache.append(lib)
    return lib


class NCC:
    def __init__(self, infile_prefix: str = None, center_y1: float = None, center_y2: float = None,
                 half_length_y1: float = None, half_length_y2: float = None, num_pixels_y1: int = None,
                 num_pixels_y2: int = None, over_sample: int = None, write_maps: bool = None,
                 write_histograms: bool = None, outfile_prefix: str = None, verbose: int = 0):
        self.lib = load()
        self.obj = self.lib.init()
        self.verbose = verbose
        self.infile_prefix = infile_prefix
        self.center_y1 = center_y1
        self.center_y2 = center_y2
        self.half_length_y1 = half_length_y1
        self.half_length_y2 = half_length_y2
        self.num_pixels_y1 = num_pixels_y1
        self.num_pixels_y2 = num_pixels_y2
        self.over_sample = over_sample
        self.write_maps = write_maps
        self.write_histograms = write_histograms
        self.outfile_prefix = outfile_prefix
        self.num_caustic_crossings = None

    def _set(self, name, value, check=None, conv=float):
        if value is None:
            return
        if check is not None:
            msg = check(value)
            if msg:
                raise ValueError(msg)
        getattr(self.lib, f"set_{name}")(self.obj, conv(value))

    @property
    def infile_prefix(self):
        return self.lib.get_infile_prefix(self.obj).decode("utf-8")

    @infile_prefix.setter
    def infile_prefix(self, value):
        if value is not None:
            self.lib.set_infile_prefix(self.obj, value.encode("utf-8"))

    center_y1 = property(lambda s: s.lib.get_center_y1(s.obj), lambda s, v: s._set("center_y1", v))
    center_y2 = property(lambda s: s.lib.get_center_y2(s.obj), lambda s, v: s._set("center_y2", v))
    half_length_y1 = property(lambda s: s.lib.get_half_length_y1(s.obj),
                              lambda s, v: s._set("half_length_y1", v,
                                                  lambda v: "half_length_y1 must be > 0" if v <= 0 else None))
    half_length_y2 = property(lambda s: s.lib.get_half_length_y2(s.obj),
                              lambda s, v: s._set("half_length_y2", v,
                                                  lambda v: "half_length_y2 must be > 0" if v <= 0 else None))
    num_pixels_y1 = property(lambda s: s.lib.get_num_pixels_y1(s.obj),
                             lambda s, v: s._set("num_pixels_y1", v,
                                                 lambda v: "num_pixels_y1 must be >= 1" if v < 1 else None, int))
    num_pixels_y2 = property(lambda s: s.lib.get_num_pixels_y2(s.obj),
                             lambda s, v: s._set("num_pixels_y2", v,
                                                 lambda v: "num_pixels_y2 must be >= 1" if v < 1 else None, int))
    over_sample = property(lambda s: s.lib.get_over_sample(s.obj),
                           lambda s, v: s._set("over_sample", v,
                                               lambda v: "over_sample must be >= 0" if v < 0 else None, int))
    write_maps = property(lambda s: bool(s.lib.get_write_maps(s.obj)), lambda s, v: s._set("write_maps", v, conv=int))
    write_histograms = property(lambda s: bool(s.lib.get_write_histograms(s.obj)),
                                lambda s, v: s._set("write_histograms", v, conv=int))

    @property
    def outfile_prefix(self):
        return self.lib.get_outfile_prefix(self.obj).decode("utf-8")

    @outfile_prefix.setter
    def outfile_prefix(self, value):
        if value is not None:
            self.lib.set_outfile_prefix(self.obj, value.encode("utf-8"))

    @property
    def center(self):
        return (self.center_y1, self.center_y2)

    @property
    def half_length(self):
        return (self.half_length_y1, self.half_length_y2)

    @property
    def num_pixels(self):
        return (self.num_pixels_y1, self.num_pixels_y2)

    @property
    def pixel_scales(self):
        return (2 * self.half_length[0] / self.num_pixels[0], 2 * self.half_length[1] / self.num_pixels[1])

    def set_caustics(self, caustics):
        """Caustics in memory, (rows, cols) complex or (rows, cols, 2) real
        (e.g. CCF.caustics); None returns to the input file."""
        if caustics is None:
            self.lib.set_caustics(self.obj, None, 0, 0)
            return
        c = np.asarray(caustics)
        if c.ndim == 3:
            c = c[..., 0] + 1j * c[..., 1]
        self._caus = np.ascontiguousarray(c, np.complex128)
        self.lib.set_caustics(self.obj, self._caus.ctypes.data, self._caus.shape[0], self._caus.shape[1])

    def value(self, name: str) -> float:
        return float(self.lib.get_value(self.obj, name.encode()))

    def run(self):
        if not self.lib.run(self.obj, self.verbose):
            raise Exception("Error running NCC")
        self.num_caustic_crossings = np.ctypeslib.as_array(self.lib.get_num_crossings(self.obj),
                                                           shape=(self.num_pixels_y2, self.num_pixels_y1)).copy()

    def save(self):
        if not self.lib.save(self.obj, self.verbose):
            raise Exception("Error saving NCC")

    def close(self):
        if getattr(self, "obj", None):
            self.lib.destroy(self.obj)
            self.obj = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

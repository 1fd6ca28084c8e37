"""Batches of IPM realizations through one graph-captured device pipeline.

A batch holds many realizations of uneven size (own seed, convergence, shear,
smooth fraction, mass function; one map size). Their star fields, quadtrees,
expansions, lattice passes and depositions run in shared launches captured
once in a CUDA graph (the C ABI's batch_* entry points). Each realization's
map equals a single IPM run of the same inputs at the same expansion order in
the FP32 form.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .mapmaker import IPM


class BatchIPM:
    def __init__(self, realizations, is_double: bool = False, expansion_order: int = 0,
                 corner_capacity: int = 0):
        self.is_double = bool(is_double)
        self.lib = _lib.load("ipm", self.is_double)
        self._np_T = np.float64 if self.is_double else np.float32
        self.h = self.lib.batch_init()
        self.members = []
        for kw in realizations:
            m = IPM(**kw, is_double=self.is_double)  # validates like a single run
            self.lib.batch_add(self.h, m.obj)
            self.members.append(m)
        self.lib.batch_set_expansion_order(self.h, int(expansion_order))
        self.lib.batch_set_corner_capacity(self.h, int(corner_capacity))

    def __len__(self):
        return self.lib.batch_size(self.h)

    def close(self):
        if getattr(self, "h", None):
            self.lib.batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, verbose: int = 0):
        if not self.lib.batch_run(self.h, int(verbose)):
            raise Exception("Error running batch")

    def rerun(self, repeats: int = 1) -> float:
        sec = C.c_double(0)
        if not self.lib.batch_rerun(self.h, int(repeats), C.byref(sec)):
            raise Exception("Error running batch")
        return sec.value

    def value(self, name: str, r: int = -1) -> float:
        return self.lib.batch_get_value(self.h, int(r), name.encode())

    @property
    def maps(self) -> np.ndarray:
        R = len(self)
        npx, npy = int(self.value("num_pixels_y1")), int(self.value("num_pixels_y2"))
        out = np.empty((R, npy, npx), self._np_T)
        if not self.lib.batch_copy_maps(self.h, out.ctypes.data):
            raise Exception("Error copying batch maps")
        return out

    def stars(self, r: int) -> np.ndarray:
        total = int(self.value("total_stars"))
        out = np.empty((total, 3), self._np_T)
        if not self.lib.batch_copy_stars(self.h, out.ctypes.data):
            raise Exception("Error copying batch stars")
        o, n = int(self.value("star_offset", r)), int(self.value("num_stars", r))
        return out[o:o + n].copy()

    @property
    def t_graph(self) -> float:
        return self.value("t_graph")


MASS_FUNCTIONS = [dict(mass_function="equal"),
                  dict(mass_function="salpeter", m_lower=0.08, m_upper=1.0),
                  dict(mass_function="kroupa", m_lower=0.01, m_upper=1.5)]


def random_realizations(n: int = 256, seed: int = 1000, first_seed: int = 1000, num_pixels: int = 1024,
                        half_length: float = 12.0, margin: float = 0.05):
    """Lens configurations for a batch: kappa_tot ~ U[0.1, 0.9], shear ~ U[0, 0.8],
    smooth_fraction ~ U[0, 0.9] drawn with numpy's PCG64(seed); draws with
    |1 - kappa -/+ shear| < margin (a shooting region of unbounded size) are
    redrawn and counted. Masses rotate equal / Salpeter (0.08-1) / Kroupa
    (0.01-1.5); star-field seeds are first_seed, first_seed + 1, ...
    Returns (list of keyword dicts for IPM, number of redraws)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out, redrawn = [], 0
    while len(out) < n:
        k, g, s = rng.uniform(0.1, 0.9), rng.uniform(0.0, 0.8), rng.uniform(0.0, 0.9)
        if abs(1 - k - g) < margin or abs(1 - k + g) < margin:
            redrawn += 1
            continue
        i = len(out)
        out.append(dict(kappa_tot=float(k), shear=float(g), smooth_fraction=float(s), random_seed=first_seed + i,
                        half_length_y1=half_length, half_length_y2=half_length, num_pixels_y1=num_pixels,
                        num_pixels_y2=num_pixels, theta_star=1.0, write_histograms=0, **MASS_FUNCTIONS[i % 3]))
    return out, redrawn

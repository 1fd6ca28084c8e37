"""Adaptive IPM: per-tile subdivision chosen by a small learned network.

The lens-plane cell lattice of a map is cut into 32 x 32-cell tiles; each tile
is deposited at a subdivision level 1, 2, 4, 8 or 16 (subcells per cell side).
`LevelNet` (8 -> 64 -> 64 -> 5, BF16 weights, FP32 accumulation) predicts the
level from per-tile features; it is trained on the device by the library's
own forward/backward kernels on labels the method generates itself (the
smallest level at which a tile's own deposit is within a tolerance of its
level-16 deposit, as a share of the tile's flux). Every run audits a seeded
random sample of tiles against level 16 and sends a tile whose chosen level
misses the tolerance to level 16.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib
from .mapmaker import IPM

LEVELS = (1, 2, 4, 8, 16)
FEATURES = ("kappa_smooth", "kappa_star_local", "shear_local", "log_det_min", "log_det_max", "critical",
            "log_star_dist", "log_map_dist")
DEFAULT_NET = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "level_net.npz")


def _fp(a):
    return a.ctypes.data_as(C.c_void_p)


class LevelNet:
    """Weights (FP32 masters; used as BF16) and feature standardisation."""

    def __init__(self, w, mu, sig):
        self.w = np.ascontiguousarray(w, np.float32)
        self.mu = np.ascontiguousarray(mu, np.float32)
        self.sig = np.ascontiguousarray(sig, np.float32)

    @classmethod
    def load(cls, path=DEFAULT_NET):
        d = np.load(path)
        return cls(d["w"], d["mu"], d["sig"])

    def save(self, path, **meta):
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.savez(path, w=self.w, mu=self.mu, sig=self.sig, **meta)

    @classmethod
    def train(cls, features, labels, epochs=30, batch=512, lr=3e-3, seed=0, is_double=False):
        """Trains on the device; returns (network, mean loss per epoch)."""
        lib = _lib.load("ipm", is_double)
        f = np.ascontiguousarray(features, np.float32)
        y = np.ascontiguousarray(labels, np.int32)
        n = len(y)
        w = np.zeros(lib.mlp_num_params(), np.float32)
        mu = np.zeros(8, np.float32)
        sig = np.zeros(8, np.float32)
        loss = np.zeros(epochs, np.float32)
        if not lib.mlp_train(_fp(f), _fp(y), n, int(epochs), int(batch), float(lr), int(seed), _fp(w), _fp(mu),
                             _fp(sig), _fp(loss)):
            raise Exception("Error training the level network")
        return cls(w, mu, sig), loss

    def gradients(self, features, labels, is_double=False):
        """Gradient of the mean cross-entropy over all samples (one minibatch)."""
        lib = _lib.load("ipm", is_double)
        f = np.ascontiguousarray(features, np.float32)
        y = np.ascontiguousarray(labels, np.int32)
        g = np.zeros(lib.mlp_num_params(), np.float32)
        loss = np.zeros(1, np.float32)
        if not lib.mlp_gradients(_fp(self.w), _fp(self.mu), _fp(self.sig), _fp(f), _fp(y), len(y), _fp(g), _fp(loss)):
            raise Exception("Error computing gradients")
        return g, float(loss[0])

    def predict(self, features, is_double=False):
        """Level classes 0..4 (levels 1, 2, 4, 8, 16)."""
        lib = _lib.load("ipm", is_double)
        f = np.ascontiguousarray(features, np.float32)
        out = np.zeros(len(f), np.int32)
        if not lib.mlp_predict(_fp(self.w), _fp(self.mu), _fp(self.sig), _fp(f), len(f), _fp(out)):
            raise Exception("Error running the level network")
        return out


class AdaptiveIPM:
    """An IPM map with per-tile subdivision.

    policy: "network" (levels from `network`), "uniform" (every tile at
    `level`) or "given" (per-tile `levels`). tolerance: the deposit error a
    tile's level may make against level 16 (labels and audit): a share of the
    tile's own flux (error_mode 0) or of the map's flux where the tile lands
    (error_mode 1). max_level: the largest level of labels and network
    choices (tiles near stars would ask for 16 at a large cost and a small
    gain in the map); the audit still sends a failing tile to 16.
    audit_bound: when more than this share of the audited tiles misses the
    tolerance at its chosen level, the choice escalates (network quantiles
    0.9, 0.95, 0.99, then every tile one level finer up to max_level).
    quantile: a tile takes the smallest level whose cumulative network
    probability reaches it (above 0.5 leans towards refining). The map inputs
    are those of IPM (keyword arguments)."""

    def __init__(self, network=None, policy="network", level=1, levels=None, tolerance=1e-3,
                 audit_fraction=0.01, audit_seed=1, audit_bound=0.05, refine_capacity=0, quantile=0.8, error_mode=0,
                 max_level=8,
                 tiled_min=1 << 30, is_double=False,
                 verbose=0,
                 **ipm_kwargs):
        self.is_double = bool(is_double)
        self.lib = _lib.load("ipm", self.is_double)
        self._np_T = np.float64 if self.is_double else np.float32
        self.h = self.lib.ada_init()
        self.base = IPM(**ipm_kwargs, is_double=self.is_double, _handle=self.lib.ada_base(self.h))
        self.verbose = verbose
        pol = {"network": 0, "uniform": 1, "given": 2}[policy]
        if level not in LEVELS:
            raise ValueError("level must be 1, 2, 4, 8 or 16")
        self.lib.ada_set_policy(self.h, pol, int(level))
        if policy == "network":
            net = network if network is not None else LevelNet.load()
            self.lib.ada_set_network(self.h, _fp(net.w), _fp(net.mu), _fp(net.sig))
        if levels is not None:
            lv = np.ascontiguousarray(levels, np.int32)
            self.lib.ada_set_levels(self.h, _fp(lv), len(lv))
        self.lib.ada_set_tolerance(self.h, float(tolerance))
        self.lib.ada_set_quantile(self.h, float(quantile))
        self.lib.ada_set_error_mode(self.h, int(error_mode))
        if max_level not in LEVELS:
            raise ValueError("max_level must be 1, 2, 4, 8 or 16")
        self.lib.ada_set_max_level(self.h, int(max_level))
        self.lib.ada_set_tiled_min(self.h, int(tiled_min))
        self.lib.ada_set_audit(self.h, float(audit_fraction), int(audit_seed))
        self.lib.ada_set_audit_bound(self.h, float(audit_bound))
        self.lib.ada_set_refine_capacity(self.h, int(refine_capacity))

    def close(self):
        if getattr(self, "h", None):
            self.base.close()
            self.lib.ada_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self):
        if not self.lib.ada_run(self.h, int(self.verbose)):
            raise Exception("Error running adaptive IPM")

    def value(self, name):
        return self.lib.ada_get_value(self.h, name.encode())

    @property
    def tiles(self):
        return int(self.value("tiles_y")), int(self.value("tiles_x"))

    @property
    def features(self) -> np.ndarray:
        n = self.lib.ada_num_tiles(self.h)
        out = np.zeros((n, 8), np.float32)
        if not self.lib.ada_copy_features(self.h, _fp(out)):
            raise Exception("Error copying features")
        return out

    def levels(self, predicted=False) -> np.ndarray:
        n = self.lib.ada_num_tiles(self.h)
        out = np.zeros(n, np.int32)
        self.lib.ada_copy_levels(self.h, _fp(out), int(bool(predicted)))
        return out

    def labels(self, tiles):
        """(classes 0..4, deposit errors of levels 1, 2, 4, 8 against 16 [n, 4])."""
        t = np.ascontiguousarray(tiles, np.int32)
        lab = np.zeros(len(t), np.int32)
        err = np.zeros((len(t), 4), np.float32)
        if not self.lib.ada_labels(self.h, _fp(t), len(t), _fp(lab), _fp(err)):
            raise Exception("Error computing labels")
        return lab, err

    @property
    def magnifications(self) -> np.ndarray:
        npx, npy = self.base.num_pixels_y1, self.base.num_pixels_y2
        out = np.zeros((npy, npx), self._np_T)
        if not self.lib.ada_copy_map(self.h, _fp(out)):
            raise Exception("Error copying the map")
        return out

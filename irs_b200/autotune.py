"""Autotuner of the lens-equation pass: expansion order against tree depth,
lattice points per thread and persistent-grid occupancy.

For one map configuration it shoots a band of lattice rows through the
leaf-tiled FP32 kernel:
  1. expansion order: the corner positions at each candidate order are
     compared with those at the largest order (31); the smallest order whose
     largest displacement stays within the target (default: the reference's
     own error budget alpha_error, in pixels) is kept. The reference's formula
     (ceil(2 log2 theta + tree_levels - log2 root_half_length -
     log2 alpha_error)) and the tree depth are reported beside it;
  2. launch shape: at that order, every (threads per CTA, CTAs per SM) pair is
     timed on the band (CUDA events, median of repeats) and the fastest kept;
     128 / 256 / 512 threads put 8 / 4 / 2 lattice points on a thread (the
     reuse of each staged star).
The result is applied with apply() to IPM / IRS objects or used for a
BatchIPM (expansion_order).
"""
from __future__ import annotations

import numpy as np

from .mapmaker import IPM

THREADS = (128, 256, 512)
CTAS_PER_SM = (8, 16, 32, 64)


def autotune(config: dict, band_rows: int = 256, target_px: float | None = None, orders=None, threads=THREADS,
             ctas=CTAS_PER_SM, repeats: int = 3, verbose: bool = False) -> dict:
    m = IPM(**config, is_double=False, precision=2)
    m.derive()
    ny = int(m.value("num_ray_threads_2"))
    lo = max(0, ny // 2 - band_rows // 2)
    hi = min(ny, lo + band_rows)
    m.lib.set_band(m.obj, lo, hi)
    npx, hly = m.num_pixels_y1, m.half_length_y1
    alpha_px = m.value("alpha_error") * npx / (2 * hly)
    target = alpha_px if target_px is None else float(target_px)

    def positions(order):
        m.expansion_order = order
        m.run()
        return m.vertices()

    ref = positions(31)
    levels = int(m.value("tree_levels"))
    m.expansion_order = 0
    m.run()
    formula = int(m.value("expansion_order"))
    cand = orders if orders is not None else list(range(max(3, formula - 6), min(31, formula + 4) + 1))
    trials = []
    chosen = 31
    for p in cand:
        v = positions(p)
        ok = np.isfinite(v).all(-1) & np.isfinite(ref).all(-1)
        err = float(np.max(np.hypot(*(v[ok] - ref[ok]).T))) if ok.any() else float("inf")
        trials.append({"order": p, "max_err_px": err})
        if verbose:
            print(f"order {p}: max displacement {err:.3g} px (target {target:.3g})")
        if err <= target and chosen == 31:
            chosen = p
    m.expansion_order = chosen
    m.run()
    shapes = []
    for t in threads:
        for c in ctas:
            m.lib.set_shoot_launch(m.obj, int(t), int(c))
            ms = []
            for _ in range(repeats):
                m.rerun(1)
                ms.append(m.value("t_lattice") * 1e3)
            shapes.append({"threads": t, "ctas_per_sm": c, "lattice_ms": float(np.median(ms))})
            if verbose:
                print(f"threads {t} ctas/SM {c}: {np.median(ms):.3f} ms")
    best = min(shapes, key=lambda d: d["lattice_ms"])
    m.close()
    return {"order": chosen, "formula_order": formula, "tree_levels": levels, "target_px": target,
            "threads": best["threads"], "ctas_per_sm": best["ctas_per_sm"], "band_rows": hi - lo,
            "order_trials": trials, "shape_trials": shapes}


def apply(obj, tuned: dict):
    """Sets the tuned order and launch shape on an IPM / IRS object."""
    obj.expansion_order = int(tuned["order"])
    obj.lib.set_shoot_launch(obj.obj, int(tuned["threads"]), int(tuned["ctas_per_sm"]))
    return obj

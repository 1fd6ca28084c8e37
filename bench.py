"""Benchmark: IPM pixels/s (and IRS rays/s) on one B200.

Default workload (the plain-IPM case at its stated substitute shear):
  IPM, Salpeter masses 0.08-1.0 with theta_star set to the Einstein radius of
  the mean mass, kappa_tot 0.45, shear 0.40 (0.55 as published puts
  1 - kappa - shear at 0, an unbounded shooting region), smooth fraction 0.5,
  circular field (~3.75e4 stars), source half-length 25, 2000 x 2000 map,
  1 cell per pixel (3720 x 23552 cells), expansion order 12, seed 2, FP32 form.

One step = the whole device pipeline on the star field resident in HBM:
quadtree build, FP64 expansions, leaf records, lattice lens equation and the
fixed-point deposition. value = pixels of all steps / device time (CUDA events,
max over ranks). e2e = the same through the public API with host buffers: per
step, IPM.run() copies the star field from host memory, runs the full pipeline
(including the histograms) and returns the map as a numpy array in host memory
(IPM.magnifications), timed on the host clock.

Both arms use one star field (workload_stars: numpy PCG64, the workload's
seed), handed to this build through set_stars.

--impl reference times the reference's own IPM on the host CPU cores (its tree,
expansions and cell-shooting kernel compiled for the host, OpenMP; the oracle's
restatement where that library was not built): each step a band of cell rows
plus the band's share of the tree's time (built once), the pixels accounted
being the band's share of the map; the whole map once beside it, and the
reference's own GPU build on the same star field (secondary.reference_gpu).
No library of this build is loaded by that arm.
Under torchrun every rank runs an independent replica (the map of one
realisation is not sharded here); value sums the replicas.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(
    name="ipm_salpeter_k0.45_g0.40_s0.5_2000px_hly25_p12",
    kappa_tot=0.45, shear=0.40, smooth_fraction=0.5, mass_function="salpeter", m_lower=0.08, m_upper=1.0,
    half_length_y1=25.0, half_length_y2=25.0, num_pixels_y1=2000, num_pixels_y2=2000, num_rays_y=1,
    random_seed=2, expansion_order=12,
)
SAFETY = 1.3  # a drawn field meets the 1.37 star-field coverage check only to within its sampling noise


def salpeter_moments(lo=0.08, hi=1.0, s=-2.35):
    """<m> and <m^2> of the mass function m^s on [lo, hi]."""
    def integral(k):
        return (hi ** (s + k + 1) - lo ** (s + k + 1)) / (s + k + 1)
    return integral(1) / integral(0), integral(2) / integral(0)


def workload_stars(n, radius, seed=2):
    """The workload's star field, shared by both arms: n stars uniform in the
    disc of the given radius (sqrt of a uniform for the radius), Salpeter
    masses 0.08-1.0 by inverse CDF; numpy PCG64 with the workload's seed."""
    rng = np.random.default_rng(seed)
    r = radius * np.sqrt(rng.random(n))
    a = 2 * np.pi * rng.random(n)
    u = rng.random(n)
    lo, hi, s = WORKLOAD["m_lower"], WORKLOAD["m_upper"], -2.35
    mass = (lo ** (s + 1) + u * (hi ** (s + 1) - lo ** (s + 1))) ** (1 / (s + 1))
    return np.stack([r * np.cos(a), r * np.sin(a), mass], 1)


def workload_config(stars, n_gpus=1):
    """The `config` object of both arms' JSON lines (identical keys and values)."""
    return {"workload": WORKLOAD["name"], "pixels": WORKLOAD["num_pixels_y1"] * WORKLOAD["num_pixels_y2"],
            "stars": int(stars), "order": WORKLOAD["expansion_order"],
            "star_field": f"numpy PCG64 seed {WORKLOAD['random_seed']}: uniform in the disc of the reference-formula "
                          "radius, Salpeter masses by inverse CDF (the same field in both arms)",
            "l2": "inputs larger than L2: the 1.4 GB corner lattice of every step",
            "parallelism": "replicas" if n_gpus > 1 else "1 GPU"}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "25"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


IRS_CASE1 = dict(kappa_tot=0.4, shear=0.3, kappa_star=0.4, theta_star=1.0, mass_function="equal",
                 half_length_y1=10.0, half_length_y2=10.0, num_pixels_y1=500, num_pixels_y2=500, num_rays_y=100,
                 light_loss=0.01, random_seed=1, expansion_order=8, write_stars=0, write_maps=0,
                 write_histograms=0)
SMALL = dict(half_length_y1=6.25, half_length_y2=6.25, num_pixels_y1=500, num_pixels_y2=500)


def make_ipm(is_double=False, precision=None, size="full", stars=True):
    """The workload as an IPM object. stars=True: the workload's star field
    (workload_stars) handed over through set_stars, as a star file would be;
    stars=False: the library draws its own field (curand, the workload's seed)."""
    import irs_b200
    w = {k: v for k, v in WORKLOAD.items() if k != "name"}
    if size == "small":  # same lens and pixel scale, 500 x 500 map (profiling captures)
        w.update(SMALL)
    probe = irs_b200.IPM(**{**w, "theta_star": 1.0}, is_double=True)
    probe.derive()
    theta = 1.0 / np.sqrt(probe.value("mean_mass"))  # Einstein radius of the mean mass
    probe.close()
    m = irs_b200.IPM(**w, theta_star=theta, is_double=is_double, precision=precision, write_stars=0, write_maps=0)
    if stars:
        d = irs_b200.IPM(**w, theta_star=theta, is_double=True)
        d.derive()
        n, rad = int(d.value("num_stars")), float(np.hypot(d.value("corner_x1"), d.value("corner_x2")))
        d.close()
        m.set_stars(workload_stars(n, rad), rectangular=False, corner=(rad, 0.0), theta_star=theta)
        m.safety_scale = SAFETY
    return m


def cpu_baseline(m, stars, threads, budget_s=12.0):
    """FP64 direct sum over all stars on a bounded random sample of cell corners,
    plus the reference polygon deposition of a band of cells, scaled to the
    lattice. The sampled direct-sum corners are also the FP64 oracle the GPU's
    corner positions are checked against (`error_vs_fp64_oracle`)."""
    from oracle import pyoracle as po
    from tests.cases import oracle_lens, to_pixels
    rng = np.random.default_rng(0)
    nx, ny = int(m.value("num_ray_threads_1")), int(m.value("num_ray_threads_2"))
    nverts = (nx + 1) * (ny + 1)
    rx, ry = m.value("ray_half_sep_1"), m.value("ray_half_sep_2")
    ox = m.value("center_x1") - m.value("half_length_x1")
    oy = m.value("center_x2") - m.value("half_length_x2")
    L = oracle_lens(m)
    n = 2000
    while True:
        ii = rng.integers(0, nx + 1, n)
        jj = rng.integers(0, ny + 1, n)
        zx = ox + 2.0 * (rx * ii)
        zy = oy + 2.0 * (ry * jj)
        t0 = time.perf_counter()
        wx, wy = po.shoot_direct(stars, L, zx, zy, threads=threads)
        dt = time.perf_counter() - t0
        if dt > budget_s / 4 or n >= 2_000_000:
            break
        n = int(n * min(8.0, max(2.0, budget_s / 2 / max(dt, 1e-6))))
    t_vert = dt / n * nverts
    v = m.vertices()
    band = v[: min(65, v.shape[0])]
    ncells_band = (band.shape[0] - 1) * (band.shape[1] - 1)
    factor = 2 * rx * ry * m.num_pixels_y1 * m.num_pixels_y2 / (4 * m.half_length_y1 * m.half_length_y2)
    t0 = time.perf_counter()
    po.ipm_deposit_ref(band, factor, m.num_pixels)
    t_dep = (time.perf_counter() - t0) / ncells_band * (nx * ny)
    total = t_vert + t_dep
    out = {"value": m.num_pixels_y1 * m.num_pixels_y2 / total, "unit": "pixels/s", "cores": threads,
           "kind": "port",
           "sample": f"FP64 direct sum over all {stars.shape[0]} stars at {n} random cell corners "
                     f"({dt:.2f} s) + reference polygon deposition of {ncells_band} cells, scaled to "
                     f"{nverts} corners and {nx * ny} cells"}
    # ---- the GPU's FP32 corner positions against the FP64 direct sum (pixels)
    px, py = to_pixels(m, wx, wy)
    err = np.hypot(v[jj, ii, 0] - px, v[jj, ii, 1] - py)
    onmap = (px > 0) & (px < m.num_pixels_y1) & (py > 0) & (py < m.num_pixels_y2)
    chk = {"corners": {"sample": f"{n} random corners of the lattice ({int(onmap.sum())} landing on the map)",
                       "median_px": float(np.median(err)), "p99_px": float(np.quantile(err, 0.99)),
                       "max_px": float(err.max()),
                       "median_px_on_map": float(np.median(err[onmap])) if onmap.any() else None}}
    # ---- a band of cell rows through the map centre: the map the GPU's corners
    # deposit against the map the direct-sum corners deposit (same deposition)
    rows = 64
    j0 = ny // 2 - rows // 2
    jb = np.arange(j0, j0 + rows + 1)
    ib = np.arange(nx + 1)
    bx, by = np.meshgrid(ox + 2.0 * (rx * ib), oy + 2.0 * (ry * jb))
    t0 = time.perf_counter()
    wx, wy = po.shoot_direct(stars, L, bx, by, threads=threads)
    t_band = time.perf_counter() - t0
    px, py = to_pixels(m, wx.reshape(bx.shape), wy.reshape(bx.shape))
    f32 = np.float32
    factor32 = float(f32(f32(f32(f32(f32(2) * f32(rx)) * f32(ry)) * f32(m.num_pixels_y1)) * f32(m.num_pixels_y2))
                     / f32(f32(f32(f32(2) * f32(m.half_length_y1)) * f32(2)) * f32(m.half_length_y2)))
    ref = po.ipm_deposit_fixed(np.stack([px, py], -1), factor32, m.num_pixels, single=True).astype(np.float64)
    got = po.ipm_deposit_fixed(v[j0:j0 + rows + 1], factor32, m.num_pixels, single=True).astype(np.float64)
    ok = ref > 0
    rel = np.abs(got[ok] - ref[ok]) / ref[ok]
    big = ref[ok] >= 0.1 * ref[ok].mean()  # pixels the band covers substantially
    chk["band_map"] = {"sample": f"cell rows {j0}..{j0 + rows} of {ny} (all {nx} columns, {rows * nx} cells, "
                                 f"{int(ok.sum())} pixels touched), direct sum {t_band:.1f} s",
                       "median_rel": float(np.median(rel)), "p99_rel": float(np.quantile(rel, 0.99)),
                       "max_rel": float(rel.max()),
                       "max_rel_covered": float(rel[big].max()), "covered_pixels": int(big.sum()),
                       "flux_weighted_rel": float(np.abs(got - ref).sum() / ref.sum())}
    return out, chk


def irs_case1_errors(threads, rows=1024):
    """The plain-IRS configuration (FP32 form, order 8) against the FP64
    direct sum over all stars, on a band of ray rows through the lattice
    centre: the rays that land in another pixel (half the summed map
    difference) and the relative error of the band's counts."""
    import irs_b200
    from oracle import pyoracle as po
    from tests.cases import oracle_lens
    r = irs_b200.IRS(**IRS_CASE1, is_double=False)
    r.derive()
    nx, ny = int(r.value("num_ray_threads_1")), int(r.value("num_ray_threads_2"))
    j0 = ny // 2 - rows // 2
    r.lib.set_band(r.obj, j0, j0 + rows)
    r.run()
    got = r.magnifications.astype(np.int64)
    rx, ry = r.value("ray_half_sep_1"), r.value("ray_half_sep_2")
    bx = r.value("center_x1") - r.value("half_length_x1") + rx
    by = r.value("center_x2") - r.value("half_length_x2") + ry
    t0 = time.perf_counter()
    wx, wy = po.shoot_direct_lattice(r.stars.astype(np.float64), oracle_lens(r), bx, by, rx, ry, 0, nx, j0, rows,
                                     threads=threads)
    dt = time.perf_counter() - t0
    ref = po.irs_bin(wx, wy, r.center, r.half_length, r.num_pixels).astype(np.int64)
    r.close()
    ok = ref > 0
    rel = np.abs(got[ok] - ref[ok]) / ref[ok]
    return {"sample": f"ray rows {j0}..{j0 + rows} of {ny} ({rows * nx} rays), direct sum over all stars {dt:.1f} s",
            "rays_received": int(ref.sum()), "rays_moved": int(np.abs(got - ref).sum() // 2),
            "fraction_moved": float(np.abs(got - ref).sum() / 2 / max(ref.sum(), 1)),
            "median_rel": float(np.median(rel)), "max_rel": float(rel.max())}


def reference_geometry():
    """The workload's star field and lattice as the reference derives them for
    a star file (ipm.cuh:370-565 with the moments of the field itself), in FP64
    through the oracle's restatement: no library of this build is loaded."""
    from oracle import pyoracle as po
    w = WORKLOAD
    mm, mm2 = salpeter_moments(w["m_lower"], w["m_upper"])
    theta = 1.0 / np.sqrt(mm)
    kstar = (1 - w["smooth_fraction"]) * w["kappa_tot"]
    hly = (w["half_length_y1"], w["half_length_y2"])
    npix = (w["num_pixels_y1"], w["num_pixels_y2"])
    d = po.derive(w["kappa_tot"], w["shear"], kstar, theta, mm, mm2, 0.001, 0, 1.37, (0.0, 0.0), hly, npix,
                  w["num_rays_y"])
    n, rad = int(d["num_stars"]), float(np.hypot(d["corner_x1"], d["corner_x2"]))
    stars = workload_stars(n, rad)
    m = stars[:, 2]
    ks = theta * theta * m.sum() / (rad * rad)  # calculate_star_params (star.cuh:124-161), circle
    g = po.derive(w["kappa_tot"], w["shear"], ks, theta, m.mean(), (m * m).mean(), 0.001, 0, SAFETY, (0.0, 0.0),
                  hly, npix, w["num_rays_y"])
    return stars, rad, theta, ks, g


def reference_gpu_leg(stars, rad, theta, repeats=3):
    """The reference's own IPM on the B200 (oracle/_ref/gpu: its lib_ipm.so
    built from its sources for sm_100a, driven through its unchanged Python
    package in a child process) on the same star field: the kernel time it
    reports (t_shoot_cells, ipm.cuh:929-934) and the wall time of run()."""
    import tempfile

    from oracle import ref_gpu as rg
    if not rg.available("ipm"):
        return {"unavailable": "oracle/_ref/gpu not built (make -C oracle refgpu needs the reference sources)"}
    w = WORKLOAD
    with tempfile.TemporaryDirectory() as td:
        sf = os.path.join(td, "stars.bin")
        rg.write_starfile(sf, stars, False, (rad, 0.0), theta, double=False)
        q = dict(kappa_tot=w["kappa_tot"], shear=w["shear"], half_length_y1=w["half_length_y1"],
                 half_length_y2=w["half_length_y2"], num_pixels_y1=w["num_pixels_y1"],
                 num_pixels_y2=w["num_pixels_y2"], num_rays_y=w["num_rays_y"], starfile=sf, safety_scale=SAFETY,
                 write_stars=0, write_maps=0, write_histograms=0)
        try:
            r = rg.run_ipm(q, is_double=False, repeats=repeats, timeout=600)
        except Exception as e:  # noqa: BLE001
            return {"unavailable": f"the reference's GPU run failed: {str(e)[:300]}"}
    npix = w["num_pixels_y1"] * w["num_pixels_y2"]
    ts = float(np.min(r["t_shoot_cells"]))
    wall = float(np.min(r["walls"]))
    return {"what": "the reference's lib_ipm.so (float) built for sm_100a, unchanged microlensing.IPM wrapper, "
                    "same star field", "t_shoot_cells_s": ts, "run_wall_s": wall,
            "pixels_per_s_shoot": npix / ts, "pixels_per_s_run": npix / wall, "repeats": repeats}


def reference_arm(args):
    """The reference's IPM on the host cores, on the same workload and star
    field: its own tree, expansions and shoot_cells_kernel
    (ipm_functions.cuh:112-170, polygon deposition polygon.cuh:349-467)
    compiled for the host under oracle/_ref (oracle/Makefile, target ref),
    OpenMP over the kernel's threads, one per core; where that library was not
    built, the oracle's restatement of the same algorithm. A step is a bounded
    sample of the workload: a band of cell rows, plus the band's share of the
    time of the tree and expansions of all stars (built and timed once); the
    pixels it accounts for are the band's share of the map. Once, outside the
    steps, the whole map (tree included) is made and its throughput compared
    with the steps'. The reference's GPU build on the
    same field is reported beside it (secondary.reference_gpu)."""
    ws, rank, local = _dist()
    if rank != 0:
        return
    from oracle import pyoracle as po
    stars, rad, theta, ks, g = reference_geometry()
    nstars = stars.shape[0]
    threads = os.cpu_count() or 1
    w = WORKLOAD
    nx, ny = int(g["num_ray_threads_1"]), int(g["num_ray_threads_2"])
    rx, ry = g["ray_half_sep_1"], g["ray_half_sep_2"]
    cx1, cx2 = g["center_x1"], g["center_x2"]
    hx1, hx2 = g["half_length_x1"], g["half_length_x2"]
    npx, npy = w["num_pixels_y1"], w["num_pixels_y2"]
    hly = (w["half_length_y1"], w["half_length_y2"])
    L = po.lens(w["kappa_tot"], w["shear"], ks, theta, 0, 1, 1, (rad, 0.0))  # circle, approximate smooth sheet
    use_ref = po.ref_available()
    band_rows = 4096  # about 1.2 s of host work per step on 16 cores

    def build():
        """The tree and expansions of all stars (the reference's own where built)."""
        if use_ref:
            return po.RefTree(stars, 1.1 * rad, order=w["expansion_order"], theta=theta,
                              alpha_error=g["alpha_error"], kind="ipm")
        return po.Tree(stars, 1.1 * rad, order=w["expansion_order"])

    def shoot(t, j0, rows):
        """Seconds to shoot and deposit cell rows j0 .. j0 + rows."""
        t0 = time.perf_counter()
        if use_ref:  # the reference's own shoot_cells_kernel (deposition included)
            # the kernel's cells are centre_x - hlx + rhs + 2 rhs (i, j), so the band
            # is the lattice of `rows` rows with its centre moved by 2 rhs_y j0
            t.shoot(L, (rx, ry), (nx, rows), (cx1, cx2 + 2 * ry * j0), (hx1, hx2), (0.0, 0.0), hly, (npx, npy),
                    threads=threads)
        else:
            ox, oy = cx1 - hx1, cx2 - hx2
            jj = np.arange(j0, j0 + rows + 1)
            ii = np.arange(nx + 1)
            X, Y = np.meshgrid(ox + 2.0 * (rx * ii), oy + 2.0 * (ry * jj))
            wx, wy = t.shoot(L, X, Y)
            px = (wx + hly[0]) * npx / (2 * hly[0])
            py = npy - (wy + hly[1]) * npy / (2 * hly[1])
            factor = 2 * rx * ry * npx * npy / (4 * hly[0] * hly[1])
            po.ipm_deposit_ref(np.stack([px, py], -1), factor, (npx, npy))
        return time.perf_counter() - t0

    t0 = time.perf_counter()
    tree = build()
    t_tree = time.perf_counter() - t0
    share = band_rows / ny
    # a step: one band of rows plus the band's share of the tree and expansions
    # (timed once above: the tree cannot be split, its cost is shared pro rata)
    def band(k):
        """Band k: rows k * band_rows onwards, wrapping at the lattice's end, so
        that consecutive steps sweep the whole lattice."""
        j0 = (k * band_rows) % ny
        n0 = min(band_rows, ny - j0)
        return shoot(tree, j0, n0) + (shoot(tree, 0, band_rows - n0) if n0 < band_rows else 0.0)

    for k in range(args.warmup):
        band(k)
    ts = np.array([band(args.warmup + k) + share * t_tree for k in range(args.steps)])
    tot = float(ts.sum())
    units = args.steps * npx * npy * share  # the bands' share of the map, in pixels
    value = units / tot
    t0 = time.perf_counter()
    full_tree = build()
    t_full = time.perf_counter() - t0 + shoot(full_tree, 0, ny)  # the whole map once, tree included
    kind = "reference" if use_ref else "port"
    what = ("the reference's own tree, expansions and shoot_cells_kernel (polygon deposition included), compiled "
            "for the host" if use_ref else "the oracle's restatement (FMM form, reference deposition)")
    sample = (f"{what}: the tree and expansions of all {nstars} stars timed once ({t_tree:.2f} s); each step "
              f"a band of {band_rows} of the {ny} cell rows (consecutive steps sweep the lattice) plus that share "
              f"of the tree's time; the pixels accounted are the band's share of the map")
    out = {
        "impl": "reference", "metric": "IPM pixels/s", "value": value, "unit": "pixels/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(nstars, args.gpus),
        "lattice": {"cells": nx * ny, "nx": nx, "ny": ny},
        "cpu_baseline": {"value": value, "unit": "pixels/s", "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "pixels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "tree_s": t_tree,
        "full_lattice": {"seconds": t_full, "pixels_per_s": npx * npy / t_full,
                         "ratio_to_band_steps": (npx * npy / t_full) / value},
        "secondary": {"reference_gpu": reference_gpu_leg(stars, rad, theta)},
    }
    print(json.dumps(out))


def batch_measure(steps):
    """The batched form: 256 realizations of uneven size (1024^2 maps, half
    length 12) through the graph-captured pipeline, its best replay; then the
    plain uniform FP64 form of every realization run singly at the same
    expansion order, the best of two runs of its device pipeline each, and the
    FP32 batch maps' error against those FP64 maps."""
    import irs_b200
    from irs_b200.batch import random_realizations

    reals, redrawn = random_realizations()
    b = irs_b200.BatchIPM(reals)
    t0 = time.perf_counter()
    b.run()
    first = time.perf_counter() - t0
    ts = [b.rerun(1) for _ in range(max(2, steps))]
    t_batch = float(np.min(ts))
    pix, cells = b.value("total_pixels"), b.value("total_cells")
    order = int(b.value("expansion_order"))
    maps = b.maps
    res = {"realizations": len(reals), "redrawn": redrawn, "stars": int(b.value("total_stars")), "cells": int(cells),
           "pixels": int(pix), "order": order, "passes": int(b.value("passes")),
           "graph_nodes": int(b.value("graph_nodes")), "graph_replay_ms": t_batch * 1e3,
           "pixels_per_s": pix / t_batch, "cells_per_s": cells / t_batch, "first_run_s": first,
           "stars_and_moments_ms": b.value("t_stars") * 1e3}
    b.close()
    t_plain, med, mx = 0.0, [], []
    for r, kw in enumerate(reals):
        s = irs_b200.IPM(**kw, is_double=True, expansion_order=order)
        s.run()
        t_plain += min(s.rerun(1), s.rerun(1))  # best of two, as the batch's best replay
        ref = s.magnifications
        s.close()
        ok = ref > 0
        rel = np.abs(maps[r][ok].astype(np.float64) - ref[ok]) / ref[ok]
        med.append(float(np.median(rel)))
        mx.append(float(rel.max()))
    res.update({"plain_fp64_s": t_plain, "plain_fp64_pixels_per_s": pix / t_plain,
                "batched_fp32_over_plain_fp64": t_plain / t_batch,
                "median_rel_err_vs_fp64": {"median_of_maps": float(np.median(med)), "max_of_maps": float(np.max(med))},
                "max_rel_err_vs_fp64": float(np.max(mx))})
    return res


ADAPTIVE_CONFIG = dict(kappa_tot=0.6, shear=0.3, smooth_fraction=0.3, mass_function="salpeter", m_lower=0.08,
                       m_upper=1.0, theta_star=1.0, half_length_y1=30.0, half_length_y2=30.0, num_pixels_y1=4096,
                       num_pixels_y2=4096, random_seed=4, write_histograms=0)


def adaptive_measure():
    """The learned-adaptive form on its configuration (4096^2 map): the
    network-chosen map (audit tolerance 1e-3 of a tile's flux on 0.25 % of
    the tiles, escalation bound 5 %) against the uniform-fine (level 16) map;
    the errors of the uniform levels 1-8; and the plain uniform FP64 form at
    level 8, whose error matches the adaptive map's, run over its whole
    lattice (2.9e10 cells) band by band: its tree and expansions once plus
    the lens equation and deposition of every band, device time."""
    import irs_b200

    def rel_err(mu, ref):
        ok = ref > 0
        r = np.abs(mu[ok].astype(np.float64) - ref[ok]) / ref[ok]
        return float(np.median(r)), float(np.quantile(r, 0.99))

    cfg = ADAPTIVE_CONFIG
    # one star field for every map below (the library's own draw for the
    # configuration's seed, as the FP32 form stores it): a plain run at
    # another num_rays_y would otherwise derive another star count
    g = irs_b200.IPM(**cfg, is_double=False)
    g.run()
    field = (g.stars.astype(np.float64), (float(g.value("rad")), 0.0))
    g.close()

    def with_field(m):
        base = m.base if hasattr(m, "base") else m
        base.set_stars(field[0], rectangular=False, corner=field[1], theta_star=cfg["theta_star"])
        base.safety_scale = SAFETY
        return m

    u16 = with_field(irs_b200.AdaptiveIPM(policy="uniform", level=16, audit_fraction=0.0, **cfg))
    u16.run()
    ref = u16.magnifications.astype(np.float64)
    u16_ms = (u16.value("t_base") + u16.value("t_adapt")) * 1e3
    u16.close()
    a = with_field(irs_b200.AdaptiveIPM(tolerance=1e-3, audit_fraction=0.0025, audit_bound=0.05, **cfg))
    a.run()  # warm-up
    runs = []
    for _ in range(3):  # the best of three warm runs (one seed: the same map each time)
        a.run()
        runs.append((a.value("t_base") + a.value("t_adapt"), a.value("t_base"), a.value("t_adapt")))
    t_ada, t_base, t_adapt = min(runs)
    mu_a = a.magnifications
    lv = a.levels()
    res = {"tiles": int(len(lv)), "levels_hist": np.bincount(np.log2(lv).astype(int), minlength=5).tolist(),
           "cells_base": int(a.value("cells_base")), "cells_evaluated": int(a.value("cells_evaluated")),
           "audit_tolerance": 1e-3, "audited": int(a.value("audited")), "audit_failures": int(a.value("audit_failures")),
           "audit_miss_rate_network": a.value("fail_rate_initial"), "audit_miss_rate_final": a.value("fail_rate"),
           "audit_miss_bound": a.value("fail_bound"), "audit_escalation": int(a.value("escalation")),
           "network_quantile_used": a.value("quantile_used"),
           "t_base_ms": t_base * 1e3, "t_adapt_ms": t_adapt * 1e3,
           "t_runs_ms": [round(r[0] * 1e3, 2) for r in runs],
           "t_select_ms": a.value("t_select") * 1e3, "t_audit_ms": a.value("t_audit") * 1e3,
           "t_refine_deposit_ms": a.value("t_refine_deposit") * 1e3, "uniform16_ms": u16_ms}
    a.close()
    med_a, p99_a = rel_err(mu_a, ref)
    res.update({"median_rel_err_vs_uniform16": med_a, "p99_rel_err_vs_uniform16": p99_a})
    for L in (1, 2, 4, 8):
        u = with_field(irs_b200.AdaptiveIPM(policy="uniform", level=L, audit_fraction=0.0, **cfg))
        u.run()
        res[f"uniform{L}_median_rel_err"] = rel_err(u.magnifications, ref)[0]
        u.close()
    # the plain uniform FP64 form at level 8 (num_rays_y = 64) over its whole lattice
    L = 8
    p = with_field(irs_b200.IPM(**{**cfg, "num_rays_y": L * L}, is_double=True))
    p.derive()
    ny, nx = int(p.value("num_ray_threads_2")), int(p.value("num_ray_threads_1"))
    rows = max(1, int(2.5e8 // (nx + 1)))  # corner buffer of a band: 4 GB at most
    t_bands, tree, acc, nb = 0.0, None, None, 0
    for lo in range(0, ny, rows):
        p.lib.set_band(p.obj, lo, min(ny, lo + rows))
        if tree is None:
            p.run()
        tb = p.rerun(1)
        band = p.value("t_lattice") + p.value("t_deposit")
        t_bands += band
        if tree is None:
            tree = tb - band
        f = p.fixed_maps()
        acc = f if acc is None else acc + f
        nb += 1
    p.close()
    t_plain = tree + t_bands
    mu_p = (np.maximum(acc.view(np.int64), 0).astype(np.float64) / 2.0 ** 32)
    res.update({"plain_fp64_level": L, "plain_fp64_cells": int(nx) * int(ny), "plain_fp64_bands": nb,
                "plain_fp64_s": t_plain, "plain_fp64_tree_s": tree,
                "plain_fp64_median_rel_err_vs_uniform16": rel_err(mu_p, ref)[0], "adaptive_s": t_ada,
                "effective_cells_per_s_adaptive": nx * ny / t_ada,
                "effective_cells_per_s_plain_fp64": nx * ny / t_plain,
                "adaptive_over_plain_fp64": t_plain / t_ada})
    return res


CONFIG3 = dict(kappa_tot=0.7, shear=0.2, smooth_fraction=0.1, theta_star=1.0, mass_function="kroupa", m_lower=0.01,
               m_upper=1.5, rectangular=True, approx=True, half_length_y1=50.0, half_length_y2=50.0,
               num_pixels_y1=8192, num_pixels_y2=8192, random_seed=3, expansion_order=16, write_histograms=0)


def config3_measure():
    """The rectangular Kroupa configuration: 8192^2 map, approximate smooth
    sheet (degree-39 series), expansion order 16; IRS at 64 rays per pixel
    (1.1e11 rays, 4.3e5 stars) and IPM at one cell per pixel (2.5e9 cells,
    6.5e5 stars), FP32 form, device time of the whole pipeline (best of 2)."""
    import irs_b200
    out = {}
    r = irs_b200.IRS(**CONFIG3, num_rays_y=64, is_double=False)
    r.run()
    ts = [r.rerun(1) for _ in range(2)]
    t = float(np.min(ts))
    out["irs"] = {"rays": int(r.num_rays_shot), "stars": int(r.num_stars), "rays_received": int(r.num_rays_received),
                  "s_per_map": t, "lattice_s": r.value("t_lattice"), "rays_per_s": r.num_rays_shot / t}
    r.close()
    m = irs_b200.IPM(**CONFIG3, num_rays_y=1, is_double=False)
    m.run()
    ts = [m.rerun(1) for _ in range(2)]
    t = float(np.min(ts))
    out["ipm"] = {"cells": int(m.value("num_ray_threads_1") * m.value("num_ray_threads_2")), "stars": int(m.num_stars),
                  "s_per_map": t, "lattice_ms": m.value("t_lattice") * 1e3, "deposit_ms": m.value("t_deposit") * 1e3,
                  "pixels_per_s": 8192 * 8192 / t}
    m.close()
    return out


def config3_errors(threads, n=4000):
    """Config-3 IPM FP32 corner positions against the FP64 direct sum over all
    stars: a seeded sample of corners of two cell rows through the lattice centre."""
    import irs_b200
    from oracle import pyoracle as po
    from tests.cases import lattice, oracle_lens, to_pixels
    m = irs_b200.IPM(**CONFIG3, num_rays_y=1, is_double=False)
    m.derive()
    ny = int(m.value("num_ray_threads_2"))
    j0 = ny // 2
    m.lib.set_band(m.obj, j0, j0 + 2)
    m.run()
    v = m.vertices()
    rng = np.random.default_rng(0)
    jj, ii = rng.integers(0, v.shape[0], n), rng.integers(0, v.shape[1], n)
    x, _ = lattice(m, vertices=True)
    oy = m.value("center_x2") - m.value("half_length_x2")
    y = oy + 2.0 * (m.value("ray_half_sep_2") * (j0 + jj).astype(np.float64))
    t0 = time.perf_counter()
    wx, wy = po.shoot_direct(m.stars.astype(np.float64), oracle_lens(m), x[ii], y, threads=threads)
    dt = time.perf_counter() - t0
    px, py = to_pixels(m, wx, wy)
    err = np.hypot(v[jj, ii, 0] - px, v[jj, ii, 1] - py)
    nstars = int(m.num_stars)
    m.close()
    return {"sample": f"{n} random corners of cell rows {j0}..{j0 + 2} of {ny}, direct sum over all "
                      f"{nstars} stars {dt:.1f} s",
            "median_px": float(np.median(err)), "p99_px": float(np.quantile(err, 0.99)), "max_px": float(err.max())}


CCF_CASES = (137, 1000, 4000)  # stars; kappa_tot 0.3, shear 0.3, kappa_star 0.27 (the reference CCF defaults)


def ccf_stars(n, seed=7, kstar=0.27):
    """Seeded equal-mass circular field of n stars and its radius (the reference's
    CCF field size for n stars, include/ccf.cuh:427-432)."""
    rng = np.random.default_rng(seed)
    rad = np.sqrt(n / kstar)
    r = rad * np.sqrt(rng.random(n))
    a = 2 * np.pi * rng.random(n)
    return np.stack([r * np.cos(a), r * np.sin(a), np.ones(n)], 1), rad


def ccf_write_stars(path, stars, rad):
    with open(path, "wb") as f:
        f.write(np.array([len(stars), 0], np.int32).tobytes())
        f.write(np.array([rad, 0.0, 1.0]).tobytes())
        f.write(np.ascontiguousarray(stars, np.float64).tobytes())


def ccf_measure():
    """Critical curves (CCF, 100 phi steps, one branch) of seeded equal-mass
    fields: device time of the root finding (branch centres + phi steps), the
    critical-curve points found per second, the largest error in 1/mu."""
    import tempfile

    import irs_b200
    res = {}
    with tempfile.TemporaryDirectory() as td:
        for n in CCF_CASES:
            stars, rad = ccf_stars(n)
            sf = os.path.join(td, f"s{n}.bin")
            ccf_write_stars(sf, stars, rad)
            c = irs_b200.CCF(kappa_tot=0.3, shear=0.3, starfile=sf, num_phi=100, write_caustics=True)
            c.run()
            c.run()  # warm
            t = c.value("t_init_roots") + c.t_ccs
            pts = c.num_roots * 101
            res[f"stars_{n}"] = {"roots": c.num_roots, "points": pts, "root_finding_ms": t * 1e3,
                                 "caustics_ms": c.value("t_caustics") * 1e3, "points_per_s": pts / t,
                                 "max_error_inv_mu": c.value("max_error"),
                                 "expansion_order": int(c.value("expansion_order"))}
            res[f"stars_{n}"]["ncc"] = ncc_measure(c.caustics)
            c.close()
    return res


def ncc_hl(caus):
    """Half length of a square NCC region holding the caustics' central part."""
    return float(np.quantile(np.abs(caus[..., :2]).ravel(), 0.9))


def ncc_measure(caus, npix=1000, over_sample=2):
    """Caustic-crossing map (NCC, 1000^2 pixels, over_sample 2) of a CCF run's
    caustics: device time of the crossings and the block maximum."""
    import irs_b200
    hl = ncc_hl(caus)
    n = irs_b200.NCC(half_length_y1=hl, half_length_y2=hl, num_pixels_y1=npix, num_pixels_y2=npix,
                     over_sample=over_sample, write_histograms=False)
    n.set_caustics(caus)
    n.run()
    n.run()  # warm
    t = n.value("t_ncc") + n.value("t_reduce")
    out = {"half_length": hl, "segments": int(caus.shape[0] * (caus.shape[1] - 1)), "pixels": npix * npix,
           "over_sample": over_sample, "ms": t * 1e3, "pixels_per_s": npix * npix / t,
           "max_crossings": int(n.value("max_num"))}
    n.close()
    return out


def ccf_cpu_reference(gpu_res, cases=(137, 400)):
    """The reference's own CCF (include/ccf.cuh, compiled for the host; its
    kernels on one host thread) on the same fields, and the GPU's curves
    against it (the two update schemes label the roots differently: matched
    at the branch centre)."""
    import tempfile

    from scipy.optimize import linear_sum_assignment

    import irs_b200
    from oracle import ccf_ref, pyoracle as po
    if not po.ref_ccf_available():
        return {"unavailable": "oracle/_ref/libref_ccf.so not built"}
    out = {}
    with tempfile.TemporaryDirectory() as td:
        for n in cases:
            stars, rad = ccf_stars(n)
            init = ccf_ref.initial_roots(stars, 2 * n, 100, 1, rad)
            lens = po.lens(0.3, 0.3, float(np.sum(stars[:, 2]) / rad ** 2), 1.0, 0, 1, 1, (rad, 0.0))
            t0 = time.perf_counter()
            rc, rw, _, rme, _ = po.ref_ccf(stars, lens, rad * 1.1, init, 100, 1)
            t_cpu = time.perf_counter() - t0
            sf = os.path.join(td, f"s{n}.bin")
            ccf_write_stars(sf, stars, rad)
            c = irs_b200.CCF(kappa_tot=0.3, shear=0.3, starfile=sf, num_phi=100, write_caustics=False)
            c.run()
            g = c.critical_curves[..., 0] + 1j * c.critical_curves[..., 1]
            t_gpu = c.value("t_init_roots") + c.t_ccs
            c.close()
            d = np.abs(rc[:, 50][:, None] - g[:, 50][None, :])
            i, j = linear_sum_assignment(d)
            perm = np.empty_like(j)
            perm[i] = j
            out[f"stars_{n}"] = {"seconds": t_cpu, "cores": 1, "max_error_inv_mu": rme,
                                 "gpu_seconds": t_gpu, "speedup": t_cpu / t_gpu,
                                 "max_curve_deviation": float(np.abs(rc - g[perm]).max())}
            if n == cases[0]:  # the reference's NCC on these caustics (1000^2, over_sample 2)
                caus = rw  # the reference's caustics
                hl = ncc_hl(np.stack([caus.real, caus.imag], -1))
                t0 = time.perf_counter()
                ref_map = po.ref_ncc(caus, (0, 0), (hl, hl), (1000, 1000), 2)
                t_ref = time.perf_counter() - t0
                import irs_b200
                nn = irs_b200.NCC(half_length_y1=hl, half_length_y2=hl, num_pixels_y1=1000, num_pixels_y2=1000,
                                  over_sample=2, write_histograms=False)
                nn.set_caustics(caus)
                nn.run()
                nn.run()
                t_g = nn.value("t_ncc") + nn.value("t_reduce")
                out["ncc_reference"] = {"seconds": t_ref, "cores": 1, "gpu_seconds": t_g, "speedup": t_ref / t_g,
                                        "map_equal": bool(np.array_equal(nn.num_caustic_crossings, ref_map)),
                                        "sample": f"caustics of the {n}-star CCF of the reference, 1000^2, x4"}
                nn.close()
    return out


def our_arm(args):
    import torch

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    m = make_ipm(is_double=False, size=args.size)
    m.run()  # moves the star field to the device and builds everything once
    stars = m._host_stars.copy()  # the workload's field, as handed to set_stars
    npix = m.num_pixels_y1 * m.num_pixels_y2
    nx, ny = int(m.value("num_ray_threads_1")), int(m.value("num_ray_threads_2"))
    ncells, nverts = nx * ny, (nx + 1) * (ny + 1)

    # ---- device-resident pipeline
    for _ in range(args.warmup):
        m.rerun(1)
    sampler = ClockSampler(local)
    barrier()
    sampler.start()
    t_steps, t_lat, t_dep, launches = [], [], [], 0
    for _ in range(args.steps):
        t_steps.append(m.rerun(1))
        t_lat.append(m.value("t_lattice"))
        t_dep.append(m.value("t_deposit"))
        launches += int(m.value("launches"))
    barrier()
    clocks = sampler.stop()
    dev_time = float(np.sum(t_steps))
    if dist is not None:
        tt = torch.tensor([dev_time], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        dev_time = float(tt.item())
    value = ws * args.steps * npix / dev_time

    # ---- end to end through the C ABI with host buffers
    e = make_ipm(is_double=False, size=args.size)  # the same field, from host memory at every run()
    for _ in range(args.warmup):
        e.run()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e.run()  # the step's result: e.magnifications, a host array
    barrier()
    e2e_time = time.perf_counter() - t0
    if dist is not None:
        tt = torch.tensor([e2e_time], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_time = float(tt.item())
    h2d = stars.size * 4
    d2h = npix * 4 + 2 * stars.size * 4

    # ---- roofline of the dominant kernel
    lat_ms, dep_ms = float(np.mean(t_lat)) * 1e3, float(np.mean(t_dep)) * 1e3
    p = m.expansion_order
    near = m.value("mean_near")
    flop_per_vertex = 11 * near + 8 * p + 30
    peaks = measured_peaks()
    sm_mhz = peaks.get("sm_max_mhz", 1965.0)
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    if lat_ms >= dep_ms:
        achieved = flop_per_vertex * nverts / (lat_ms * 1e-3) / 1e12
        roof = {"kernel": "shoot_f32 (lattice lens equation)", "bound": "fp32", "achieved": achieved,
                "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak, "traffic": None,
                "peak_source": "148 SMs x 128 FP32 lanes x 2 x sm_max_mhz of MEASURED_PEAKS.json (derived)",
                "algorithmic": f"(11 x {near:.2f} near stars + 8 x {p} + 30) flop x {nverts} corners"}
    else:
        bytes_ = 16.0 * nverts + 8.0 * npix
        achieved = bytes_ / (dep_ms * 1e-3) / 1e9
        peak = peaks.get("hbm_gbs", 6650.0)
        # DRAM traffic measured with ncu (dram__bytes_read.sum + dram__bytes_write.sum) on the 500^2 case of
        # the same lens and pixel scale: 519 MB for 29.2 M cells, 17.8 B per cell, scaled to this launch
        traffic = 17.8 * ncells / 1e9
        roof = {"kernel": "ipm_deposit_cells", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "traffic_unit": "GB per launch",
                "traffic_source": "ncu on the 500^2 case (17.8 B per cell), scaled by cells",
                "limiter": "instruction issue and latency (ncu, 500^2 case: 65 % issue-active, ALU pipe 51 %)",
                "algorithmic": f"16 B x {nverts} corner positions + 8 B x {npix} map words"}
    # the lens-equation kernel against the FP32 FMA roofline, whichever kernel dominates
    lens_tflops = flop_per_vertex * nverts / (lat_ms * 1e-3) / 1e12
    roof_lens = {"kernel": "shoot_f32 (lattice lens equation)", "bound": "fp32", "achieved": lens_tflops,
                 "peak": fp32_peak, "unit": "TFLOP/s", "frac": lens_tflops / fp32_peak, "ms": lat_ms,
                 "peak_source": "148 SMs x 128 FP32 lanes x 2 x sm_max_mhz of MEASURED_PEAKS.json (derived)",
                 "algorithmic": f"(11 x {near:.2f} near stars + 8 x {p} + 30) flop x {nverts} corners"}

    # ---- secondary measurements (not the headline): the plain FP64 form of the
    # same IPM workload, and IRS on the plain-IRS case in both forms
    extra = {}
    if not args.no_extra:
        plain = make_ipm(is_double=True, size=args.size)
        plain.run()
        tp = [plain.rerun(1) for _ in range(max(2, args.steps // 2))]
        extra["ipm_fp64_plain"] = {"pixels_per_s": npix / float(np.mean(tp)), "ms_per_step": float(np.mean(tp)) * 1e3,
                                   "lattice_ms": plain.value("t_lattice") * 1e3,
                                   "deposit_ms": plain.value("t_deposit") * 1e3,
                                   "tree_expansions_ms": (plain.value("t_pipeline") - plain.value("t_shoot")) * 1e3}
        extra["ipm_fp32_over_fp64"] = float(np.mean(tp)) / (dev_time / args.steps)
        plain.close()
        import irs_b200
        for dbl, key in [(False, "irs_case1_fp32"), (True, "irs_case1_fp64_plain")]:
            r = irs_b200.IRS(**IRS_CASE1, is_double=dbl)
            r.run()
            ts = [r.rerun(1) for _ in range(3)]
            rays = r.num_rays_shot
            extra[key] = {"rays_per_s": rays / float(np.mean(ts)), "rays": int(rays), "stars": int(r.num_stars),
                          "ms_per_step": float(np.mean(ts)) * 1e3, "shoot_ms": r.value("t_lattice") * 1e3,
                          "rays_received": int(r.num_rays_received)}
            if not dbl:  # the lens kernel against the FP32 FMA roofline (flop per ray as for a lattice corner)
                fl = (11 * r.value("mean_near") + 8 * r.expansion_order + 30) * rays / (r.value("t_lattice") * 1e12)
                extra[key]["lens_tflops"] = fl
                extra[key]["lens_frac_of_fp32_peak"] = fl / fp32_peak
            r.close()
        # the workload's lens through the graph-captured pipeline (one realization, the
        # library's own star field of the workload's seed), against the same realization run singly
        import irs_b200
        w = {k: v for k, v in WORKLOAD.items() if k not in ("name", "expansion_order")}
        gb = irs_b200.BatchIPM([{**w, "theta_star": m.theta_star}], expansion_order=p)
        gb.run()
        tg = [gb.rerun(1) for _ in range(max(3, args.steps))]
        seeded = make_ipm(is_double=False, size=args.size, stars=False)
        seeded.run()
        extra["ipm_graph_single"] = {"pixels_per_s": npix / float(np.median(tg)),
                                     "ms_per_step": float(np.median(tg)) * 1e3,
                                     "graph_nodes": int(gb.value("graph_nodes")),
                                     "map_equals_single_run": bool(np.array_equal(gb.maps[0],
                                                                                  seeded.magnifications))}
        seeded.close()
        gb.close()
        extra["config3"] = config3_measure()
        extra["batched_256"] = batch_measure(args.steps)
        extra["learned_adaptive"] = adaptive_measure()
        extra["ccf"] = ccf_measure()

    if rank == 0:
        cpu, errs = None, None
        if ws == 1 and not args.no_cpu:
            cpu, errs = cpu_baseline(m, stars.astype(np.float64), os.cpu_count() or 1)
            if not args.no_extra:
                cpu["ccf_reference"] = ccf_cpu_reference(extra.get("ccf"))
            errs["irs_case1"] = irs_case1_errors(os.cpu_count() or 1)
            if not args.no_extra:
                errs["config3_ipm_corners"] = config3_errors(os.cpu_count() or 1)
        out = {
            "metric": "IPM pixels/s", "value": value, "unit": "pixels/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_time / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(m.num_stars, ws) if args.size == "full" else
            {**workload_config(m.num_stars, ws), "workload": WORKLOAD["name"] + "_small500px"},
            "lattice": {"cells": ncells, "nx": nx, "ny": ny},
            "form": "FP32 leaf-relative, compensated near field, FP64 expansions",
            "e2e": {"value": ws * args.steps * npix / e2e_time, "unit": "pixels/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "roofline": roof,
            "roofline_lens": roof_lens,
            "kernels_ms": {"lattice": lat_ms, "deposit": dep_ms, "pipeline": dev_time / args.steps * 1e3},
            "mean_near_stars": near,
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "error_vs_fp64_oracle": errs,
            "secondary": extra,
        }
        print(json.dumps(out))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-extra", action="store_true", help="skip the secondary measurements")
    ap.add_argument("--size", default="full", choices=["full", "small"],
                    help="small: 500 x 500 map at the same pixel scale (for profiler captures)")
    ap.add_argument("--case", default=None, choices=["config3-irs-band", "config3-ipm-band", "adaptive"],
                    help="profiler capture of one case: config3-irs-band = the rectangular Kroupa IRS configuration "
                         "(order 16, 64 rays per pixel) on 512 ray rows through the lattice centre, --steps runs; "
                         "adaptive = the learned-adaptive map (4096^2), --steps runs")
    args = ap.parse_args()
    if args.case:
        profile_case(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        our_arm(args)


def profile_case(args):
    """A small case for profiler captures (not a bench line): prints the
    device time per run of the IRS lens-equation kernel or of the IPM
    deposition on a band of the rectangular Kroupa configuration, or of the
    adaptive map's base and adaptive passes."""
    import irs_b200
    if args.case == "adaptive":
        a = irs_b200.AdaptiveIPM(tolerance=1e-3, audit_fraction=0.0025, audit_bound=0.05, **ADAPTIVE_CONFIG)
        for _ in range(max(1, args.steps)):
            a.run()
        print(json.dumps({"case": args.case, "t_base_ms": a.value("t_base") * 1e3, "t_adapt_ms": a.value("t_adapt") * 1e3,
                          "t_refine_deposit_ms": a.value("t_refine_deposit") * 1e3,
                          "cells_evaluated": a.value("cells_evaluated")}))
        a.close()
        return
    if args.case == "config3-ipm-band":  # the 512 lattice rows through the centre
        m = irs_b200.IPM(**CONFIG3, num_rays_y=1, is_double=False)
        m.derive()
        ny = int(m.value("num_ray_threads_2"))
        m.lib.set_band(m.obj, ny // 2 - 256, ny // 2 + 256)
        m.run()
        ts = []
        for _ in range(max(1, args.steps)):
            m.rerun(1)
            ts.append(m.value("t_deposit"))
        cells = int(m.value("num_ray_threads_1")) * 512
        print(json.dumps({"case": args.case, "cells": cells, "deposit_ms": float(np.min(ts)) * 1e3,
                          "cells_per_s": cells / float(np.min(ts))}))
        m.close()
        return
    r = irs_b200.IRS(**CONFIG3, num_rays_y=64, is_double=False)
    r.derive()
    ny = int(r.value("num_ray_threads_2"))
    r.lib.set_band(r.obj, ny // 2 - 256, ny // 2 + 256)
    r.run()
    ts = []
    for _ in range(max(1, args.steps)):
        r.rerun(1)
        ts.append(r.value("t_lattice"))
    print(json.dumps({"case": args.case, "rays": int(r.num_rays_shot), "lattice_ms": float(np.min(ts)) * 1e3,
                      "rays_per_s": r.num_rays_shot / float(np.min(ts)), "mean_near_stars": r.value("mean_near"),
                      "order": r.expansion_order}))
    r.close()


if __name__ == "__main__":
    main()

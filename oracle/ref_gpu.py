"""The reference's own GPU code, run as a comparison fixture (test
infrastructure and the reference arm of bench.py; never part of the product).

`make -C oracle refgpu` builds, from the weisluke/irs sources, its
`src/lib_ipm.cu` (float and double) and the IRS command-line tool
`src/main_ipm_irs.cu -D is_irs` with the reference's own `compile` flags
(`nvcc -std=c++20 --use_fast_math -O3`) plus the B200 target, into
oracle/_ref/gpu/bin/, and copies its Python package `microlensing/` unchanged
beside it (the layout `microlensing/IPM/lib_ipm.py:5` loads from).

Every call runs in a child process: the reference's `IPM.run()` and `IRS.run()`
begin with `cudaDeviceReset()` (include/ipm.cuh:164, include/irs.cuh:161),
which would free every allocation of the caller's CUDA context.

Functions:
  available()                       the build is present
  write_starfile(path, stars, ...)  a star field in the reference's .bin layout
                                    (include/star.cuh:498-534)
  read_starfile(path)               the same layout, float or double
  run_ipm(params, ...)              the reference's IPM through its unchanged
                                    `microlensing.IPM.IPM` wrapper
  run_irs(params, ...)              the reference's `irs_gpu` tool
  read_param_info(path)             `*_parameter_info.txt` as a dict
  read_map(path)                    a `*_magnifications.bin` map
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REFGPU = os.path.join(HERE, "_ref", "gpu")


def available(kind: str = "ipm") -> bool:
    need = {"ipm": ["bin/lib_ipm.so", "bin/lib_ipm_double.so", "microlensing/IPM/ipm.py"],
            "irs": ["bin/irs_gpu", "bin/irs_gpu_double"]}[kind]
    return all(os.path.exists(os.path.join(REFGPU, f)) for f in need)


def write_starfile(path: str, stars: np.ndarray, rectangular: bool, corner, theta: float, double: bool = True):
    """nstars (int), rectangular (int), corner (complex T; (|corner|, 0) for a
    circle), theta (T), then {x1, x2, m} per star in T (star.cuh:498-534)."""
    T = np.float64 if double else np.float32
    c = (float(corner[0]), float(corner[1])) if rectangular else (float(np.hypot(*corner)), 0.0)
    with open(path, "wb") as f:
        f.write(np.array([len(stars), int(bool(rectangular))], np.int32).tobytes())
        f.write(np.array([c[0], c[1], theta], T).tobytes())
        f.write(np.ascontiguousarray(stars, T).tobytes())


def read_starfile(path: str):
    """(stars float64 [N, 3], rectangular, corner, theta): float or double by
    the file size, as star.cuh:175-260 decides."""
    raw = open(path, "rb").read()
    n, rect = np.frombuffer(raw[:8], np.int32)
    for T in (np.float64, np.float32):
        b = np.dtype(T).itemsize
        if len(raw) == 8 + 3 * b + 3 * b * n:
            hdr = np.frombuffer(raw[8:8 + 3 * b], T)
            st = np.frombuffer(raw[8 + 3 * b:], T).reshape(n, 3).astype(np.float64)
            return st, int(rect), (float(hdr[0]), float(hdr[1])), float(hdr[2])
    raise ValueError(f"{path}: size matches neither a float nor a double star file of {n} stars")


def read_param_info(path: str) -> dict:
    out = {}
    for line in open(path):
        p = line.split()
        if len(p) == 2:
            try:
                out[p[0]] = float(p[1])
            except ValueError:
                out[p[0]] = p[1]
    return out


def read_map(path: str, dtype) -> np.ndarray:
    """`write_array` layout (array_functions.cuh:280-306): int nrows, int
    ncols, then the row-major data."""
    raw = open(path, "rb").read()
    ny, nx = np.frombuffer(raw[:8], np.int32)
    return np.frombuffer(raw[8:], dtype).reshape(ny, nx).copy()


def _worker(spec_path: str):
    """Child process: the reference IPM through its unchanged wrapper."""
    import time
    spec = json.load(open(spec_path))
    sys.path.insert(0, REFGPU)
    from microlensing.IPM.ipm import IPM  # the reference's own package, unchanged

    m = IPM(**spec["params"], verbose=0, is_double=spec["is_double"])
    walls, shoots = [], []
    for _ in range(spec["repeats"]):
        t0 = time.perf_counter()
        m.run()
        walls.append(time.perf_counter() - t0)
        if not spec["is_double"]:  # lib_ipm_double.py binds no get_t_shoot_cells
            shoots.append(float(m.t_shoot_cells))
    if spec.get("save"):
        if not m.lib.save(m.obj, 0):
            raise RuntimeError("reference IPM save() failed")
    out = {"magnifications": m.magnifications, "stars": m.stars, "walls": np.array(walls),
           "t_shoot_cells": np.array(shoots), "num_stars": m.num_stars, "corner": np.array(m.corner)}
    if m.write_parities:
        out["minima"] = m.magnifications_minima
        out["saddles"] = m.magnifications_saddles
    np.savez(spec["out"], **out)


def run_ipm(params: dict, is_double: bool = False, repeats: int = 1, outdir: str | None = None,
            timeout: float = 900.0) -> dict:
    """The reference IPM with `params` (keyword arguments of
    microlensing.IPM.IPM). With `outdir`, the reference's save() also writes
    its files there (prefix outdir/) and `param_info` is returned."""
    if not available("ipm"):
        raise RuntimeError("the reference's GPU build (oracle/_ref/gpu) is missing")
    with tempfile.TemporaryDirectory() as td:
        p = dict(params)
        if outdir is not None:
            p["outfile_prefix"] = os.path.join(outdir, "")
        spec = {"params": p, "is_double": bool(is_double), "repeats": int(repeats), "save": outdir is not None,
                "out": os.path.join(td, "out.npz")}
        sp = os.path.join(td, "spec.json")
        json.dump(spec, open(sp, "w"))
        r = subprocess.run([sys.executable, "-m", "oracle.ref_gpu", sp], cwd=ROOT, capture_output=True, text=True,
                           timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"reference IPM failed (rc {r.returncode}): {r.stderr[-2000:]} {r.stdout[-2000:]}")
        z = np.load(spec["out"])
        out = {k: z[k] for k in z.files}
    if outdir is not None:
        out["param_info"] = read_param_info(os.path.join(outdir, "ipm_parameter_info.txt"))
    return out


IRS_OPTS = {"kappa_tot": "-k", "shear": "-y", "smooth_fraction": "-s", "kappa_star": "-ks", "theta_star": "-t",
            "mass_function": "-mf", "m_solar": "-ms", "m_lower": "-ml", "m_upper": "-mh", "light_loss": "-ll",
            "rectangular": "-r", "approx": "-a", "safety_scale": "-ss", "starfile": "-sf", "center_y1": "-cy1",
            "center_y2": "-cy2", "half_length_y1": "-hly1", "half_length_y2": "-hly2", "num_pixels_y1": "-npy1",
            "num_pixels_y2": "-npy2", "num_rays_y": "-nry", "random_seed": "-rs", "write_stars": "-ws",
            "write_maps": "-wm", "write_parities": "-wp", "write_histograms": "-wh"}


def run_irs(params: dict, outdir: str, is_double: bool = False, timeout: float = 900.0) -> dict:
    """The reference's `irs_gpu` tool (option table src/main_ipm_irs.cu:41-72)
    with its outputs under outdir/: the ray-count map, the parameter info and
    the wall time of the process."""
    import time
    if not available("irs"):
        raise RuntimeError("the reference's GPU build (oracle/_ref/gpu) is missing")
    exe = os.path.join(REFGPU, "bin", "irs_gpu_double" if is_double else "irs_gpu")
    args = [exe]
    for k, v in params.items():
        if isinstance(v, bool):
            v = int(v)
        args += [IRS_OPTS[k], str(v)]
    args += ["-wm", "1", "-o", os.path.join(outdir, "")]
    t0 = time.perf_counter()
    r = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
    wall = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError(f"reference irs_gpu failed (rc {r.returncode}): {r.stderr[-2000:]} {r.stdout[-2000:]}")
    info = read_param_info(os.path.join(outdir, "irs_parameter_info.txt"))
    mp = read_map(os.path.join(outdir, "irs_magnifications.bin"), np.int32)
    return {"magnifications": mp, "param_info": info, "wall": wall}


if __name__ == "__main__":
    _worker(sys.argv[1])

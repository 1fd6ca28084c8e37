"""Readers and writers of the files the map makers exchange with their users:
parameter lists, star fields, 2-d arrays (maps) and histograms.

Same names, arguments and results as the reference's helper module
(microlensing/Util/util.py:5-125), so scripts and notebooks written against
it read this library's outputs unchanged. File layouts, all native-endian:

* parameter list (`*_parameter_info.txt`): one `key value` pair per line,
  whitespace separated (ipm.cuh:1133-1207 writes it);
* star field (`*_stars.bin`, also the `starfile` input): int32 number of
  stars, int32 rectangular flag, two values of the corner (x1, x2) — for a
  circular field (radius, 0) — one value theta_star, then x1, x2, mass per
  star; values float32 or float64 (star.cuh:498-534);
* 2-d array (`*_magnifications*.bin`): int32 rows, int32 columns, then the
  values row by row, (re, im) pairs for complex data
  (array_functions.cuh:280-306);
* histogram (`*_histogram.txt`): integer `value count` lines
  (array_functions.cuh:318-349).
"""
import numpy as np

_STAR_TYPES = {np.dtype(np.float32): np.float32, np.dtype(np.float64): np.float64}


def read_params(fname: str) -> dict:
    """`key value` lines -> dict. A value that parses as a number becomes an
    int when it is integral (and finite), else a float; any other value stays
    the string. Blank lines are skipped; a line with other than two fields
    raises ValueError."""
    params = {}
    with open(fname) as f:
        for n, line in enumerate(f, 1):
            fields = line.split()
            if not fields:
                continue
            if len(fields) != 2:
                raise ValueError(f"{fname}:{n}: expected 'key value', got {line.rstrip()!r}")
            key, text = fields
            try:
                v = float(text)
            except ValueError:
                params[key] = text
                continue
            params[key] = int(v) if np.isfinite(v) and v == int(v) else v
    return params


def _star_type(dtype):
    t = _STAR_TYPES.get(np.dtype(dtype))
    if t is None:
        raise ValueError("dtype must be np.float32 or np.float64")
    return t


def read_stars(fname: str, dtype=np.float32):
    """A star-field file -> (stars [n, 3] of x1, x2, mass; rectangular flag;
    corner (2,); theta_star), values of type `dtype` (the file's own type:
    float32 unless it was written as float64)."""
    t = _star_type(dtype)
    raw = np.fromfile(fname, dtype=np.uint8)
    nstars, rect = np.frombuffer(raw[:8].tobytes(), dtype=np.int32)
    body = np.frombuffer(raw[8:].tobytes(), dtype=t)
    corner = body[:2].copy()
    theta_star = body[2]
    stars = body[3:].reshape(int(nstars), 3).copy()
    return stars, bool(rect), corner, theta_star


def write_stars(fname: str, nstars: int, rectangular: bool, corner, theta_star: float, stars, dtype=np.float32):
    """Write a star-field file (layout in the module docstring). `fname` must
    end in .bin and `dtype` be np.float32 or np.float64 (ValueError
    otherwise); `stars` holds x1, x2, mass per star and is written whole."""
    if not fname.endswith(".bin"):
        raise ValueError("fname must be a .bin file")
    t = _star_type(dtype)
    head = np.array([nstars, 1 if rectangular else 0], dtype=np.int32)
    vals = np.concatenate([np.asarray(corner, dtype=t).ravel()[:2], np.asarray([theta_star], dtype=t),
                           np.asarray(stars, dtype=t).ravel()])
    with open(fname, "wb") as f:
        f.write(head.tobytes())
        f.write(vals.tobytes())


def read_array(fname: str, dtype, is_complex: bool = False):
    """A 2-d array file -> array [rows, cols] of `dtype` ([rows, cols, 2] for
    complex data stored as (re, im) pairs)."""
    raw = np.fromfile(fname, dtype=np.uint8)
    nrows, ncols = (int(v) for v in np.frombuffer(raw[:8].tobytes(), dtype=np.int32))
    dat = np.frombuffer(raw[8:].tobytes(), dtype=dtype).copy()
    return dat.reshape((nrows, ncols, 2) if is_complex else (nrows, ncols))


def read_hist(fname: str):
    """A histogram file -> int32 array [bins, 2] of (value, number of pixels)."""
    return np.loadtxt(fname, dtype=np.int32)

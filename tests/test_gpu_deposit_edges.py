"""Deposition edge cases on the GPU, on corner lattices given directly.

The reference tests its deposition only through whole maps; the cases here
are the ones its polygon code has to get right on the way (ipm_functions.cuh:
168-216, polygon.cuh:349-467): cell edges lying exactly on pixel lines (a lens
with no deflection), corners that are NaN, cells partly or wholly outside the
map, triangles over the 1e4 area limit and cells of zero area. The lattice
is deposited through the allocation-free entry point and compared bit for bit
with the oracle's fixed-point deposition; where the reference polygon
algorithm is exact (pixel-aligned cells), also with it.
"""
import ctypes

import numpy as np
import pytest

from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def _lattice(kind):
    rng = np.random.default_rng(7)
    if kind == "aligned":
        return np.stack(np.meshgrid(np.arange(5, 26, 1.0), np.arange(4, 31, 1.0)), -1)
    if kind == "half_aligned":
        return np.stack(np.meshgrid(np.arange(-3, 45, 0.5), np.arange(-2, 44, 0.5)), -1)
    if kind == "jitter_edges":
        v = np.stack(np.meshgrid(np.arange(-8, 48, 0.75), np.arange(-8, 48, 0.75)), -1)
        return v + rng.normal(0, 0.3, v.shape)
    if kind == "nan_huge_degenerate":
        v = np.stack(np.meshgrid(np.linspace(2, 38, 31), np.linspace(1, 37, 29)), -1) + rng.normal(0, 0.4, (29, 31, 2))
        v[3, 4] = np.nan
        v[10, 7, 1] = np.nan
        v[15, 15] = (1.0e5, -3.0e5)      # cells around it exceed the area limit
        v[20, 20:23] = v[20, 19]         # zero-area cells
        v[0, :, 1] = -50.0               # a row of cells reaching far outside
        return v
    raise ValueError(kind)


@pytest.mark.parametrize("dbl", [False, True])
@pytest.mark.parametrize("kind", ["aligned", "half_aligned", "jitter_edges", "nan_huge_degenerate"])
def test_deposit_edge_lattices(gpu, dbl, kind):
    import torch
    import irs_b200._lib as L

    lib = L.load("ipm", dbl)
    T, tdt = (ctypes.c_double, torch.float64) if dbl else (ctypes.c_float, torch.float32)
    f = lib.ipm_deposit_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong, T, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    v = np.ascontiguousarray(_lattice(kind), np.float64)
    ncy, ncx = v.shape[0] - 1, v.shape[1] - 1
    npx, npy = 40, 36
    factor = 0.75
    d_v = torch.from_numpy(v).to("cuda")
    d_map = torch.full((npy, npx), -1.0, dtype=tdt, device="cuda")
    rc = f(d_v.data_ptr(), ncx, ncy, factor, npx, npy, d_map.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    got = d_map.cpu().numpy()
    q = po.ipm_deposit_fixed(v, np.float32(factor) if not dbl else factor, (npx, npy), single=not dbl)
    want = (q.astype(np.float64) * 2.0 ** -32).astype(got.dtype)
    np.testing.assert_array_equal(got, want)
    if kind in ("aligned", "half_aligned"):
        np.testing.assert_array_equal(got, po.ipm_deposit_ref(v, factor, (npx, npy)).astype(got.dtype))

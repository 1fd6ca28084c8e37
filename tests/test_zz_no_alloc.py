"""The allocation-free deposition entry point, for callers that cannot let a
library allocate device memory (their own memory pool or budget owns it, or a
latency-critical loop cannot afford the synchronisation of cudaMalloc).

It is called through the C ABI on a corner lattice already on the device and
its map is compared with the map that the allocating path (run()) produced
from the same corners, twice in a row: the deposition is fixed point and
deterministic, so the tolerance is exact equality, as for the other deposition
tests. This file is collected last so that a run stopping at the first failure
has run every other test before it.
"""
import ctypes

import numpy as np
import pytest

import irs_b200
from tests.cases import IPM_SMALL

pytestmark = pytest.mark.gpu


def _bind(lib, T):
    f = lib.ipm_deposit_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong, T, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


@pytest.mark.parametrize("dbl", [False, True])
def test_no_alloc_deposit_matches_allocating_path(gpu, dbl):
    import torch

    m = irs_b200.IPM(**IPM_SMALL, is_double=dbl, expansion_order=12)
    m.run()
    verts = m.vertices()
    ncy, ncx = verts.shape[0] - 1, verts.shape[1] - 1
    npx, npy = m.num_pixels
    rhs1, rhs2 = m.value("ray_half_sep_1"), m.value("ray_half_sep_2")
    hx, hy = m.half_length
    if dbl:
        T, tdt = ctypes.c_double, torch.float64
        factor = 2 * rhs1 * rhs2 * npx * npy / (2 * hx * 2 * hy)
    else:
        T, tdt = ctypes.c_float, torch.float32
        f32 = np.float32
        factor = float(f32(f32(f32(f32(f32(2) * f32(rhs1)) * f32(rhs2)) * f32(npx)) * f32(npy))
                       / f32(f32(f32(f32(2) * f32(hx)) * f32(2)) * f32(hy)))
    fn = _bind(m.lib, T)
    d_verts = torch.from_numpy(np.ascontiguousarray(verts)).to("cuda")
    stream = torch.cuda.current_stream()
    for call in range(2):
        d_map = torch.full((npy, npx), -1.0, dtype=tdt, device="cuda")
        rc = fn(d_verts.data_ptr(), ncx, ncy, factor, npx, npy, d_map.data_ptr(), stream.cuda_stream)
        assert rc == 0, f"call {call} returned {rc}"
        torch.cuda.synchronize()
        got = d_map.cpu().numpy()
        np.testing.assert_array_equal(got, m.magnifications)


def test_no_alloc_rejects_sizes_beyond_the_limit(gpu):
    lib = irs_b200.IPM(**IPM_SMALL).lib
    fn = _bind(lib, ctypes.c_float)
    # 2048 x 600 pixels exceeds 1024 * 1024 pixels in all: rejected before any GPU work
    assert fn(ctypes.c_void_p(16), 4, 4, 0.5, 2048, 600, ctypes.c_void_p(16), None) == 1
    # 1025 rows exceed the 1024-row limit
    assert fn(ctypes.c_void_p(16), 4, 4, 0.5, 64, 1025, ctypes.c_void_p(16), None) == 1


def test_no_alloc_accepts_a_wide_map(gpu):
    """2048 x 512 pixels: within 1024 * 1024 pixels in all and 1024 rows. A
    coarse unit lattice over the map deposits one unit of area per pixel."""
    import torch
    lib = irs_b200.IPM(**IPM_SMALL).lib
    fn = _bind(lib, ctypes.c_float)
    npx, npy = 2048, 512
    v = np.stack(np.meshgrid(np.arange(0, npx + 1, 4.0), np.arange(0, npy + 1, 4.0)), -1)
    d_v = torch.from_numpy(np.ascontiguousarray(v)).to("cuda")
    d_map = torch.full((npy, npx), -1.0, dtype=torch.float32, device="cuda")
    # each 4 x 4 cell has area 16 = two triangles of 8: factor 8 spreads 1 per pixel
    rc = fn(d_v.data_ptr(), v.shape[1] - 1, v.shape[0] - 1, 8.0, npx, npy, d_map.data_ptr(),
            torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    np.testing.assert_allclose(d_map.cpu().numpy(), np.ones((npy, npx), np.float32), rtol=0, atol=1e-6)

"""One magnification map split over several GPUs.

Each rank (one process per GPU, torch.distributed) computes a contiguous band
of lattice rows -- rays for IRS, cells for IPM -- of the same realisation:
every rank builds the same star field (same seed, deterministic generation),
the same tree and expansions, shoots only its band into a full-size integer
map (IRS ray counts, IPM 64-bit fixed point), and one all-reduce (sum) over
the ranks gives the map. Integer sums do not depend on the order of the
reduction, so the result is bit-identical to the single-GPU map. On NCCL the
reduction runs on device buffers over NVLink; on gloo it runs on host copies.
"""
from __future__ import annotations

import numpy as np


def band_of(rank: int, world: int, nrows: int) -> tuple[int, int]:
    """Rows [first, last) of `rank`'s band: contiguous, sizes differ by at most one."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("rank must be in [0, world)")
    return (rank * nrows) // world, ((rank + 1) * nrows) // world


def integer_map_dtype(kind: str):
    return np.int32 if kind == "irs" else np.uint64


def reduce_integer_map(partial: np.ndarray, group=None) -> np.ndarray:
    """Sum a host integer map over the ranks of `group` (uint64 sums wrap modulo 2^64, as on the GPU)."""
    import torch
    import torch.distributed as dist
    a = np.ascontiguousarray(partial)
    t = torch.from_numpy(a.view(np.int64) if a.dtype == np.uint64 else a).clone()
    dist.all_reduce(t, group=group)
    out = t.numpy()
    return out.view(np.uint64) if a.dtype == np.uint64 else out


def sharded_run(maker, group=None):
    """Compute `maker`'s map (an irs_b200.IPM or IRS) over the ranks of `group`.

    Returns (total, minima, saddles) as magnifications (IPM) or ray counts
    (IRS); minima / saddles are None without write_parities.
    """
    import torch
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    kind = maker._kind
    seed = torch.tensor([int(maker.random_seed)], dtype=torch.int64)
    if dist.get_backend(group) == "nccl":
        seed = seed.cuda()
    dist.broadcast(seed, src=0, group=group)
    seed = int(seed.item())
    if seed == 0 and not maker.starfile and maker._host_stars is None:
        raise ValueError("a sharded run needs a fixed random_seed (or a star file) shared by all ranks")
    maker.random_seed = seed
    maker.derive()
    nrows = int(maker.value("num_ray_threads_2"))
    lo, hi = band_of(rank, world, nrows)
    maker.lib.set_band(maker.obj, lo, hi)
    maker.run()
    npy, npx = maker.num_pixels_y2, maker.num_pixels_y1
    par = maker.write_parities
    names = ["minima", "saddles"] if par else ["total"]
    if dist.get_backend(group) == "nccl":
        tdt = torch.int32 if kind == "irs" else torch.int64
        bufs = [torch.zeros((npy, npx), dtype=tdt, device="cuda") for _ in names]
        ptrs = [b.data_ptr() for b in bufs]
        args = ([ptrs[0], None, None] if not par else [None, ptrs[0], ptrs[1]])
        if not maker.lib.copy_maps_device(maker.obj, *args):
            raise RuntimeError("copy_maps_device failed")
        for b in bufs:
            dist.all_reduce(b, group=group)
        maps = [b.cpu().numpy() for b in bufs]
        if kind == "ipm":
            maps = [m.view(np.uint64) for m in maps]
    else:
        if kind == "ipm":
            host = maker.fixed_maps()
            host = list(host) if par else [host]
        else:
            host = ([maker.magnifications_minima, maker.magnifications_saddles] if par
                    else [maker.magnifications])
        maps = [reduce_integer_map(h.astype(integer_map_dtype(kind)), group) for h in host]
    if kind == "ipm":
        T = np.float64 if maker.is_double else np.float32
        # modulo 2^64, read as signed; a few units below zero read as 0
        maps = [(np.maximum(m.view(np.int64), 0).astype(np.float64) / 2.0 ** 32).astype(T) for m in maps]
    if par:
        return maps[0] + maps[1], maps[0], maps[1]
    return maps[0], None, None

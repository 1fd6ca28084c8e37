"""Row-band sharding of one map over ranks with an integer all-reduce: the
partition logic and the reduction run as world-size-2 gloo ranks on CPU (the
oracle's fixed-point deposition stands in for each rank's GPU band); the GPU
test checks on one device that bands of the real kernels sum to the full map."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from irs_b200.sharded import band_of, reduce_integer_map


def test_band_partition_covers_rows_once():
    for world in (1, 2, 3, 8):
        for nrows in (0, 1, 7, 23552):
            bands = [band_of(r, world, nrows) for r in range(world)]
            assert bands[0][0] == 0 and bands[-1][1] == nrows
            for (a, b), (c, d) in zip(bands, bands[1:]):
                assert b == c and a <= b
            sizes = [b - a for a, b in bands]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        band_of(2, 2, 10)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _lattice():
    rng = np.random.default_rng(5)
    v = np.stack(np.meshgrid(np.linspace(-4, 44, 61), np.linspace(-6, 40, 53)), -1)
    return v + rng.normal(0, 0.45, v.shape)


def _worker(rank, world, port, out):
    import torch.distributed as dist

    from oracle import pyoracle as po
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    v = _lattice()
    ncells = v.shape[0] - 1
    lo, hi = band_of(rank, world, ncells)
    part = po.ipm_deposit_fixed(v[lo:hi + 1], 0.75, (40, 40), single=True)
    full = reduce_integer_map(part)
    if rank == 0:
        np.save(out, full)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_band_reduction_is_exact(tmp_path):
    from oracle import pyoracle as po
    out = str(tmp_path / "sum.npy")
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    got = np.load(out)
    ref = po.ipm_deposit_fixed(_lattice(), 0.75, (40, 40), single=True)
    np.testing.assert_array_equal(got, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["ipm", "irs"])
def test_gpu_bands_sum_to_full_map(gpu, kind):
    import irs_b200
    from tests.cases import IPM_SMALL, IRS_SMALL
    cls, cfg = (irs_b200.IPM, IPM_SMALL) if kind == "ipm" else (irs_b200.IRS, IRS_SMALL)
    full = cls(**cfg, expansion_order=10)
    full.run()
    nrows = int(full.value("num_ray_threads_2"))
    acc = None
    for r in range(3):
        m = cls(**cfg, expansion_order=10)
        m.lib.set_band(m.obj, *band_of(r, 3, nrows))
        m.run()
        part = m.fixed_maps() if kind == "ipm" else m.magnifications.astype(np.int64)
        acc = part if acc is None else acc + part
    if kind == "ipm":
        np.testing.assert_array_equal(acc, full.fixed_maps())
    else:
        np.testing.assert_array_equal(acc, full.magnifications)


def _sharded_worker(rank, world, port, kind, out):
    import torch.distributed as dist

    import irs_b200
    from irs_b200.sharded import sharded_run
    from tests.cases import IPM_SMALL, IRS_SMALL
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    cls, cfg = (irs_b200.IPM, IPM_SMALL) if kind == "ipm" else (irs_b200.IRS, IRS_SMALL)
    m = cls(**cfg, expansion_order=10)
    total, _, _ = sharded_run(m)
    if rank == 0:
        np.save(out, total)
    m.close()
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["ipm", "irs"])
def test_sharded_run_two_gloo_ranks_on_one_gpu(gpu, tmp_path, kind):
    """The product's sharded_run with two ranks (processes) sharing cuda:0,
    each shooting its band, reduced over gloo: the same map as one object."""
    import irs_b200
    from tests.cases import IPM_SMALL, IRS_SMALL
    out = str(tmp_path / "map.npy")
    mp.spawn(_sharded_worker, args=(2, _free_port(), kind, out), nprocs=2, join=True)
    cls, cfg = (irs_b200.IPM, IPM_SMALL) if kind == "ipm" else (irs_b200.IRS, IRS_SMALL)
    full = cls(**cfg, expansion_order=10)
    full.run()
    np.testing.assert_array_equal(np.load(out), full.magnifications)
    full.close()

"""Multi-process (world size 2, gloo, CPU) tests of the sharding logic: the
ranks split a day's samples, each computes its piece of the TOD (with the C
oracle standing in for the GPU kernel, which does not exist on this host),
and the gathered TOD equals the single-process result exactly.  Detector and
day splits agree on every rank and cover every item once."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from tod_generation_mapbased_beam_b200 import sharding as SH


def test_sample_shard_covers_exactly():
    for n in (0, 1, 7, 100, 101):
        for world in (1, 2, 3, 8):
            got = [SH.sample_shard(n, r, world) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            sizes = [b - a for a, b in got]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        SH.sample_shard(10, 2, 2)


def test_detector_shards_balance_and_cover():
    rng = np.random.default_rng(0)
    costs = rng.lognormal(0.0, 1.5, 64)
    for world in (1, 2, 3, 8):
        sh = SH.detector_shards(costs, world)
        assert sorted(i for s in sh for i in s) == list(range(64))
        loads = [costs[s].sum() for s in sh]
        # LPT: the heaviest rank carries at most the mean plus the largest item
        assert max(loads) <= costs.sum() / world + costs.max() + 1e-9


def test_day_shard_round_robin():
    assert SH.day_shard(0, 10, 0, 3) == [0, 3, 6, 9]
    assert SH.day_shard(0, 10, 2, 3) == [2, 5, 8]
    assert sorted(d for r in range(4) for d in SH.day_shard(5, 20, r, 4)) == list(range(5, 20))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _tod_piece(start, stop):
    """(3, stop - start) TOD of samples [start, stop) of a small spin scan
    (C oracle, FP64 pointing)."""
    import oracle
    from tod_generation_mapbased_beam_b200 import workloads as W

    nside = 16
    beam = W.pole_gaussian_beam(240.0, 64, 0.99, search_fwhm=1.5)
    th, ph, ps = W.spin_scan(200, 20.0)
    th, ph, ps = th[start:stop], ph[start:stop], ps[start:stop]
    sky = W.white_sky(nside, 5)
    B = stop - start
    out = np.zeros((3, B))
    if B:
        rot, beta = oracle.rotation_vectors_f64(0.0, 0.0, ph.astype(np.float64), th.astype(np.float64))
        params = oracle.rotation_params_f64(rot, ph, th, ps.astype(np.float64) - beta)
        oracle.gather_accum_fused(beam.vec_orig.astype(np.float64), *params, nside, sky, beam.beam_vals, B,
                                  beam.S, out, 1, 2, nthreads=1, f64=True)
    return out


def _worker(rank, world, port, result_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        a, b = SH.sample_shard(200, rank, world)
        full = SH.gather_shards(torch.from_numpy(_tod_piece(a, b)), 200)
        costs = np.arange(1, 21, dtype=np.float64) ** 1.5
        mine = SH.detector_shards(costs, world)[rank]
        got = [None] * world
        dist.all_gather_object(got, mine)
        if rank == 0:
            np.savez(result_path, tod=full.numpy(), **{f"det{r}": np.array(v) for r, v in enumerate(got)})
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_equals_single_process(tmp_path):
    import oracle

    oracle.build()
    world = 2
    path = str(tmp_path / "res.npz")
    mp.start_processes(_worker, args=(world, _free_port(), path), nprocs=world, join=True, start_method="spawn")
    res = np.load(path)
    assert np.array_equal(res["tod"], _tod_piece(0, 200))
    costs = np.arange(1, 21, dtype=np.float64) ** 1.5
    ref = SH.detector_shards(costs, world)
    for r in range(world):
        assert list(res[f"det{r}"]) == ref[r]

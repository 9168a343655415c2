"""One run spread over several GPUs: photon-id shards (tmc_b200_run_device_range) whose integer
tallies add up to the whole run bit for bit, and the int64 all-reduce that adds them (two gloo
ranks on CPU; on GPUs the same call runs over NCCL)."""

from __future__ import annotations

import os

import numpy as np
import pytest

import tissuemc_b200 as tmc


@pytest.mark.parametrize("photons,world", [(1, 1), (7, 3), (1_000_000, 8), (2**31, 8), (10, 10)])
def test_shard_ranges_partition_the_photon_ids(photons, world):
    ranges = [tmc.shard_range(photons, r, world) for r in range(world)]
    assert ranges[0][0] == 0
    for (f0, c0), (f1, _) in zip(ranges, ranges[1:]):
        assert f0 + c0 == f1
    assert sum(c for _, c in ranges) == photons
    assert max(c for _, c in ranges) - min(c for _, c in ranges) <= 1


def test_range_validation_happens_before_any_device_work():
    spec = tmc.workload("slab_n14")
    opt = tmc.options(batches=10)
    bogus = 0x1000  # never dereferenced: the range is rejected first
    for first, count in [(0, 0), (spec.photons, 1), (spec.photons - 5, 6), (2**40, 1)]:
        with pytest.raises(tmc.ConfigError, match="photon range"):
            tmc.run_device_range(spec, opt, first, count, bogus)


def _allreduce_worker(rank: int, world: int, port: int, q) -> None:
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rng = np.random.default_rng(rank)
    mine = rng.integers(0, 2**64, size=1000, dtype=np.uint64, endpoint=False)
    mine[:4] = np.uint64(2**63) + np.uint64(rank)  # sums that wrap around 2^64
    t = torch.from_numpy(mine.view(np.int64).copy())
    dist.all_reduce(t)
    q.put((rank, mine, t.numpy().view(np.uint64).copy()))
    dist.barrier()
    dist.destroy_process_group()


def test_int64_allreduce_adds_unsigned_tallies_modulo_2_64():
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world = 2
    procs = [ctx.Process(target=_allreduce_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    parts = {r: mine for r, mine, _ in got}
    with np.errstate(over="ignore"):
        expect = parts[0] + parts[1]  # numpy uint64 addition wraps modulo 2^64
    for _, _, summed in got:
        np.testing.assert_array_equal(summed, expect)


def _raw_of_range(spec, opt, first, count):
    import torch

    sz = tmc.query_sizes(spec, opt)
    d = torch.empty(int(sz.device_words), dtype=torch.int64, device="cuda")
    tmc.run_device_range(spec, opt, first, count, d.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return d[:int(sz.tally_words)].cpu().numpy().view(np.uint64)


@pytest.mark.gpu
@pytest.mark.parametrize("name,photons,cuts", [("slab_n14", 200_000, [1, 77_777, 150_000]),
                                               ("skin5", 40_000, [20_000]),
                                               ("slab_n14", 50_000, [10_000, 20_000, 30_000, 40_000])])
def test_shards_add_up_to_the_whole_run_bit_for_bit(name, photons, cuts):
    import torch

    spec = tmc.workload(name)
    spec.photons = photons
    opt = tmc.options(batches=10, seed=3)
    sz = tmc.query_sizes(spec, opt)
    words = int(sz.tally_words)
    whole = torch.empty(int(sz.device_words), dtype=torch.int64, device="cuda")
    tmc.run_device(spec, opt, whole.data_ptr(), torch.cuda.current_stream().cuda_stream)
    whole = whole[:words].cpu().numpy().view(np.uint64)
    bounds = [0, *cuts, photons]
    total = np.zeros(words, np.uint64)
    with np.errstate(over="ignore"):
        for a, b in zip(bounds, bounds[1:]):
            total += _raw_of_range(spec, opt, a, b - a)
    np.testing.assert_array_equal(total, whole)
    # and the decoded shard sum is the run
    res = tmc.decode(spec, opt, total)
    assert int(res.photons.sum()) == photons
    assert int(res.anomalies.sum()) == 0

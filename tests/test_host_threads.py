"""The host side of the C ABI called from many threads at once (ctypes releases the GIL, so the
C++ runs concurrently): reading .mci files, validating runs and sizing their buffers, drawing sweep
configurations and their cost estimates, and decoding raw tallies give, in every thread, the same
results as one call alone."""

from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

import numpy as np

import tissuemc_b200 as tmc


def _work(i: int):
    spec = tmc.parse_mci(tmc.CONFIGS / "skin5.mci")[0]
    opt = tmc.options(batches=10 + i % 7, seed=i)
    sz = tmc.query_sizes(spec, opt)
    cfgs = tmc.sweep_sample(100 + i % 3, 64)
    cost = tmc.sweep_costs(cfgs)
    raw = np.arange(int(sz.tally_words), dtype=np.uint64) * np.uint64(2**32)
    res = tmc.decode(spec, opt, raw)
    return (int(sz.tally_words), bytes(cfgs), cost.tobytes(), float(res.rd.sum()), float(res.a_z.sum()))


def test_host_entry_points_agree_across_threads():
    alone = [_work(i) for i in range(21)]
    with ThreadPoolExecutor(max_workers=8) as pool:
        together = list(pool.map(_work, list(range(21)) * 4))
    assert together == alone * 4

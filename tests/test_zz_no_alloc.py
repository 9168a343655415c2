"""The allocation-free entry point, tmc_b200_run_static.

It serves callers that cannot call cudaMalloc — a host program running while a stream is being
captured into a CUDA graph, or a framework that owns all device memory through its own pool — by
keeping the walk's scratch (claim counter and fixed-point tallies) in a static device array of the
library. These tests call it through the C ABI and hold it to the regular entry point,
tmc_b200_run, bit for bit (integer tallies: the tolerance is zero), on consecutive calls that
reuse the same array. This file is collected last on purpose.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import tissuemc_b200 as tmc

FIELDS = ("raw", "rd", "tt", "absorbed", "events", "anomalies", "a_z", "rd_r", "tt_r", "a_rz", "rd_ra", "tt_ra",
          "photons", "first_photon")


def _call_static(spec: tmc.RunSpec, opt: tmc.COptions) -> tmc.RunResult:
    """tmc_b200_run_static through ctypes, with every output (raw included) owned by the caller."""
    return tmc.run_static(spec, opt)


def _same(a: tmc.RunResult, b: tmc.RunResult) -> None:
    for f in FIELDS:
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
    assert a.specular == b.specular


@pytest.mark.gpu
def test_static_entry_point_matches_run_on_consecutive_calls():
    slab = tmc.workload("slab_n14")
    three = tmc.parse_mci(tmc.CONFIGS.parent.parent / "tests" / "golden" / "validation" / "v3_three_layer.mci")[0]
    cases = [
        (slab, tmc.options(photons=300_000, batches=80, seed=1)),
        (slab, tmc.options(photons=300_000, batches=80, seed=1)),  # same call again: scratch reused
        (three, tmc.options(photons=100_000, batches=10, seed=4)),  # another shape after a bigger one
        (slab, tmc.options(photons=50_000, batches=5, seed=2, fast_math=False)),
    ]
    for spec, opt in cases:
        words = int(tmc.query_sizes(spec, opt).tally_words)
        assert words <= tmc.STATIC_SCRATCH_WORDS
        got = _call_static(spec, opt)
        ref = tmc.run(spec, opt)
        _same(got, ref)
        assert int(got.events.sum()) > 0 and got.device == ref.device


def test_static_entry_point_rejects_runs_beyond_its_scratch():
    skin = tmc.workload("skin5")
    opt = tmc.options(batches=100)
    assert int(tmc.query_sizes(skin, opt).tally_words) > tmc.STATIC_SCRATCH_WORDS
    with pytest.raises(tmc.ConfigError, match="static scratch"):
        _call_static(skin, opt)


def test_static_entry_point_needs_the_raw_buffer():
    lib = tmc.lib()
    spec = tmc.workload("slab_n14").to_c()
    opt = tmc.options(photons=1000, batches=2)
    res = tmc.CResult()  # all NULL, raw included
    st = tmc.CStatus()
    rc = lib.tmc_b200_run_static(ctypes.byref(spec), ctypes.byref(opt), ctypes.byref(res), ctypes.byref(st))
    assert rc == tmc.BAD_ARGUMENT and b"raw" in st.message

"""The allocation-free entry point, tmc_b200_run_static.

It serves callers that cannot call cudaMalloc — a framework that owns all device memory through
its own pool, or a plugin host that gives each plugin a fixed memory budget — by keeping the walk's
scratch (claim counter and fixed-point tallies) in a static device array of the library. These tests call it through the C ABI and hold it to the regular entry point,
tmc_b200_run, bit for bit (integer tallies: the tolerance is zero), on consecutive calls that
reuse the same array. This file is collected last on purpose.
"""

from __future__ import annotations

import ctypes
import json
import subprocess
import sys
import textwrap
from pathlib import Path

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


# Run in a fresh process, so that nothing else has set the device up: the allocation-free entry
# point is called first and alone, and the device's free memory must not move across later calls.
_FRESH = textwrap.dedent("""
    import json, sys
    sys.path.insert(0, sys.argv[1])
    import numpy as np
    import torch
    import tissuemc_b200 as tmc

    slab = tmc.workload("slab_n14")
    opt = tmc.options(photons=200_000, batches=20, seed=3)
    first = tmc.run_static(slab, opt)                   # sets the device up
    free_after_first = torch.cuda.mem_get_info(0)[0]
    second = tmc.run_static(slab, opt)
    third = tmc.run_static(slab, opt)
    free_after_third = torch.cuda.mem_get_info(0)[0]
    ref = tmc.run(slab, opt)                            # the regular entry point, which allocates
    same = all(np.array_equal(getattr(a, f), getattr(ref, f))
               for a in (first, second, third) for f in ("raw", "rd", "tt", "absorbed", "events", "a_rz"))
    print(json.dumps({"free_after_first": free_after_first, "free_after_third": free_after_third,
                      "same": same, "device": torch.cuda.current_device()}))
""")


@pytest.mark.gpu
def test_static_entry_point_allocates_nothing_in_a_fresh_process():
    root = Path(__file__).resolve().parents[1]
    p = subprocess.run([sys.executable, "-c", _FRESH, str(root)], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    out = json.loads(p.stdout.strip().splitlines()[-1])
    assert out["same"]
    assert out["free_after_first"] == out["free_after_third"], out
    assert out["device"] == 0

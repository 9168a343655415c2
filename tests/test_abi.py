"""The C ABI without a GPU: the library loads, exports every declared entry point, validates runs
with the reference's messages, reads .mci files with line-numbered errors, sizes and decodes the
tally buffer, and plans shared-memory tiles (CPU only; no compute call reaches a device)."""

from __future__ import annotations

import ctypes
import math
import re
from pathlib import Path

import numpy as np
import pytest

import tissuemc_b200 as tmc
from conftest import ROOT, has_gpu

HEADER = ROOT / "include" / "tissuemc_b200.h"
THREE_LAYER = ROOT / "tests" / "golden" / "validation" / "v3_three_layer.mci"


def declared_functions() -> list[str]:
    return sorted(set(re.findall(r"\b(tmc_b200_\w+)\s*\(", HEADER.read_text())))


def test_library_exports_every_declared_entry_point():
    lib = tmc.lib()
    names = declared_functions()
    assert len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(tmc.PROTOTYPES), "Python prototypes and header disagree"


def test_only_the_c_abi_is_exported():
    import subprocess

    out = subprocess.run(["nm", "-D", "--defined-only", str(tmc.LIB_PATH)], capture_output=True, text=True).stdout
    text_syms = [ln.split()[-1] for ln in out.splitlines() if " T " in ln]
    assert text_syms and all(s.startswith("tmc_b200_") for s in text_syms), text_syms


def test_struct_sizes_match_the_header_layout():
    # two 8-byte-aligned doubles after int32 fields: check the ctypes mirror against the C layout
    assert ctypes.sizeof(tmc.Layer) == 40
    assert ctypes.sizeof(tmc.CRunSpec) == 8 + 16 + 12 + 4 + 16 + 8 + 16 * 40
    assert ctypes.sizeof(tmc.CStatus) == 516
    assert ctypes.sizeof(tmc.CAdamTensor) == 7 * 8 + 4 * 4  # seven pointers, rows, cols, decay, first block


def test_version_and_defaults():
    lib = tmc.lib()
    assert lib.tmc_b200_abi_version() == 2
    assert b"sm_100a" in lib.tmc_b200_version()
    o = tmc.COptions()
    lib.tmc_b200_default_options(ctypes.byref(o))
    assert (o.seed, o.batches, o.photons, o.rung, o.profiles, o.fast_math) == (1, 10, 0, 0, 1, 1)


def _spec(**kw):
    base = dict(layers=[(1.37, 1, 100, 0.9, 0.1)], photons=1000)
    base.update(kw)
    return tmc.RunSpec(**base)


@pytest.mark.parametrize("kw,opt,message", [
    ({"photons": 0}, {}, "number of photons must be > 0"),
    ({"dz": 0.0}, {}, "dz and dr must be > 0"),
    ({"nr": 0}, {}, "grid bin counts must be >= 1"),
    ({"n_above": 0.9}, {}, "ambient refractive indices must be >= 1"),
    ({"layers": []}, {}, "at least one layer is required"),
    ({"layers": [(1.4, 1, 1, 0, 1)] * 17}, {}, "at most 16 layers are supported"),
    ({"layers": [(0.9, 1, 1, 0, 1)]}, {}, "layer 1: n must be >= 1"),
    ({"layers": [(1.4, -1, 1, 0, 1)]}, {}, "layer 1: mua and mus must be >= 0"),
    ({"layers": [(1.4, 0, 0, 0, 1)]}, {}, "layer 1: clear layers (mua = mus = 0) are not supported"),
    ({"layers": [(1.4, 1, 1, 1.0, 1)]}, {}, "layer 1: g must be in (-1, 1)"),
    ({"layers": [(1.4, 1, 1, 0, 0.0)]}, {}, "layer 1: thickness must be finite and > 0"),
    ({"layers": [(1.4, 1, 1, 0, math.inf)]}, {}, "layer 1: thickness must be finite and > 0"),
    ({}, {"batches": 0}, "batches must be >= 1"),
    ({}, {"batches": 1001}, "batches cannot exceed the number of photons"),
    ({}, {"rung": 2}, "rung must be 0, 1, 3, 5, 6, 7 or 8 (rungs 2 and 4 are not built yet)"),
    ({}, {"profiles": False}, "--no-profiles is a diagnostic for rung 6 only"),
    ({}, {"photons": 2**31 + 1}, "photons per run"),
    ({"nr": 100000, "nz": 100000}, {}, "tally grid is too large"),
])
def test_validation_messages_follow_the_reference(kw, opt, message):
    # texts of include/tissuemc/config.hpp:38-66 and src/cuda/engine.cu:328-350
    with pytest.raises(tmc.ConfigError) as e:
        tmc.query_sizes(_spec(**kw), tmc.options(**opt))
    assert message in str(e.value)


def test_query_sizes():
    s = _spec(nz=7, nr=5, na=3, layers=[(1.4, 1, 10, 0.5, 0.1)] * 2)
    sz = tmc.query_sizes(s, tmc.options(batches=4))
    assert (sz.batches, sz.layers, sz.nz, sz.nr, sz.na) == (4, 2, 7, 5, 3)
    assert (sz.absorbed, sz.a_rz, sz.ra) == (8, 35, 15)
    assert sz.tally_words == 4 * (4 + 2) + 35 + 2 * 15
    assert sz.device_words == sz.tally_words + 1  # the tallies, then the launch's claim counter


def test_decode_is_exact_integer_arithmetic():
    s = _spec(nz=3, nr=2, na=2, layers=[(1.4, 1, 10, 0.5, 0.1)] * 2, photons=10)
    o = tmc.options(batches=3)
    words = int(tmc.query_sizes(s, o).tally_words)
    raw = np.zeros(words, dtype=np.uint64)
    S = 6
    for b in range(3):
        raw[b * S:(b + 1) * S] = [(b + 1) << 32, 3 << 31, 100 + b, b, 1 << 30, 1 << 29]
    arz = np.arange(1, 7, dtype=np.uint64) << np.uint64(32)  # (nr=2, nz=3)
    raw[18:24] = arz
    raw[24:28] = [1 << 32, 2 << 32, 3 << 32, 4 << 32]
    raw[28:32] = [5 << 32, 0, 0, 7 << 32]
    r = tmc.decode(s, o, raw)
    assert r.photons.tolist() == [4, 3, 3] and r.first_photon.tolist() == [0, 4, 7]
    assert r.rd.tolist() == [1.0, 2.0, 3.0] and r.tt.tolist() == [1.5, 1.5, 1.5]
    assert r.events.tolist() == [100, 101, 102] and r.anomalies.tolist() == [0, 1, 2]
    assert r.absorbed.tolist() == [[0.25, 0.125]] * 3
    assert r.a_rz.tolist() == [[1, 2, 3], [4, 5, 6]]
    assert r.a_z.tolist() == [5, 7, 9]
    assert r.rd_r.tolist() == [3, 7] and r.tt_r.tolist() == [5, 7]
    assert r.specular == pytest.approx(((1 - 1.4) / (1 + 1.4)) ** 2, rel=1e-15)
    assert np.array_equal(r.raw, raw)


def test_plan_fits_whole_grids_and_tiles_big_ones():
    slab = tmc.workload("slab_n14")
    p = tmc.plan(slab, tmc.options(batches=80))
    assert (p.tr_a, p.tz_a, p.tr_rd, p.tr_tt, p.cross, p.batch_smem) == (50, 20, 50, 50, 0, 1)
    assert p.smem_bytes <= 232448 and p.grid == 148 * 4
    skin = tmc.workload("skin5")
    p = tmc.plan(skin, tmc.options(batches=100))
    assert p.cross == 1 and 0 < p.tr_a < 500 and 0 < p.tz_a < 400
    assert p.smem_bytes <= (233472 // 4) - 1024
    # a tiny shared-memory budget sends everything to global memory but stays valid
    p = tmc.plan(skin, tmc.options(batches=100, smem_budget=4096))
    ring = 64 * p.threads  # every lane's random-word ring (16 words) stays in shared memory
    assert p.smem_bytes <= max(4096, ring + 5 * 96) + 16 and p.cross == 0 and p.tr_a == 0


def test_plan_follows_the_tile_options():
    """The tile options the autotuner searches: the core tile's depth, the shared rows of R_d(r,a) and
    T_t(r,a), and the cross; every combination stays within the per-block budget."""
    skin = tmc.workload("skin5")
    base = tmc.plan(skin, tmc.options(batches=100))
    p = tmc.plan(skin, tmc.options(batches=100, tile_tz=40))
    assert p.tz_a == 40 and p.tr_a > base.tr_a and p.cross == 1
    p = tmc.plan(skin, tmc.options(batches=100, tile_tz=4000))  # clamped: the cross holds the last column
    assert p.tz_a == 399
    p = tmc.plan(skin, tmc.options(batches=100, tile_ra_rows=-1))
    assert p.tr_rd == p.tr_tt == 0 and p.tr_a * p.tz_a > base.tr_a * base.tz_a
    p = tmc.plan(skin, tmc.options(batches=100, tile_ra_rows=10))
    assert p.tr_rd == p.tr_tt == 10
    p = tmc.plan(skin, tmc.options(batches=100, tile_cross=-1))
    assert p.cross == 0 and p.tr_a * p.tz_a > base.tr_a * base.tz_a
    for tz in (-1, 0, 1, 17, 400):
        for rows in (-1, 0, 3, 500):
            for cross in (-1, 0, 1):
                for bps in (1, 2, 3, 4):
                    q = tmc.plan(skin, tmc.options(batches=100, tile_tz=tz, tile_ra_rows=rows, tile_cross=cross),
                                 regs_blocks_per_sm=bps)
                    assert q.smem_bytes <= min(232448, 233472 // bps - 1024)
                    assert 0 <= q.tr_a <= 500 and 0 <= q.tz_a <= 400 and 0 <= q.tr_rd <= 500
    p = tmc.plan(skin, tmc.options(batches=100, tile_tz=-1))
    assert p.tr_a == p.tz_a == 0 and p.cross == 1
    for bad, msg in (({"tile_tz": -2}, "tile_tz"), ({"tile_ra_rows": -2}, "tile_ra_rows"),
                     ({"tile_cross": 2}, "tile_cross")):
        with pytest.raises(tmc.ConfigError, match=msg):
            tmc.plan(skin, tmc.options(batches=100, **bad))


def test_plan_keeps_the_batch_totals_and_the_cross_before_rows():
    """The batch totals and the cross (the clamped last row and column of A(r,z)) are the words every
    running photon shares; the planner places them before the rows of R_d(r,a) and T_t(r,a), so a
    smaller budget per block (smaller blocks, more of them) or a request for many rows costs rows,
    not the shared words."""
    skin = tmc.workload("skin5")
    for threads, bps in ((256, 4), (224, 5), (192, 6), (128, 9)):
        o = tmc.options(batches=100, tile_tz=-1)
        o.threads_per_block = threads
        p = tmc.plan(skin, o, regs_blocks_per_sm=bps)
        assert p.batch_smem == 1 and p.cross == 1, (threads, bps)
        assert p.smem_bytes <= min(232448, 233472 // bps - 1024)
    p = tmc.plan(skin, tmc.options(batches=100, tile_tz=-1, tile_ra_rows=500))
    assert p.cross == 1 and 17 < p.tr_rd < 500


def test_plan_smem_per_block_never_exceeds_the_device():
    rng = np.random.default_rng(0)
    for _ in range(200):
        nl = int(rng.integers(1, 17))
        s = _spec(nz=int(rng.integers(1, 2000)), nr=int(rng.integers(1, 2000)), na=int(rng.integers(1, 90)),
                  layers=[(1.4, 1, 10, 0.5, 0.1)] * nl, photons=10**6)
        bps = int(rng.integers(1, 9))
        p = tmc.plan(s, tmc.options(batches=int(rng.integers(1, 500))), regs_blocks_per_sm=bps)
        assert p.smem_bytes <= min(232448, 233472 // bps - 1024)
        assert 0 <= p.tr_a <= s.nr and 0 <= p.tz_a <= s.nz and 0 <= p.tr_rd <= s.nr


def test_parse_bundled_and_validation_inputs():
    s = tmc.parse_mci(THREE_LAYER)[0]
    assert s.photons == 1_000_000 and (s.nz, s.nr, s.na) == (40, 50, 1)
    assert s.layers[0] == (1.37, 1.0, 100.0, 0.9, 0.1) and s.layers[2] == (1.37, 2.0, 10.0, 0.7, 0.2)
    skin = tmc.workload("skin5")
    assert skin.photons == 10**8 and len(skin.layers) == 5 and (skin.nz, skin.nr, skin.na) == (400, 500, 30)
    for p in (ROOT / "tests" / "golden" / "validation").glob("*.mci"):
        assert len(tmc.parse_mci(p)) == 1


def _parse_error(tmp_path: Path, text: str) -> str:
    f = tmp_path / "x.mci"
    f.write_text(text)
    with pytest.raises(tmc.ConfigError) as e:
        tmc.parse_mci(f)
    return str(e.value)


@pytest.mark.parametrize("old,new,where", [
    ("1.0                 # file version", "2.0", "line 1"),
    ("v3_three_layer.mco A", "v3.mco B", "line 5"),
    ("1000000             # number of photons", "1000000.5", "line 6"),
    ("1.37 1 10 0 0.1     # layer 2", "1.37 1 10 0", "line 12"),
    ("1.37 1 100 0.9 0.1  # layer 1: n mua[1/cm] mus[1/cm] g d[cm]", "1.37 1 100 abc 0.1", "line 11"),
])
def test_parse_errors_name_the_line(tmp_path, old, new, where):
    text = THREE_LAYER.read_text()
    assert old in text
    msg = _parse_error(tmp_path, text.replace(old, new, 1))
    assert where in msg and "x.mci" in msg


@pytest.mark.parametrize("old,new", [
    ("1.37 1 100 0.9 0.1", "1.37 1 100 1.0 0.1"),  # g = 1
    ("1.37 1 100 0.9 0.1", "1.37 -1 100 0.9 0.1"),  # mua < 0
    ("1.37 1 100 0.9 0.1", "1.37 0 0 0 0.1"),  # clear layer
    ("1000000             # number of photons", "0"),
    ("3                   # number of layers", "17"),
    ("40 50 1", "40 50 0"),
])
def test_parse_rejects_invalid_runs(tmp_path, old, new):
    text = THREE_LAYER.read_text()
    assert old in text
    _parse_error(tmp_path, text.replace(old, new, 1))


def test_parse_rejects_truncated_and_overlong_files(tmp_path):
    assert "unexpected end of file" in _parse_error(tmp_path, "")
    assert "unexpected end of file" in _parse_error(tmp_path, "1.0\n1\ncomp.mco A\n")
    assert "unexpected extra content" in _parse_error(tmp_path, THREE_LAYER.read_text() + "extra\n")
    with pytest.raises(tmc.ConfigError, match="cannot open"):
        tmc.parse_mci(tmp_path / "definitely_missing.mci")


def test_null_arguments_are_rejected():
    lib = tmc.lib()
    st = tmc.CStatus()
    assert lib.tmc_b200_run(None, None, None, ctypes.byref(st)) == tmc.BAD_ARGUMENT
    assert lib.tmc_b200_query_sizes(None, None, None, ctypes.byref(st)) == tmc.BAD_ARGUMENT
    n = ctypes.c_int32()
    assert lib.tmc_b200_parse_mci(None, None, 0, ctypes.byref(n), ctypes.byref(st)) == tmc.BAD_ARGUMENT


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_run_without_a_device_fails_loudly():
    with pytest.raises(tmc.EngineError) as e:
        tmc.run(_spec(), batches=2)
    assert e.value.code == tmc.NO_DEVICE and "no usable CUDA device found" in str(e.value)
    assert not tmc.available()


def test_physics_probe_rejects_bad_arguments_before_touching_a_device():
    for kw in ({"what": "hg", "g": 1.0}, {"what": "step", "g": 0.5, "mu_t": 0.0}, {"what": "hg", "g": 0.5, "samples": 0}):
        with pytest.raises(tmc.ConfigError, match="probe"):
            tmc.probe_physics(**kw)

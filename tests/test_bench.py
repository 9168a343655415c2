"""bench.py on the CPU: the reference arm's JSON line (it times the reference's own CPU engine),
the clock-sample parser that flags throttled runs, and the roofline peaks (measured or
fallback)."""

from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

import oracle

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref/tissuemc not built")
def test_reference_arm_prints_one_json_line():
    p = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload", "slab_n14",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert p.returncode == 0, p.stderr
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "photons/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["steps"] == 1
    assert d["e2e"] == {"value": d["value"], "unit": "photons/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and "slab_n14" in cb["sample"]


def test_clock_summary_reads_throttle_reasons():
    sys.path.insert(0, str(ROOT))
    import bench

    c = bench.Clocks(0)
    c.lines = ["0, 1965, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Not Active",
               "0, 1320, 1965, 998.7, 0x4, Not Active, Not Active, Not Active, Active",
               "0, 1800, 1965, 900.0, 0x0, Not Active, Not Active, Not Active, Not Active",
               "garbage line"]
    s = c.summary()
    assert s["samples"] == 3 and s["sm_mhz"] == 1800.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    c.lines = ["0, 900, 1965, 400.0, 0x8, Active, Not Active, Active, Not Active"]
    assert c.summary()["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]


def test_roofline_peaks_say_whether_they_were_measured(tmp_path, monkeypatch):
    sys.path.insert(0, str(ROOT))
    import bench

    monkeypatch.setattr(bench, "ROOT", tmp_path)
    value, note = bench._peak("bf16_tflops", 1590.0)
    assert value == 1590.0 and "fallback" in note
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"gemm": {"bf16_tflops": 1651.9}, "hbm_gbs": 6650}))
    value, note = bench._peak("bf16_tflops", 1590.0)
    assert value == 1651.9 and "measured" in note
    assert bench._peak("hbm_gbs", 1.0) == (6650.0, "hbm_gbs of MEASURED_PEAKS.json (measured)")
    assert bench._peak("sm_max_mhz", 1965.0)[1].startswith("fallback")


def test_issue_roofline_of_the_walk_and_the_sweep():
    """The FP32/SFU issue roofline with the frozen per-step operation counts: skin5 (604.20
    interaction + 14.30 boundary steps per photon) and the sweep workload (141.1 + 3.8) on 148 SMs
    at 1965 MHz are SFU-bound at 6.38e8 and 2.73e9 photons/s."""
    sys.path.insert(0, str(ROOT))
    import bench

    peak, bound, f_tot, s_tot = bench.issue_roofline(bench.STEPS_PER_PHOTON["skin5"], 148, 1965.0)
    assert bound == "sfu" and abs(peak / 6.38e8 - 1) < 5e-3
    assert abs(f_tot - (604.20 * 61 + 14.30 * 25)) < 1e-9 and abs(s_tot - (604.20 * 12 + 14.30 * 3)) < 1e-9
    peak, bound, _, _ = bench.issue_roofline(bench.SWEEP_STEPS_PER_PHOTON, 148, 1965.0)
    assert bound == "sfu" and abs(peak / 2.73e9 - 1) < 5e-3

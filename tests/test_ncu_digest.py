"""The Nsight Compute digest tool (tissuemc_b200/bin/ncu_digest, host C++): kernel selection,
grouping, averaging and side-by-side comparison on a fixture cut from real captures
(tests/golden/make_ncu_sample.py)."""

from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

from tissuemc_b200 import build as b

SAMPLE = Path(__file__).parent / "golden" / "ncu_sample.csv"


def _digest(*args: str) -> subprocess.CompletedProcess:
    return subprocess.run([str(b.DIGEST), *args], capture_output=True, text=True, timeout=60)


def test_digest_groups_one_kernel():
    p = _digest(str(SAMPLE), "--kernel", "walk_kernel")
    assert p.returncode == 0, p.stderr
    out = p.stdout
    assert "1 launch(es) of void walk_kernel<1>(WalkParams)" in out
    for title in ("Launch and occupancy", "Issue and active lanes", "Pipe utilisation", "Warp stalls",
                  "Local memory", "L2 and DRAM"):
        assert f"### {title}" in out, title
    row = next(line for line in out.splitlines() if line.startswith("| smsp__thread_inst_executed_per_inst_executed"))
    assert row.split("|")[3].strip() == "20.000"
    assert "| launch__registers_per_thread | register/thread | 62.000 |" in out


def test_all_launches_are_averaged_and_two_captures_sit_side_by_side(tmp_path):
    p = _digest(str(SAMPLE))
    assert p.returncode == 0 and "2 launch(es)" in p.stdout
    # the same file twice, restricted to different kernels: columns A and B
    a = tmp_path / "a.csv"
    a.write_text(SAMPLE.read_text())
    p = _digest(str(SAMPLE), str(a), "--kernel", "ensemble_infer")
    assert p.returncode == 0
    row = next(line for line in p.stdout.splitlines() if line.startswith("| launch__block_size"))
    assert [c.strip() for c in row.split("|")[3:5]] == ["576.0", "576.0"]


def test_errors():
    assert _digest().returncode == 2
    assert _digest(str(SAMPLE), "--kernel", "no_such_kernel").returncode == 1
    assert _digest("/nonexistent.csv").returncode == 2
    assert _digest(str(SAMPLE), "--kernel", "(").returncode == 2


@pytest.mark.parametrize("text", ["", "==PROF== nothing here\n"])
def test_rejects_files_without_a_header(tmp_path, text):
    f = tmp_path / "x.csv"
    f.write_text(text)
    assert _digest(str(f)).returncode == 2

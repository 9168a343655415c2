"""The persistent kernels' work distribution (tissuemc_b200/csrc/work_queue.cuh) emulated on the CPU
with warps and lanes in random interleavings: every photon launched exactly once, batch sizes as
TissueMC's BatchPlan gives them, and the sweep's item queue covering every photon of every
configuration once (tests/emulation/work_queue.cpp). The same header is compiled into both kernels."""

from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_work_distribution_in_emulated_warps(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    exe = tmp_path / "work_queue"
    subprocess.run([cxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", str(ROOT / "tests/emulation/work_queue.cpp"),
                    "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    assert "all properties hold" in out.stdout

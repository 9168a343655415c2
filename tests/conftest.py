"""Test configuration: the `gpu` marker, import paths, and an in-tree build of the engine and the
oracles when they are missing (nothing here falls back to a CPU path: GPU tests need the CUDA
library and a device)."""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on a B200)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    from tissuemc_b200 import build as b

    if not b.LIB.exists() or not b.CLI.exists() or not b.DIGEST.exists():
        b.build()
    if not (ROOT / "oracle" / "liboracle.so").exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), str(ROOT / "oracle" / "liboracle.so")],
                       check=True)
    yield


@pytest.fixture(scope="session")
def golden():
    import json

    g = ROOT / "tests" / "golden"
    return {
        "kat": json.loads((g / "philox_kat.json").read_text()),
        "refs": json.loads((g / "references.json").read_text()),
        "hf": json.loads((g / "h_function.json").read_text()),
        "runs": json.loads((g / "ref_runs.json").read_text()),
        "dir": g,
    }


def has_gpu() -> bool:
    try:
        import tissuemc_b200 as t

        return t.available()
    except Exception:
        return False

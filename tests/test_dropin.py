"""The drop-in as a TissueMC maintainer would build it: the reference's own `tissuemc` command line
and CPU engine (src/cli/main.cpp, src/cpu/engine.cpp, src/io/mci.cpp, src/io/json_out.cpp) with
tissuemc_b200/csrc/host/run_cuda.cpp compiled against the reference's headers in place of
src/cuda/engine.cu (the boundary include/tissuemc/cuda_engine.hpp:9-14, called from
src/cli/main.cpp:142-147), linked to libtissuemc_b200.so. oracle/Makefile's `dropin` target builds it
into oracle/_ref/tissuemc_dropin from the TissueMC sources (TISSUEMC_REF, or a `reference` directory
beside this repository); where the sources are absent the prebuilt binary is used."""

from __future__ import annotations

import json
import os
import subprocess
from pathlib import Path

import pytest

import oracle
import tissuemc_b200 as tmc
from conftest import has_gpu
from gates import from_oracle, from_reference_json, identical_photon_gaps

ROOT = Path(__file__).resolve().parents[1]
DROPIN = ROOT / "oracle" / "_ref" / "tissuemc_dropin"
REF = Path(os.environ.get("TISSUEMC_REF", ROOT.parent / "reference"))
V3 = ROOT / "tests" / "golden" / "validation" / "v3_three_layer.mci"


def _binary() -> Path:
    if not DROPIN.exists():
        pytest.skip("the drop-in build needs the TissueMC sources (TISSUEMC_REF) and was not built here")
    return DROPIN


@pytest.mark.skipif(not (REF / "src" / "cli" / "main.cpp").exists(), reason="TissueMC sources not present")
def test_the_reference_cli_compiles_and_links_against_the_engine():
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "dropin", f"REF={REF}"], check=True)
    nm = subprocess.run(["nm", "-C", "--undefined-only", str(DROPIN)], capture_output=True, text=True, check=True)
    assert "tmc_b200_run" in nm.stdout  # run_cuda resolves to this engine's C ABI


def test_version_is_the_reference_cli():
    p = subprocess.run([str(_binary()), "--version"], capture_output=True, text=True)
    assert p.returncode == 0 and p.stdout.strip() == "tissuemc 0.1.0"


def test_its_cpu_engine_is_untouched():
    p = subprocess.run([str(_binary()), "run", str(V3), "--photons", "2000", "--batches", "2", "--engine", "cpu"],
                       capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    assert "(cpu, float64)" in p.stdout


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_no_device_is_the_reference_error():
    p = subprocess.run([str(_binary()), "run", str(V3), "--engine", "cuda"], capture_output=True, text=True)
    assert p.returncode == 1
    assert "no usable CUDA device found" in p.stderr


@pytest.mark.gpu
def test_dropin_gpu_run_meets_the_identical_photon_gates(tmp_path):
    """--engine cuda on the three-layer validation input: the reference's JSON, read as its own
    readers read it, meets the reference's identical-photon limits against the float32 CPU path."""
    out = tmp_path / "r.json"
    p = subprocess.run([str(_binary()), "run", str(V3), "--engine", "cuda", "--photons", "300000", "--batches", "20",
                        "--seed", "5", "--output", str(out)], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    run = json.loads(out.read_text())["runs"][0]
    assert run["engine"] == "cuda" and run["precision"] == "float32" and run["anomalies"] == 0
    spec = tmc.parse_mci(V3)[0]
    o = oracle.run(oracle.Spec(layers=list(spec.layers), dz=spec.dz, dr=spec.dr, nz=spec.nz, nr=spec.nr, na=spec.na,
                               n_above=spec.n_above, n_below=spec.n_below), 300_000, 20, 5, 32, threads=0)
    gaps = identical_photon_gaps(from_oracle(o), from_reference_json(run), profiles=("a_z", "rd_r"))
    bad = [str(g) for g in gaps if not g.passed]
    assert not bad, "\n".join(bad)

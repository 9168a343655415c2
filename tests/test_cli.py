"""The `tissuemc` command line: options, exit codes and messages of the reference's
src/cli/main.cpp:18-204 (exit 2 on usage errors, 1 on run errors or anomalies)."""

from __future__ import annotations

import json
import subprocess

import pytest

import tissuemc_b200 as tmc
from conftest import has_gpu

CLI = str(tmc.CLI_PATH)
SLAB = str(tmc.CONFIGS / "slab_n14.mci")


def run(*args):
    return subprocess.run([CLI, *args], capture_output=True, text=True)


def test_version():
    p = run("--version")
    assert p.returncode == 0 and p.stdout.startswith("tissuemc ")


@pytest.mark.parametrize("args,needle", [
    ((), "usage"),
    (("run",), "usage"),
    (("run", SLAB, "--bogus"), "unknown option '--bogus'"),
    (("run", SLAB, "--precision", "float16"), "--precision must be float64 or float32"),
    (("run", SLAB, "--gpu-tally", "int8"), "--gpu-tally must be float64 or float32"),
    (("run", SLAB, "--engine", "cpu"), "B200 engine only"),
    (("run", SLAB, "--engine", "tpu"), "--engine must be cuda or b200"),
    (("run", SLAB, "--photons", "-5"), "expects a non-negative integer"),
    (("run", SLAB, "--batches"), "needs a value"),
    (("run", SLAB, "--step-cap", "0"), "--step-cap must be between 1 and 4294967295"),
])
def test_usage_errors_exit_2(args, needle):
    p = run(*args)
    assert p.returncode == 2
    assert needle in p.stderr


def test_bad_input_file_exits_1_with_line(tmp_path):
    f = tmp_path / "bad.mci"
    f.write_text("1.0\n1\nx.mco A\n100\n0.1 0.1\n1 1 1\n1\n1.0\n1.4 1 1 2.0 1\n1.0\n")
    p = run("run", str(f))
    assert p.returncode == 1
    assert "line 10: invalid run: layer 1: g must be in (-1, 1)" in p.stderr
    p = run("run", str(tmp_path / "missing.mci"))
    assert p.returncode == 1 and "cannot open" in p.stderr


def test_invalid_options_exit_1_with_config_message():
    p = run("run", SLAB, "--photons", "5", "--batches", "6")
    assert p.returncode == 1 and "batches cannot exceed the number of photons" in p.stderr


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_no_device_exits_1():
    p = run("run", SLAB)
    assert p.returncode == 1 and "no usable CUDA device found" in p.stderr


@pytest.mark.gpu
def test_run_writes_reference_json_layout(tmp_path):
    out = tmp_path / "r.json"
    p = run("run", SLAB, "--photons", "100000", "--batches", "10", "--seed", "3", "--output", str(out))
    assert p.returncode == 0, p.stderr
    assert "diffuse  R_d  =" in p.stdout and "conservation residual" in p.stdout
    doc = json.loads(out.read_text())
    r = doc["runs"][0]
    ref_keys = ["tissuemc_version", "engine", "precision", "seed", "threads", "photons", "output_name",
                "n_above", "n_below", "layers", "grid", "specular", "wall_seconds", "kernel_seconds",
                "device", "tally_precision", "rung", "profiles", "events", "anomalies", "summary",
                "batches", "a_z", "rd_r"]
    assert list(r)[:len(ref_keys)] == ref_keys
    assert r["engine"] == "cuda" and r["precision"] == "float32" and r["photons"] == 100000
    assert len(r["a_rz"]) == 50 and len(r["a_rz"][0]) == 20 and len(r["rd_ra"][0]) == 30
    assert abs(sum(r["a_z"]) - sum(sum(b["absorbed"]) for b in r["batches"])) < 1e-9 * sum(r["a_z"])


@pytest.mark.gpu
def test_anomalies_make_the_run_exit_1(tmp_path):
    """A step cap far below a packet's length ends every packet as an anomaly; the command line
    then exits 1 with the reference's warning (src/cli/main.cpp:162-168) and records them."""
    out = tmp_path / "r.json"
    p = run("run", SLAB, "--photons", "20000", "--batches", "4", "--step-cap", "3", "--output", str(out))
    assert p.returncode == 1, p.stderr
    assert "anomalies (non-finite weight or non-unit direction)" in p.stderr
    r = json.loads(out.read_text())["runs"][0]
    assert r["anomalies"] > 0 and sum(b["anomalies"] for b in r["batches"]) == r["anomalies"]
    p = run("run", SLAB, "--photons", "20000", "--batches", "4")
    assert p.returncode == 0, p.stderr

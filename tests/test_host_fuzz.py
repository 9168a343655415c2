"""The host programs on random input: the `tissuemc` command line on random option lists and the
ncu digest on mutated CSV captures. Each ends with its documented exit status (0, 1 on run or input
errors, 2 on usage errors) and never on a signal. The walk itself is never reached on valid options
here: every run goes to a .mci whose photons the options make invalid, or to a device-less path."""

from __future__ import annotations

import random
import subprocess
from pathlib import Path

import tissuemc_b200 as tmc
from tissuemc_b200 import build as b

SLAB = str(tmc.CONFIGS / "slab_n14.mci")
SAMPLE = Path(__file__).parent / "golden" / "ncu_sample.csv"

OPTIONS = ["--photons", "--batches", "--seed", "--threads", "--precision", "--engine", "--rung", "--gpu-tally",
           "--no-profiles", "--output", "--mco", "--bogus", "-h", "--help", "--version", "run"]
VALUES = ["0", "1", "-1", "7", "99999999999999999999", "1e3", "float32", "float64", "cuda", "b200", "cpu", "",
          "x", "--photons", "6", "8", "9", "/nonexistent/dir/out.json", "nan"]


def test_cli_exit_codes_on_random_option_lists(tmp_path):
    rng = random.Random(7)
    seen = set()
    for _ in range(300):
        args = ["run", SLAB] if rng.random() < 0.8 else []
        for _ in range(rng.randint(0, 6)):
            args.append(rng.choice(OPTIONS))
            if rng.random() < 0.8:
                args.append(rng.choice(VALUES))
        # keep every run away from the device: more batches than photons is a validation error
        args += ["--photons", "5", "--batches", "6"]
        p = subprocess.run([str(tmc.CLI_PATH), *args], capture_output=True, text=True, timeout=60, cwd=tmp_path)
        assert p.returncode in (0, 1, 2), (args, p.returncode, p.stderr[-500:])
        seen.add(p.returncode)
    assert {1, 2} <= seen


def test_digest_exit_codes_on_mutated_captures(tmp_path):
    rng = random.Random(11)
    lines = SAMPLE.read_text().splitlines()
    f = tmp_path / "m.csv"
    for _ in range(200):
        m = list(lines)
        for _ in range(rng.randint(1, 5)):
            k = rng.randrange(len(m))
            op = rng.randrange(5)
            if op == 0:
                del m[k]
            elif op == 1:
                m[k] = m[k][: rng.randrange(len(m[k]) + 1)]  # cut a record short
            elif op == 2:
                m[k] = m[k].replace(",", ",,", 1)  # shift the fields
            elif op == 3:
                m[k] = m[k].replace('"', "", rng.randint(1, 3))  # unbalanced quotes
            else:
                m.insert(k, '"' + "9" * rng.randint(1, 400) + '"')
            if not m:
                m = [""]
        f.write_text("\n".join(m) + "\n")
        for extra in ([], ["--kernel", "walk"], ["--kernel", "("]):
            p = subprocess.run([str(b.DIGEST), str(f), *extra], capture_output=True, text=True, timeout=60)
            assert p.returncode in (0, 1, 2), (extra, p.returncode, p.stderr[-500:])

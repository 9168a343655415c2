"""The C++ .mci reader on thousands of mutated inputs (deleted, duplicated, replaced and swapped
tokens, truncations, huge and non-finite numbers, long lines, stray bytes): every input either
parses into runs that pass validation (up to this engine's own limits on photons per run and tally
bins, which the reference's reader does not check) or is rejected with a ConfigError; the process
never crashes.
The mutations run in a child process, so a crash fails the test instead of the whole suite."""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

CHILD = r'''
import random, sys, tempfile
from pathlib import Path
sys.path.insert(0, sys.argv[1])
import tissuemc_b200 as tmc

seeds = [p.read_text() for p in sorted((Path(sys.argv[1]) / "tests" / "golden" / "validation").glob("*.mci"))]
seeds += [p.read_text() for p in sorted((Path(sys.argv[1]) / "tissuemc_b200" / "configs").glob("*.mci"))]
odd = ["nan", "inf", "-inf", "1e400", "-1e400", "0", "-0", "1e-400", "4294967297", "-1", "18446744073709551617",
       "0x10", "1,5", "", "#", "# c", "\x00", "\xff\xfe", "A", "B", "x" * 5000, "1" * 400, "3.", ".5", "1e", "--1"]
rng = random.Random(20261204)
accepted = rejected = 0
with tempfile.TemporaryDirectory() as d:
    f = Path(d) / "fuzz.mci"
    for i in range(int(sys.argv[2])):
        toks = rng.choice(seeds).replace("\n", " \n ").split(" ")
        for _ in range(rng.randint(1, 4)):
            k = rng.randrange(len(toks))
            op = rng.randrange(6)
            if op == 0:
                del toks[k]
            elif op == 1:
                toks.insert(k, toks[rng.randrange(len(toks))])
            elif op == 2:
                toks[k] = rng.choice(odd)
            elif op == 3:
                j = rng.randrange(len(toks)); toks[k], toks[j] = toks[j], toks[k]
            elif op == 4:
                toks = toks[:k]
            else:
                toks[k] = str(rng.uniform(-1e3, 1e3) if rng.random() < 0.5 else rng.randint(-10, 10**7))
            if not toks:
                toks = [""]
        f.write_bytes(" ".join(toks).encode("utf-8", "surrogateescape"))
        try:
            runs = tmc.parse_mci(f)
        except tmc.ConfigError:
            rejected += 1
            continue
        accepted += 1
        for r in runs:  # what the reader accepts, validation accepts, up to this engine's own limits
            try:
                tmc.query_sizes(r, tmc.options(batches=min(10, max(1, r.photons))))
            except tmc.ConfigError as e:
                assert "photons per run" in str(e) or "tally grid is too large" in str(e), str(e)
print(f"ok accepted={accepted} rejected={rejected}")
'''


def test_mci_reader_survives_mutated_inputs():
    out = subprocess.run([sys.executable, "-c", CHILD, str(ROOT), "3000"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, (out.returncode, out.stderr[-3000:])
    assert out.stdout.startswith("ok"), out.stdout
    accepted = int(out.stdout.split("accepted=")[1].split()[0])
    assert accepted > 0  # some mutations keep the file valid (comments, numbers within range)

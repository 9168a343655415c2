"""Regenerate the golden fixtures in tests/golden/ from the TissueMC reference (run in a container
that has the reference sources; the GPU box never reads them).

    python tests/golden/make_golden.py [--ref PATH]   (default: a `reference` directory beside the repo)

Writes:
  philox_kat.json     the Random123 known-answer vectors quoted in the reference's
                      tests/cpp/test_philox.cpp:24-30 (read from that file as text)
  references.json     the published validation values of configs/validation/references.json
  validation/*.mci    the reference's validation and benchmark inputs (configs/)
  h_function.json     the reference's analytic H-function oracle (python/tissuemc_analysis/
                      oracle.py:84-105) evaluated for the O1 and V2 media, by importing it
  ref_runs.json       outputs of the reference's own CPU engine (oracle/_ref/tissuemc, built from
                      the reference sources by oracle/Makefile) on small cases, float64 and
                      float32 transport: per-batch sums, events, anomalies, a_z and rd_r
"""

from __future__ import annotations

import argparse
import json
import re
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402

# (name, .mci source, photons, batches, seed)
CASES = [
    ("slab_n14", "bundled:slab_n14.mci", 20000, 10, 1),
    ("slab_n14_full", "bundled:slab_n14.mci", 1000000, 80, 1),
    ("skin5", "bundled:skin5.mci", 200000, 20, 7),
    ("v1_slab", "validation/v1_slab.mci", 20000, 10, 3),
    ("v2_semi_infinite", "validation/v2_semi_infinite.mci", 5000, 10, 4),
    ("v3_three_layer", "validation/v3_three_layer.mci", 20000, 20, 1),
    ("o1_semi_infinite_matched", "validation/o1_semi_infinite_matched.mci", 5000, 10, 5),
    ("tissue_g09", "bench/tissue_g09.mci", 500, 5, 2),
]


def kat_vectors(ref: Path) -> list[dict]:
    text = (ref / "tests/cpp/test_philox.cpp").read_text()
    out = []
    for m in re.finditer(r"check_kat\(\{\{([^}]*)\}\},\s*\{\{([^}]*)\}\},\s*\{\{([^}]*)\}\}\)", text):
        ints = [[int(v.strip().rstrip("u"), 0) for v in g.split(",")] for g in m.groups()]
        out.append({"ctr": ints[0], "key": ints[1], "out": ints[2]})
    if len(out) != 3:
        raise SystemExit(f"expected 3 known-answer vectors, found {len(out)}")
    return out


def mci_text(ref: Path, src: str) -> str:
    if src.startswith("bundled:"):
        return (ROOT / "tissuemc_b200" / "configs" / src.split(":", 1)[1]).read_text()
    return (ref / "configs" / src).read_text()


def slim(run: dict) -> dict:
    keep = ("engine", "precision", "seed", "photons", "specular", "events", "anomalies", "summary",
            "a_z", "rd_r", "grid", "layers", "n_above", "n_below")
    out = {k: run[k] for k in keep}
    out["batches"] = [{k: b[k] for k in ("first_photon", "photons", "rd", "tt", "absorbed", "events",
                                         "anomalies")} for b in run["batches"]]
    return out


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", type=Path, default=ROOT.parent / "reference")
    args = ap.parse_args()
    ref = args.ref
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), f"REF={ref}"], check=True)

    (HERE / "philox_kat.json").write_text(json.dumps(kat_vectors(ref), indent=1) + "\n")
    shutil.copyfile(ref / "configs/validation/references.json", HERE / "references.json")
    vdir = HERE / "validation"
    vdir.mkdir(exist_ok=True)
    for p in sorted((ref / "configs/validation").glob("*.mci")) + [ref / "configs/bench/tissue_g09.mci"]:
        shutil.copyfile(p, vdir / p.name)

    sys.path.insert(0, str(ref / "python"))
    from tissuemc_analysis import oracle as h_oracle  # the reference's own analytic oracle

    hf = {}
    for name, (mua, mus, n) in {"o1": (10.0, 90.0, 1.0), "v2": (10.0, 90.0, 1.5)}.items():
        r = h_oracle.semi_infinite_isotropic(mua, mus, n, 1.0)
        hf[name] = {"mua": mua, "mus": mus, "n_medium": n, "n_ambient": 1.0, "rd": r.rd, "rsp": r.rsp,
                    "total": r.total}
    (HERE / "h_function.json").write_text(json.dumps(hf, indent=1) + "\n")

    runs = {}
    for name, src, photons, batches, seed in CASES:
        text = mci_text(ref, src)
        for prec in ("float64", "float32"):
            r = oracle.run_reference(text, photons, batches, seed, prec, threads=8)
            runs[f"{name}/{prec}"] = {"mci": text, "photons": photons, "batches": batches, "seed": seed,
                                      "result": slim(r)}
    (HERE / "ref_runs.json").write_text(json.dumps(runs) + "\n")
    print("wrote", sorted(p.name for p in HERE.iterdir()))
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""Parity rules of the TissueMC reference, restated for the tests (test infrastructure).

* ``compare`` — the published-value rule of python/tissuemc_analysis/stats.py:48-64:
  |ours - ref| <= 3 * sqrt(se_ours^2 + se_ref^2) + rounding.
* ``identical_photon_gaps`` — the identical-photon limits of
  python/tissuemc_analysis/cross_engine.py:42-51, 75-121 (totals <= 0.25 SE, per batch <= 5e-3
  relative, events <= 1e-3 relative, no anomalies, profile totals <= 1e-4 relative, cumulative
  profile shape <= 1e-3 of the total), applied to a_z and rd_r as the reference applies them, and
  extended here to T_t(r) and to the flattened 2-D tallies A(r,z), R_d(r,a), T_t(r,a).
* ``bin_z_scores`` — per-bin |z| between two runs for every bin above a count floor, with each
  bin's standard error from the spread of its per-batch sums.
* ``conservation`` — validate.py:134-153: the residual of R_d + T_t + A + R_sp - 1 within 3 SE plus
  a floor (1e-6 for float32 transport).
"""

from __future__ import annotations

import itertools
import math
from dataclasses import dataclass

import numpy as np

Z_LIMIT = 3.0
MAX_TOTAL_SE = 0.25
MAX_BATCH_REL = 5e-3
MAX_EVENTS_REL = 1e-3
MAX_PROFILE_TOTAL_REL = 1e-4
MAX_PROFILE_SHAPE = 1e-3
CONSERVATION_FLOOR = {"float64": 1e-12, "float32": 1e-6}


@dataclass(frozen=True)
class Gap:
    name: str
    value: float
    limit: float

    @property
    def passed(self) -> bool:
        return self.value <= self.limit

    def __str__(self) -> str:
        return f"[{'PASS' if self.passed else 'FAIL'}] {self.name}: {self.value:.3e} (limit {self.limit:.1e})"


def batch_estimate(sums, photons) -> tuple[float, float]:
    sums = [float(s) for s in sums]
    photons = [float(p) for p in photons]
    mean = math.fsum(sums) / sum(photons)
    n = len(sums)
    if n < 2:
        return mean, math.nan
    per = [s / p for s, p in zip(sums, photons, strict=True)]
    c = math.fsum(per) / n
    ss = math.fsum((x - c) ** 2 for x in per)
    return mean, math.sqrt(ss / (n - 1) / n)


def compare(ours: float, se_ours: float, ref: float, se_ref: float = 0.0, rounding: float = 0.0):
    se = math.hypot(se_ours, se_ref)
    diff = ours - ref
    z = diff / se if se > 0 else (0.0 if diff == 0 else math.copysign(math.inf, diff))
    return z, abs(diff) <= Z_LIMIT * se + rounding


@dataclass
class Run:
    """Engine-neutral view of one run: per-batch sums plus profiles (numpy)."""

    photons: np.ndarray
    rd: np.ndarray
    tt: np.ndarray
    absorbed: np.ndarray  # per batch, all layers summed
    events: int
    anomalies: int
    specular: float
    profiles: dict  # name -> flat array


def from_engine(res) -> Run:
    prof = {"a_z": res.a_z, "rd_r": res.rd_r, "tt_r": res.tt_r, "a_rz": res.a_rz.ravel(),
            "rd_ra": res.rd_ra.ravel(), "tt_ra": res.tt_ra.ravel()}
    return Run(res.photons.astype(float), res.rd, res.tt, res.absorbed.sum(axis=1), int(res.events.sum()),
               int(res.anomalies.sum()), res.specular, prof)


def from_oracle(o) -> Run:
    prof = {"a_z": o.a_z, "rd_r": o.rd_r, "tt_r": o.tt_ra.sum(axis=1), "a_rz": o.a_rz.ravel(),
            "rd_ra": o.rd_ra.ravel(), "tt_ra": o.tt_ra.ravel()}
    return Run(o.photons.astype(float), o.rd, o.tt, o.absorbed.sum(axis=1), int(o.events.sum()),
               int(o.anomalies.sum()), o.specular, prof)


def from_reference_json(r: dict) -> Run:
    b = r["batches"]
    prof = {"a_z": np.array(r["a_z"]), "rd_r": np.array(r["rd_r"])}
    return Run(np.array([x["photons"] for x in b], float), np.array([x["rd"] for x in b]),
               np.array([x["tt"] for x in b]), np.array([math.fsum(x["absorbed"]) for x in b]),
               int(r["events"]), int(r["anomalies"]), float(r["specular"]), prof)


def _profile_gaps(name: str, pa: np.ndarray, pb: np.ndarray, total_se: float | None = None) -> list[Gap]:
    """Total and shape gaps of one profile. The reference's limit on a profile total (1e-4
    relative) is kept for the profiles it gates (a_z, rd_r) and for the 2-D arrays whose totals
    are those same sums (a_rz, rd_ra). T_t(r) and T_t(r,a) sum to T_t, which the reference gates at
    0.25 standard errors of the total: when `total_se` (the SE of the summed weight) is given, the
    total gap is gated that way instead."""
    pa, pb = list(map(float, pa)), list(map(float, pb))
    if not pa or len(pa) != len(pb):
        return []
    total = math.fsum(pa)
    if total == 0:
        return [Gap(f"{name}: both empty", float(math.fsum(pb) != 0), 0.0)]
    ca, cb = list(itertools.accumulate(pa)), list(itertools.accumulate(pb))
    shape = max(abs(x - y) for x, y in zip(ca, cb, strict=True)) / abs(total)
    gap = abs(total - math.fsum(pb))
    if total_se is not None:
        first = Gap(f"{name}: total gap / SE", gap / total_se, MAX_TOTAL_SE)
    else:
        first = Gap(f"{name}: total relative gap", gap / abs(total), MAX_PROFILE_TOTAL_REL)
    return [first, Gap(f"{name}: worst cumulative gap / total", shape, MAX_PROFILE_SHAPE)]


def identical_photon_gaps(a: Run, b: Run, profiles=("a_z", "rd_r", "tt_r", "a_rz", "rd_ra", "tt_ra")) -> list[Gap]:
    if not np.array_equal(a.photons, b.photons):
        raise ValueError("the two runs do not use the same batches")
    gaps = []
    tt_total_se = None
    for key in ("rd", "tt", "absorbed"):
        sa, sb = getattr(a, key), getattr(b, key)
        ma, sea = batch_estimate(sa, a.photons)
        mb, seb = batch_estimate(sb, b.photons)
        se = max(sea, seb)
        if key == "tt":
            tt_total_se = se * float(np.sum(a.photons))
        gaps.append(Gap(f"{key}: total gap / SE", abs(ma - mb) / se, MAX_TOTAL_SE))
        rel = [abs(x - y) / abs(x) for x, y in zip(sa, sb, strict=True) if x != 0]
        gaps.append(Gap(f"{key}: worst per-batch relative gap", max(rel) if rel else 0.0, MAX_BATCH_REL))
    gaps.append(Gap("events: relative gap", abs(a.events - b.events) / a.events, MAX_EVENTS_REL))
    gaps.append(Gap("anomalies (both runs)", float(a.anomalies + b.anomalies), 0.0))
    for name in profiles:
        if name in a.profiles and name in b.profiles:
            gaps += _profile_gaps(name, a.profiles[name], b.profiles[name],
                                  tt_total_se if name in ("tt_r", "tt_ra") else None)
    return gaps


def bin_z_scores(ours: np.ndarray, ref: np.ndarray, ref_batches: np.ndarray, counts: np.ndarray,
                 floor: int) -> tuple[np.ndarray, int]:
    """|z| per bin with >= floor contributing scores. The standard error of a bin's total is the
    standard error of its per-batch sums (ref_batches: (B, bins)) times B; ours is assumed to have
    the same variance (same photons, same physics), so the gap's SE is sqrt(2) times that."""
    b = ref_batches.shape[0]
    se_total = ref_batches.std(axis=0, ddof=1) * math.sqrt(b)
    mask = counts >= floor
    se = np.sqrt(2.0) * se_total[mask]
    z = np.abs(ours[mask] - ref[mask]) / np.where(se > 0, se, np.inf)
    return z, int(mask.sum())


def conservation(run: Run, precision: str = "float32") -> tuple[float, float, bool]:
    mean, se = batch_estimate(run.rd + run.tt + run.absorbed, run.photons)
    resid = mean + run.specular - 1.0
    _, ok = compare(resid, se, 0.0, 0.0, CONSERVATION_FLOOR[precision])
    return resid, se, ok

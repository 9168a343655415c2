"""Parity rules of the TissueMC reference, restated for the tests (test infrastructure).

* ``compare`` — the published-value rule of python/tissuemc_analysis/stats.py:48-64:
  |ours - ref| <= 3 * sqrt(se_ours^2 + se_ref^2) + rounding.
* ``identical_photon_gaps`` — the identical-photon limits of
  python/tissuemc_analysis/cross_engine.py:42-51, 75-121 (totals <= 0.25 SE, per batch <= 5e-3
  relative, events <= 1e-3 relative, no anomalies, profile totals <= 1e-4 relative, cumulative
  profile shape <= 1e-3 of the total), applied to a_z and rd_r as the reference applies them, and
  extended here to T_t(r) and to the flattened 2-D tallies A(r,z), R_d(r,a), T_t(r,a).
* ``bin_z_scores`` — per-bin |z| between two runs of the same photons for every bin above a count
  floor, with each bin's standard error from the spread of the reference run's per-batch sums.
* ``per_photon_bins`` / ``bin_z_two_runs`` — per-bin |z| between two runs of any photon counts, each
  side with its own standard error from its own per-batch sums (the reference's batch estimate,
  src/io/json_out.cpp:37-64, applied to every bin); ``family_check`` judges the |z| of many
  independent bins at once (a fixed |z| < 3 on every one of 10^4-10^5 independent bins fails by
  chance alone: 0.3 % of them exceed 3 under the null).
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
    """|z| per bin with >= floor contributing scores, for two runs of the SAME photons and batches.
    The standard error of a bin's total is the standard error of the reference run's per-batch sums
    (ref_batches: (B, bins)) times B; the other run has the same photons, hence the same variance,
    so the gap's SE is taken as sqrt(2) times that. For runs of different photons use
    bin_z_two_runs."""
    b = ref_batches.shape[0]
    se_total = ref_batches.std(axis=0, ddof=1) * math.sqrt(b)
    mask = counts >= floor
    se = np.sqrt(2.0) * se_total[mask]
    z = np.abs(ours[mask] - ref[mask]) / np.where(se > 0, se, np.inf)
    return z, int(mask.sum())


def per_photon_bins(batches: np.ndarray, photons: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Per-photon mean of every bin and its standard error from per-batch sums: batches is (B, bins)
    summed weight, photons (B,) photons per batch. The mean is the total over all photons; the SE is
    the sample standard deviation of the per-batch per-photon values over sqrt(B), as the reference
    estimates R_d, T_t and A (src/io/json_out.cpp:37-64)."""
    batches = np.asarray(batches, dtype=np.float64)
    n = np.asarray(photons, dtype=np.float64)
    b = batches.shape[0]
    mean = batches.sum(axis=0) / n.sum()
    se = (batches / n[:, None]).std(axis=0, ddof=1) / math.sqrt(b)
    return mean, se


def bin_z_two_runs(a_batches: np.ndarray, a_photons: np.ndarray, b_batches: np.ndarray, b_photons: np.ndarray,
                   counts: np.ndarray, floor: int) -> tuple[np.ndarray, int]:
    """|z| per bin with >= floor contributing scores (counts: of either run) between two runs of any
    photon counts: the difference of the per-photon means over the root sum of squares of the two
    standard errors, each from its own run's per-batch sums."""
    ma, sa = per_photon_bins(a_batches, a_photons)
    mb, sb = per_photon_bins(b_batches, b_photons)
    mask = np.asarray(counts).ravel() >= floor
    se = np.hypot(sa, sb)[mask]
    z = np.abs(ma - mb)[mask] / np.where(se > 0, se, np.inf)
    return z, int(mask.sum())


@dataclass(frozen=True)
class Family:
    """Verdict on the |z| of n independent bins: the count above 3 against its null expectation,
    and the largest |z| against the bound that n independent Student-t draws stay under with
    probability 1 - alpha (Bonferroni)."""

    n: int
    over3: int
    over3_limit: float
    zmax: float
    zmax_limit: float

    @property
    def passed(self) -> bool:
        return self.over3 <= self.over3_limit and self.zmax < self.zmax_limit

    def __str__(self) -> str:
        return (f"[{'PASS' if self.passed else 'FAIL'}] {self.n} bins: {self.over3} with |z| > 3 "
                f"(limit {self.over3_limit:.0f}), max |z| {self.zmax:.2f} (limit {self.zmax_limit:.2f})")


def family_check(z: np.ndarray, dof: int, alpha: float = 1e-3) -> Family:
    """Judge |z| of independent bins whose standard errors come from `dof` + 1 batches. Under the
    null, |z| follows Student's t with about `dof` degrees of freedom: P(|z| > 3) = p3; the count
    above 3 may exceed n p3 by twice itself plus five binomial standard deviations (the SE estimates
    of neighbouring bins are correlated through shared photons), and the maximum must stay below
    the two-sided 1 - alpha / n quantile."""
    from scipy import stats

    z = np.asarray(z, dtype=np.float64)
    n = int(z.size)
    if n == 0:
        return Family(0, 0, 0.0, 0.0, math.inf)
    p3 = 2.0 * float(stats.t.sf(3.0, dof))
    limit3 = 2.0 * n * p3 + 5.0 * math.sqrt(n * p3 * (1 - p3))
    zlim = float(stats.t.isf(alpha / (2.0 * n), dof))
    return Family(n, int((z > 3.0).sum()), limit3, float(z.max()), zlim)


def conservation(run: Run, precision: str = "float32") -> tuple[float, float, bool]:
    mean, se = batch_estimate(run.rd + run.tt + run.absorbed, run.photons)
    resid = mean + run.specular - 1.0
    _, ok = compare(resid, se, 0.0, 0.0, CONSERVATION_FLOOR[precision])
    return resid, se, ok

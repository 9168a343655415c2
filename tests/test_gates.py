"""The per-bin parity gates (tests/gates.py) on the CPU: two independent float64 oracle runs of one
medium pass them, and a run with a planted routing mistake (weight moved between bins) fails them.
The mistakes are planted in the oracle's output, on the CPU."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from gates import bin_z_two_runs, family_check, per_photon_bins

SLAB = oracle.Spec(layers=[(1.4, 5.0, 95.0, 0.8, 0.05)], dz=0.0025, dr=0.005, nz=20, nr=50, na=30)
FLOOR = 1000


@pytest.fixture(scope="module")
def two_runs():
    a = oracle.run(SLAB, 300_000, 60, 11, 64, threads=0, counts=True, per_batch_bins=True)
    b = oracle.run(SLAB, 100_000, 40, 12, 64, threads=0, counts=True, per_batch_bins=True)
    return a, b


def _flat(o, name):
    return getattr(o, "b_" + name).reshape(len(o.photons), -1)


def test_per_photon_bins_is_the_batch_estimate():
    rng = np.random.default_rng(1)
    sums = rng.normal(10.0, 1.0, size=(8, 3))
    photons = np.array([100, 100, 101, 99, 100, 100, 100, 100])
    mean, se = per_photon_bins(sums, photons)
    per = sums / photons[:, None]
    assert np.allclose(mean, sums.sum(0) / photons.sum())
    assert np.allclose(se, per.std(0, ddof=1) / np.sqrt(8))


def test_independent_runs_of_different_sizes_pass(two_runs):
    a, b = two_runs
    for name in ("a_rz", "rd_ra", "tt_ra"):
        counts = np.minimum(getattr(a, "n_" + name), getattr(b, "n_" + name)).ravel()
        z, n = bin_z_two_runs(_flat(a, name), a.photons, _flat(b, name), b.photons, counts, FLOOR)
        if n == 0:
            continue
        fam = family_check(z, dof=39)
        assert fam.passed, (name, str(fam))
    z, _ = bin_z_two_runs(_flat(a, "a_rz"), a.photons, _flat(a, "a_rz"), a.photons, a.n_a_rz.ravel(), FLOOR)
    assert not z.any()  # a run against itself


@pytest.mark.parametrize("plant", ["shifted_row", "lost_tile", "scaled"])
def test_a_planted_routing_mistake_fails(two_runs, plant):
    a, b = two_runs
    bad = _flat(b, "a_rz").reshape(len(b.photons), SLAB.nr, SLAB.nz).copy()
    if plant == "shifted_row":  # deposits of radius bin 3 land in bin 4
        bad[:, 4] += bad[:, 3]
        bad[:, 3] = 0
    elif plant == "lost_tile":  # a shared tile that is never flushed
        bad[:, :5, :4] = 0
    else:  # a fixed-point scale off by 10 % (1 % is below one bin's SE: the totals' gate catches that)
        bad *= 1.10
    counts = np.minimum(a.n_a_rz, b.n_a_rz).ravel()
    z, n = bin_z_two_runs(_flat(a, "a_rz"), a.photons, bad.reshape(len(b.photons), -1), b.photons, counts, FLOOR)
    assert n > 100
    assert not family_check(z, dof=39).passed

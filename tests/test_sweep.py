"""The batched sweep: the configuration sampler, validation and the photon-cost estimate that orders
configurations inside a launch (CPU, the estimate against the oracle), and on the GPU bit-for-bit
agreement of every configuration with its own single run, graph reuse across sweeps, the plain
loop baseline, the autotuner, the per-configuration summaries, and oracle parity on a few
configurations."""

from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
import tissuemc_b200 as tmc
from gates import from_engine, from_oracle, identical_photon_gaps


def _scaled(cfgs, cap):
    """A copy of the configurations with photon counts capped (tests need small runs)."""
    out = (tmc.CSweepConfig * len(cfgs))()
    for i, c in enumerate(cfgs):
        out[i] = c
        out[i].photons = min(int(c.photons), cap)
    return out


def test_sampler_is_deterministic_and_in_range():
    a = tmc.sweep_sample(11, 512)
    b = tmc.sweep_sample(11, 40)
    assert all(bytes(a[i]) == bytes(b[i]) for i in range(40))  # config c does not depend on n
    assert bytes(tmc.sweep_sample(12, 1)[0]) != bytes(a[0])
    for c in a:
        assert 1 <= c.num_layers <= 3 and 10_000 <= c.photons <= 1_000_000
        assert c.n_above == 1.0 and c.n_below == 1.0
        ns = {c.layers[i].n for i in range(c.num_layers)}
        assert len(ns) == 1 and 1.33 <= ns.pop() <= 1.5
        for i in range(c.num_layers):
            L = c.layers[i]
            assert 0.01 <= L.mua <= 10 and 0.7 <= L.g <= 0.95 and 0.01 <= L.d <= 1
            assert 1 <= L.mus * (1 - L.g) <= 50 * (1 + 1e-12)
    counts = np.bincount([c.num_layers for c in a], minlength=4)[1:]
    assert counts.min() > 120  # about a third each


def test_sizes_and_validation_name_the_configuration():
    cfgs = tmc.sweep_sample(3, 8)
    opt = tmc.sweep_options()
    sz = tmc.sweep_sizes(cfgs, opt)
    lmax = max(c.num_layers for c in cfgs)
    assert sz.max_layers == lmax
    assert sz.words_per_config == 10 * (4 + lmax) + 64 * 64 + 2 * 64
    assert sz.summary_per_config == 67
    cfgs[5].layers[0].g = 1.0
    with pytest.raises(tmc.ConfigError, match="configuration 5: layer 1: g must be in"):
        tmc.sweep_sizes(cfgs, opt)
    cfgs = tmc.sweep_sample(3, 2)
    cfgs[1].photons = 3
    with pytest.raises(tmc.ConfigError, match="configuration 1: batches cannot exceed"):
        tmc.sweep_sizes(cfgs, opt)
    with pytest.raises(tmc.ConfigError, match="item_photons"):
        tmc.sweep_sizes(tmc.sweep_sample(3, 2), tmc.sweep_options(item_photons=-1))
    for bad, msg in (({"tile_r": 8}, "both be 0"), ({"tile_r": -1, "tile_z": 4}, "both be 0"),
                     ({"tile_r": 65, "tile_z": 4}, "cannot exceed the grid"),
                     ({"tile_r": 32, "tile_z": 32}, "more than 32 KB")):
        with pytest.raises(tmc.ConfigError, match=msg):
            tmc.sweep_sizes(tmc.sweep_sample(3, 2), tmc.sweep_options(**bad))


def _single_run_raw(c, opt):
    """One configuration through tmc_b200_run, widened to the sweep layout."""
    spec = tmc.config_spec(c, opt)
    r = tmc.run(spec, photons=int(c.photons), batches=opt.batches, seed=int(c.seed), fast_math=bool(opt.fast_math))
    return r


def test_photon_cost_estimate_ranks_configurations_like_the_oracle():
    """The sweep runs its configurations longest photons first by an estimate of the steps per
    photon; its ranking agrees with the steps the float64 oracle measures (one photon per batch)."""
    from scipy.stats import spearmanr

    cfgs = tmc.sweep_sample(1, 256)
    cost = tmc.sweep_costs(cfgs)
    assert np.isfinite(cost).all() and (cost > 0).all()
    opt = tmc.sweep_options()
    measured = []
    for c in cfgs:
        spec = tmc.config_spec(c, opt)
        o = oracle.run(oracle.Spec(layers=list(spec.layers), dz=spec.dz, dr=spec.dr, nz=1, nr=1, na=1,
                                   n_above=spec.n_above, n_below=spec.n_below), 64, 64, int(c.seed), 64)
        measured.append(float((o.events + o.boundary_steps).mean()))
    rho = spearmanr(cost, measured).correlation
    assert rho > 0.9, rho
    # the heaviest quarter by the estimate holds most of the heaviest quarter by measurement
    k = len(cfgs) // 4
    top_est, top_meas = set(np.argsort(-cost)[:k]), set(np.argsort(-np.array(measured))[:k])
    assert len(top_est & top_meas) >= 0.75 * k
    with pytest.raises(tmc.ConfigError, match="configuration 1"):
        bad = tmc.sweep_sample(1, 2)
        bad[1].num_layers = 0
        tmc.sweep_costs(bad)


@pytest.mark.gpu
def test_every_configuration_equals_its_single_run_bit_for_bit():
    opt = tmc.sweep_options()
    cfgs = _scaled(tmc.sweep_sample(21, 48), 6000)
    res = tmc.sweep_run(cfgs, opt, raw=True)
    lmax = max(c.num_layers for c in cfgs)
    nb = opt.batches
    for i, c in enumerate(cfgs):
        r = _single_run_raw(c, opt)
        nl = c.num_layers
        block = res.raw[i]
        rows = block[: nb * (4 + lmax)].reshape(nb, 4 + lmax)
        assert np.array_equal(rows[:, : 4 + nl], r.raw[: nb * (4 + nl)].reshape(nb, 4 + nl)), i
        assert not rows[:, 4 + nl:].any()
        assert np.array_equal(block[nb * (4 + lmax):], r.raw[nb * (4 + nl):]), i


@pytest.mark.gpu
def test_loop_baseline_gives_the_same_tallies():
    opt = tmc.sweep_options()
    cfgs = _scaled(tmc.sweep_sample(5, 64), 4000)
    a = tmc.sweep_run(cfgs, opt, raw=True)
    b = tmc.sweep_run_loop(cfgs, opt, raw=True)
    assert np.array_equal(a.raw, b.raw)
    assert a.seconds > 0 and b.seconds > 0


@pytest.mark.gpu
def test_graph_is_reused_for_new_configurations_and_stays_exact():
    opt = tmc.sweep_options()
    first = _scaled(tmc.sweep_sample(100, 96), 3000)
    second = _scaled(tmc.sweep_sample(200, 40), 5000)  # fewer configurations: same captured graph
    a1 = tmc.sweep_run(first, opt, raw=True)
    b = tmc.sweep_run(second, opt, raw=True)
    a2 = tmc.sweep_run(first, opt, raw=True)
    assert np.array_equal(a1.raw, a2.raw) and np.array_equal(a1.summary, a2.summary)
    ref = tmc.sweep_run_loop(second, opt, raw=True)
    assert np.array_equal(b.raw, ref.raw)


@pytest.mark.gpu
def test_summaries_follow_from_the_tallies():
    opt = tmc.sweep_options()
    cfgs = _scaled(tmc.sweep_sample(9, 32), 8000)
    res = tmc.sweep_run(cfgs, opt, raw=True)
    nb, nr = opt.batches, opt.nr
    for i, c in enumerate(cfgs):
        lmax = (res.raw.shape[1] - nr * opt.nz - 2 * nr * opt.na) // nb - 4
        rows = res.raw[i, : nb * (4 + lmax)].reshape(nb, 4 + lmax).astype(np.float64)
        k = 1.0 / (2.0**32 * int(c.photons))
        s = res.summary[i]
        assert math.isclose(s[nr], rows[:, 0].sum() * k, rel_tol=1e-12)
        assert math.isclose(s[nr + 1], rows[:, 1].sum() * k, rel_tol=1e-12, abs_tol=1e-300)
        assert math.isclose(s[nr + 2], rows[:, 4:].sum() * k, rel_tol=1e-12)
        assert math.isclose(s[:nr].sum(), s[nr], rel_tol=1e-9)
        spec = tmc.config_spec(c, opt)
        rsp = ((spec.n_above - spec.layers[0][0]) / (spec.n_above + spec.layers[0][0])) ** 2
        assert abs(s[nr] + s[nr + 1] + s[nr + 2] + rsp - 1) < 5e-3  # conservation per configuration


@pytest.mark.gpu
def test_sweep_of_totals_only_keeps_the_batch_totals():
    """Without profile tallies (profiles = 0, a kernel of its own) every configuration's batch totals
    (R_d, T_t, events, anomalies, absorbed weight per layer) are the same bits as with them, and the
    profile words stay zero."""
    cfgs = _scaled(tmc.sweep_sample(13, 64), 5000)
    on = tmc.sweep_run(cfgs, tmc.sweep_options(), raw=True)
    off = tmc.sweep_run(cfgs, tmc.sweep_options(profiles=0), raw=True)
    opt = tmc.sweep_options()
    nb = opt.batches
    lmax = (on.raw.shape[1] - opt.nr * opt.nz - 2 * opt.nr * opt.na) // nb - 4
    head = nb * (4 + lmax)
    assert np.array_equal(on.raw[:, :head], off.raw[:, :head])
    assert not off.raw[:, head:].any() and on.raw[:, head:].any()
    assert np.array_equal(on.summary[:, opt.nr:], off.summary[:, opt.nr:])


@pytest.mark.gpu
@pytest.mark.parametrize("tile", [(8, 8), (16, 16), (16, 32), (64, 4)])
def test_per_warp_tile_gives_the_same_tallies(tile):
    """Deposits of the configuration a warp is working on go to the warp's shared tile and are
    handed to the global tallies when the warp moves to another configuration: the integer sums
    are the same bits as without the tile (and as each configuration's single run)."""
    cfgs = _scaled(tmc.sweep_sample(31, 200), 5000)
    ref = tmc.sweep_run(cfgs, tmc.sweep_options(), raw=True)
    for item in (64, 256):
        got = tmc.sweep_run(cfgs, tmc.sweep_options(tile_r=tile[0], tile_z=tile[1], item_photons=item), raw=True)
        assert np.array_equal(ref.raw, got.raw), (tile, item)
        assert np.array_equal(ref.summary, got.summary)


@pytest.mark.gpu
def test_autotuner_picks_a_valid_shape():
    cfgs = _scaled(tmc.sweep_sample(8, 128), 2000)
    opt, best = tmc.sweep_autotune(cfgs, tmc.sweep_options())
    assert opt.threads_per_block in (128, 256) and opt.item_photons in (64, 256, 1024)
    assert (opt.tile_r, opt.tile_z) in ((0, 0), (8, 8), (16, 16), (16, 32))
    assert best > 0
    ref = tmc.sweep_run(cfgs, tmc.sweep_options(), raw=True)
    tuned = tmc.sweep_run(cfgs, opt, raw=True)
    assert np.array_equal(ref.raw, tuned.raw)  # the launch shape never changes results


@pytest.mark.gpu
@pytest.mark.parametrize("idx", [0, 1, 2])
def test_sweep_configurations_match_the_oracle_on_identical_photons(idx):
    opt = tmc.sweep_options()
    cfgs = _scaled(tmc.sweep_sample(77, 3), 200_000)
    res = tmc.sweep_run(cfgs, opt, raw=True)
    c = cfgs[idx]
    spec = tmc.config_spec(c, opt)
    g = tmc.decode(spec, tmc.options(photons=int(c.photons), batches=opt.batches, seed=int(c.seed)),
                   _narrow(res.raw[idx], max(x.num_layers for x in cfgs), c.num_layers, opt))
    o = oracle.run(oracle.Spec(layers=list(spec.layers), dz=spec.dz, dr=spec.dr, nz=spec.nz, nr=spec.nr,
                               na=spec.na, n_above=spec.n_above, n_below=spec.n_below),
                   int(c.photons), opt.batches, int(c.seed), 32, threads=0)
    bad = [str(x) for x in identical_photon_gaps(from_oracle(o), from_engine(g)) if not x.passed]
    assert not bad, bad


def _narrow(block, lmax, nl, opt):
    nb = opt.batches
    rows = block[: nb * (4 + lmax)].reshape(nb, 4 + lmax)[:, : 4 + nl].ravel()
    return np.concatenate([rows, block[nb * (4 + lmax):]])


@pytest.mark.gpu
def test_single_configuration_and_sixteen_layers():
    opt = tmc.sweep_options(batches=4)
    spec = tmc.RunSpec(layers=[(1.3 + 0.01 * i, 0.5, 20 + i, 0.8, 0.02) for i in range(16)])
    cfgs = (tmc.CSweepConfig * 1)(tmc.sweep_config(spec, 20_000, 99))
    res = tmc.sweep_run(cfgs, opt, raw=True)
    r = _single_run_raw(cfgs[0], opt)
    assert np.array_equal(res.raw[0], r.raw)


@pytest.mark.gpu
def test_full_size_sweep_properties():
    """The 4096-configuration sweep at its full photon counts (9.1e8 photons): for every
    configuration the 2-D tallies are exact integer refinements of the batch totals (sum of
    A(r,z) = sum of absorbed, of R_d(r,a) = R_d, of T_t(r,a) = T_t), no anomaly, and energy is
    conserved within its batch spread and the float32 transport's rounding drift — the worst
    configuration's residual equals the float32 CPU engine's on identical photons."""
    opt = tmc.sweep_options()
    cfgs = tmc.sweep_sample(1, 4096)
    res = tmc.sweep_run(cfgs, opt, raw=True)
    nb, nr, nz, na = opt.batches, opt.nr, opt.nz, opt.na
    lmax = (res.raw.shape[1] - nr * nz - 2 * nr * na) // nb - 4
    assert res.raw.shape[0] == 4096
    worst, worst_i, worst_resid = -1.0, 0, None
    for i, c in enumerate(cfgs):
        block = res.raw[i]
        rows = block[: nb * (4 + lmax)].reshape(nb, 4 + lmax)
        a_rz = block[nb * (4 + lmax): nb * (4 + lmax) + nr * nz]
        rd_ra = block[nb * (4 + lmax) + nr * nz: nb * (4 + lmax) + nr * nz + nr * na]
        tt_ra = block[nb * (4 + lmax) + nr * nz + nr * na:]
        with np.errstate(over="ignore"):
            assert a_rz.sum(dtype=np.uint64) == rows[:, 4:].sum(dtype=np.uint64), i
            assert rd_ra.sum(dtype=np.uint64) == rows[:, 0].sum(dtype=np.uint64), i
            assert tt_ra.sum(dtype=np.uint64) == rows[:, 1].sum(dtype=np.uint64), i
        assert not rows[:, 3].any(), i  # anomalies
        assert rows[:, 2].all(), i  # events in every batch
        spec = tmc.config_spec(c, opt)
        rsp = ((spec.n_above - spec.layers[0][0]) / (spec.n_above + spec.layers[0][0])) ** 2
        per = np.full(nb, int(c.photons) // nb, dtype=np.float64)
        per[: int(c.photons) % nb] += 1
        resid = (rows[:, 0] + rows[:, 1] + rows[:, 4:].sum(1)).astype(np.float64) / 2.0**32 / per + rsp - 1.0
        se = resid.std(ddof=1) / math.sqrt(nb)
        # a family-wise bound over 4096 configurations (t with 9 degrees of freedom), plus the
        # float32 weight's rounding drift, which grows with the interactions per photon
        events = rows[:, 2].sum() / int(c.photons)
        assert abs(resid.mean()) <= 8 * se + 1e-6 + 1e-8 * events, (i, resid.mean(), se, events)
        if abs(resid.mean()) > worst:
            worst, worst_i, worst_resid = abs(resid.mean()), i, resid
    # the largest residual is the float32 transport's own: the CPU engine in float32 on identical
    # photons leaves the same one
    c = cfgs[worst_i]
    spec = tmc.config_spec(c, opt)
    o = oracle.run(oracle.Spec(layers=list(spec.layers), dz=spec.dz, dr=spec.dr, nz=spec.nz, nr=spec.nr, na=spec.na,
                               n_above=spec.n_above, n_below=spec.n_below),
                   int(c.photons), nb, int(c.seed), 32, threads=0)
    o_resid = (o.rd + o.tt + o.absorbed.sum(1)) / o.photons + o.specular - 1.0
    print(f"worst conservation residual {worst_resid.mean():.3e} (configuration {worst_i}); float32 CPU engine "
          f"{o_resid.mean():.3e}")
    assert abs(worst_resid.mean() - o_resid.mean()) <= 0.05 * abs(o_resid.mean()) + 1e-8

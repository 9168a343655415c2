"""Parity of the B200 walk with the oracle and the reference's own outputs (needs a GPU).

Gates (tests/gates.py): on identical photons (same seed and batches) the GPU's float32 transport
must meet the reference's cross-engine limits against the float32 CPU path; against the float64 CPU
engine every total and every profile bin with at least FLOOR contributing scores must have
|z| < 3; energy is conserved to 3 SE + 1e-6; no anomalies; integer tallies make runs bitwise
reproducible and independent of the batching.
"""

from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest

import oracle
import tissuemc_b200 as tmc
from gates import (batch_estimate, bin_z_scores, bin_z_two_runs, compare, conservation, family_check, from_engine,
                   from_oracle, from_reference_json, identical_photon_gaps)

pytestmark = pytest.mark.gpu

FLOOR = 1000  # contributing scores per bin for the per-bin |z| test


def _ospec(s: tmc.RunSpec) -> oracle.Spec:
    return oracle.Spec(layers=list(s.layers), dz=s.dz, dr=s.dr, nz=s.nz, nr=s.nr, na=s.na,
                       n_above=s.n_above, n_below=s.n_below)


def _assert_gaps(gaps):
    bad = [str(g) for g in gaps if not g.passed]
    assert not bad, "\n".join(bad)


@pytest.fixture(scope="module")
def slab():
    return tmc.workload("slab_n14")


@pytest.fixture(scope="module")
def slab_gpu(slab):
    return tmc.run(slab, photons=1_000_000, batches=80, seed=1)


def test_slab_identical_photons_vs_reference_float32(golden, slab_gpu):
    """cfg 'slab_n14' at its full 1e6 photons vs the reference CPU engine's float32 run."""
    ref = from_reference_json(golden["runs"]["slab_n14_full/float32"]["result"])
    _assert_gaps(identical_photon_gaps(ref, from_engine(slab_gpu), profiles=("a_z", "rd_r")))


def test_slab_identical_photons_vs_oracle_float32_2d(slab, slab_gpu):
    o = oracle.run(_ospec(slab), 1_000_000, 80, 1, 32, threads=0)
    _assert_gaps(identical_photon_gaps(from_oracle(o), from_engine(slab_gpu)))


def test_slab_vs_float64_engine_z_below_3(golden, slab, slab_gpu):
    ref = golden["runs"]["slab_n14_full/float64"]["result"]
    r = from_reference_json(ref)
    g = from_engine(slab_gpu)
    for key in ("rd", "tt", "absorbed"):
        m_ref, se_ref = batch_estimate(getattr(r, key), r.photons)
        m, se = batch_estimate(getattr(g, key), g.photons)
        z, ok = compare(m, se, m_ref, se_ref)
        assert ok and abs(z) < 3, (key, m, m_ref, z)
    o = oracle.run(_ospec(slab), 1_000_000, 80, 1, 64, threads=0, counts=True, per_batch_bins=True)
    for name, ours, ref_t, ref_b, cnt in (
        ("a_rz", slab_gpu.a_rz, o.a_rz, o.b_a_rz, o.n_a_rz),
        ("rd_ra", slab_gpu.rd_ra, o.rd_ra, o.b_rd_ra, o.n_rd_ra),
        ("tt_ra", slab_gpu.tt_ra, o.tt_ra, o.b_tt_ra, o.n_tt_ra),
    ):
        z, n = bin_z_scores(ours.ravel(), ref_t.ravel(), ref_b.reshape(ref_b.shape[0], -1), cnt.ravel(), FLOOR)
        assert n > 0
        assert z.max() < 3, (name, float(z.max()), n)


def test_slab_conservation_and_anomalies(slab_gpu):
    resid, se, ok = conservation(from_engine(slab_gpu))
    assert ok, (resid, se)
    assert int(slab_gpu.anomalies.sum()) == 0


def test_profiles_are_projections_of_the_2d_tallies(slab_gpu):
    r = slab_gpu
    assert np.array_equal(r.a_z, r.a_rz.sum(axis=0)) or np.allclose(r.a_z, r.a_rz.sum(axis=0), rtol=1e-15)
    assert math.isclose(r.rd_r.sum(), r.rd.sum(), rel_tol=1e-12)
    assert math.isclose(r.tt_r.sum(), r.tt.sum(), rel_tol=1e-12)
    assert math.isclose(r.a_z.sum(), r.absorbed.sum(), rel_tol=1e-12)


def test_runs_are_bitwise_reproducible(slab):
    a = tmc.run(slab, photons=200_000, batches=10, seed=5)
    b = tmc.run(slab, photons=200_000, batches=10, seed=5)
    assert np.array_equal(a.raw, b.raw)
    c = tmc.run(slab, photons=200_000, batches=10, seed=6)
    assert not np.array_equal(a.raw, c.raw)


def test_profiles_do_not_depend_on_batching(slab):
    a = tmc.run(slab, photons=100_003, batches=1, seed=3)
    b = tmc.run(slab, photons=100_003, batches=7, seed=3)
    # integer tallies: the same photons give the same sums, whatever the batches
    assert np.array_equal(a.raw[-(a.a_rz.size + 2 * a.rd_ra.size):], b.raw[-(b.a_rz.size + 2 * b.rd_ra.size):])
    assert int(a.events.sum()) == int(b.events.sum())
    assert b.photons.tolist() == oracle.batch_sizes(100_003, 7).tolist()
    assert list(b.first_photon) == list(np.cumsum([0] + list(b.photons[:-1])))


def test_exact_math_variant_passes_the_same_gates(slab):
    g = tmc.run(slab, photons=300_000, batches=20, seed=2, fast_math=False)
    o = oracle.run(_ospec(slab), 300_000, 20, 2, 32, threads=0)
    _assert_gaps(identical_photon_gaps(from_oracle(o), from_engine(g)))


def test_profiles_off_diagnostic_keeps_totals(slab):
    a = tmc.run(slab, photons=50_000, batches=5, seed=9, rung=6)
    b = tmc.run(slab, photons=50_000, batches=5, seed=9, rung=6, profiles=False)
    assert np.array_equal(a.rd, b.rd) and np.array_equal(a.tt, b.tt) and np.array_equal(a.absorbed, b.absorbed)
    assert np.array_equal(a.events, b.events)
    assert not b.a_rz.any() and not b.rd_ra.any() and not b.a_z.any()


def test_run_device_then_decode_equals_run(slab):
    torch = pytest.importorskip("torch")
    opt = tmc.options(photons=30_000, batches=3, seed=4)
    sz = tmc.query_sizes(slab, opt)
    buf = torch.empty(int(sz.device_words), dtype=torch.int64, device="cuda:0")
    stream = torch.cuda.current_stream()
    tmc.run_device(slab, opt, buf.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    raw = buf[:int(sz.tally_words)].cpu().numpy().view(np.uint64)
    dec = tmc.decode(slab, opt, raw)
    ref = tmc.run(slab, opt)
    assert np.array_equal(dec.raw, ref.raw)


def test_device_runs_on_two_streams_at_once_are_independent(slab):
    """Two tmc_b200_run_device calls on two streams, with no synchronisation between them (and a
    tmc_b200_run while they may still be running): each launch claims its photons from a counter in
    its own buffer, so each buffer holds exactly the tallies of that run alone."""
    torch = pytest.importorskip("torch")
    skin = tmc.workload("skin5")
    jobs = [(slab, tmc.options(photons=400_000, batches=8, seed=1)),
            (skin, tmc.options(photons=30_000, batches=3, seed=2)),
            (slab, tmc.options(photons=123_457, batches=5, seed=9))]
    bufs, streams = [], []
    for spec, opt in jobs:
        sz = tmc.query_sizes(spec, opt)
        bufs.append((torch.full((int(sz.device_words),), -1, dtype=torch.int64, device="cuda:0"), int(sz.tally_words)))
        streams.append(torch.cuda.Stream(device=0))
    torch.cuda.synchronize()
    for (spec, opt), (buf, _), st in zip(jobs, bufs, streams):
        tmc.run_device(spec, opt, buf.data_ptr(), st.cuda_stream)
    alone_mid = tmc.run(*jobs[0])  # the regular entry point while the device runs may be in flight
    torch.cuda.synchronize()
    for (spec, opt), (buf, words) in zip(jobs, bufs):
        got = buf[:words].cpu().numpy().view(np.uint64)
        assert np.array_equal(got, tmc.run(spec, opt).raw)
    assert np.array_equal(alone_mid.raw, tmc.run(*jobs[0]).raw)


# ---------------------------------------------------------------- edge cases and other media
# Photons for the edge-case identical-photon tests. A float32 last-bit difference (SFU functions,
# fused multiply-adds) now and then sends one packet down another path; the reference's profile-total
# limit (1e-4 relative) is meant for full-size runs, and at 1e5 photons it tolerates only two or three
# such packets. The expected gap shrinks as 1/sqrt(photons), so these runs use 3e5.
EDGE_PHOTONS = 300_000


def _parity(spec: tmc.RunSpec, photons: int, batches: int, seed: int, profiles=("a_z", "rd_r", "tt_r")):
    g = tmc.run(spec, photons=photons, batches=batches, seed=seed)
    o = oracle.run(_ospec(spec), photons, batches, seed, 32, threads=0)
    return g, o, identical_photon_gaps(from_oracle(o), from_engine(g), profiles=profiles)


def test_single_photon_and_one_photon_per_batch(slab):
    g = tmc.run(slab, photons=1, batches=1, seed=1)
    o = oracle.run(_ospec(slab), 1, 1, 1, 32, threads=1)
    assert int(g.events[0]) == int(o.events[0])
    g = tmc.run(slab, photons=37, batches=37, seed=1)
    o = oracle.run(_ospec(slab), 37, 37, 1, 32, threads=1)
    assert g.photons.tolist() == [1] * 37
    assert abs(int(g.events.sum()) - int(o.events.sum())) <= 2


def test_single_bin_grid():
    spec = tmc.RunSpec(layers=[(1.37, 1, 100, 0.9, 0.1), (1.37, 1, 10, 0, 0.1), (1.37, 2, 10, 0.7, 0.2)],
                       dz=0.01, dr=0.01, nz=1, nr=1, na=1)
    g, o, gaps = _parity(spec, EDGE_PHOTONS, 10, 1)
    _assert_gaps(gaps)
    assert math.isclose(g.a_rz[0, 0], g.absorbed.sum(), rel_tol=1e-12)


def test_sixteen_layers_with_mismatched_indices():
    layers = [(1.3 + 0.02 * i, 0.5 + 0.1 * i, 50 + 5 * i, 0.5 + 0.02 * i, 0.01 + 0.002 * i) for i in range(16)]
    spec = tmc.RunSpec(layers=layers, dz=0.01, dr=0.01, nz=40, nr=40, na=5, n_above=1.0, n_below=1.2)
    _, _, gaps = _parity(spec, EDGE_PHOTONS, 10, 8)
    _assert_gaps(gaps)


@pytest.mark.parametrize("g_aniso", [0.0, -0.3, 0.95])
def test_anisotropy_extremes(g_aniso):
    spec = tmc.RunSpec(layers=[(1.5, 2, 50, g_aniso, 0.05)], dz=0.005, dr=0.005, nz=20, nr=40, na=10)
    _, _, gaps = _parity(spec, EDGE_PHOTONS, 10, 21)
    _assert_gaps(gaps)


def test_absorbing_slab_closed_form():
    n, mua, d = 1.5, 5.0, 0.1
    tau = mua * d
    spec = tmc.RunSpec(layers=[(n, mua, 0.0, 0.0, d)])
    photons = 1_000_000
    g = tmc.run(spec, photons=photons, batches=20, seed=99)
    rsp = 0.04
    loop = 1 / (1 - 0.04 * 0.04 * math.exp(-2 * tau))
    t_exact = (1 - rsp) * math.exp(-tau) * 0.96 * loop
    r_exact = (1 - rsp) * math.exp(-2 * tau) * 0.04 * 0.96 * loop

    def se(x):
        p = x / (1 - rsp)
        return (1 - rsp) * math.sqrt(p * (1 - p) / photons)

    assert abs(g.tt.sum() / photons - t_exact) < 5 * se(t_exact)
    assert abs(g.rd.sum() / photons - r_exact) < 5 * se(r_exact)
    assert abs((g.rd.sum() + g.tt.sum() + g.absorbed.sum()) / photons + g.specular - 1) < 1e-5


@pytest.mark.parametrize("case", ["o1", "v2"])
def test_semi_infinite_vs_h_function(golden, case):
    hf = golden["hf"][case]
    spec = tmc.RunSpec(layers=[(hf["n_medium"], hf["mua"], hf["mus"], 0.0, 1e8)])
    g = tmc.run(spec, photons=1_000_000, batches=20, seed=11)
    m, se = batch_estimate(g.rd, g.photons)
    _, ok = compare(m, se, hf["rd"])
    assert ok, (m, se, hf["rd"])


@pytest.mark.parametrize("case", ["v1_slab", "v3_three_layer"])
def test_published_validation_values(golden, case):
    spec = tmc.parse_mci(golden["dir"] / "validation" / f"{case}.mci")[0]
    photons = 1_000_000
    g = tmc.run(spec, photons=photons, batches=20, seed=1)
    est = {"rd": batch_estimate(g.rd, g.photons), "tt": batch_estimate(g.tt, g.photons)}
    for chk in golden["refs"]["cases"][case]["checks"]:
        if chk["quantity"] not in est:
            continue
        m, se = est[chk["quantity"]]
        rounding = 0.5 * 10 ** (-chk["decimals"]) if "decimals" in chk else 0.0
        se_ref = chk.get("se", se * math.sqrt(photons / chk["n_photons"]) if "n_photons" in chk else 0.0)
        z, ok = compare(m, se, chk["value"], se_ref, rounding)
        assert ok, (case, chk, m, se, z)


# ---------------------------------------------------------------- the five-layer stack (tiled tallies)
@pytest.fixture(scope="module")
def skin():
    return tmc.workload("skin5")


def test_skin5_identical_photons_vs_oracle(skin):
    g, o, gaps = _parity(skin, 200_000, 20, 9, profiles=("a_z", "rd_r", "tt_r", "a_rz", "rd_ra", "tt_ra"))
    _assert_gaps(gaps)


def test_skin5_matches_reference_golden_run(golden, skin):
    ref = golden["runs"]["skin5/float32"]
    g = tmc.run(skin, photons=ref["photons"], batches=ref["batches"], seed=ref["seed"])
    _assert_gaps(identical_photon_gaps(from_reference_json(ref["result"]), from_engine(g), profiles=("a_z", "rd_r")))


def test_skin5_full_size_properties(skin):
    """1e8 photons: conservation, no anomalies, exact projections, bitwise reproducibility."""
    a = tmc.run(skin, batches=100, seed=1)
    assert int(a.photons.sum()) == 100_000_000
    resid, se, ok = conservation(from_engine(a))
    assert ok, (resid, se)
    assert int(a.anomalies.sum()) == 0
    assert math.isclose(a.a_z.sum(), a.absorbed.sum(), rel_tol=1e-12)
    assert math.isclose(a.rd_r.sum(), a.rd.sum(), rel_tol=1e-12)
    b = tmc.run(skin, batches=100, seed=1)
    assert np.array_equal(a.raw, b.raw)


def test_skin5_vs_float64_engine_independent_seeds(skin):
    """Totals against an independent float64 run (different seed): |z| < 3."""
    g = tmc.run(skin, photons=2_000_000, batches=20, seed=101)
    o = oracle.run(_ospec(skin), 200_000, 20, 202, 64, threads=0)
    for key in ("rd", "tt", "absorbed"):
        sg = getattr(g, key) if key != "absorbed" else g.absorbed.sum(axis=1)
        so = getattr(o, key) if key != "absorbed" else o.absorbed.sum(axis=1)
        m, se = batch_estimate(sg, g.photons)
        mo, seo = batch_estimate(so, o.photons)
        z, ok = compare(m, se, mo, seo)
        assert ok, (key, m, mo, z)


# Per-bin parity of the five-layer stack, the workload whose A(r,z) grid (500 x 400) does not fit in
# shared memory: its deposits go through the shared core tile, the shared "cross" (last row and
# column) and the global spill, so every routing path of the tally is covered.
PROFILES_2D = ("a_rz", "rd_ra", "tt_ra")


def _gpu_batch_bins(spec: tmc.RunSpec, opt) -> tuple[np.ndarray, dict]:
    """Per-batch 2-D tallies of one GPU run: each batch of the run's BatchPlan is walked as its own
    photon-id shard (tmc_b200_run_device_range, the same streams and batch membership as in the
    whole run) into a buffer of its own, then decoded."""
    torch = pytest.importorskip("torch")
    sz = tmc.query_sizes(spec, opt)
    words, dwords = int(sz.tally_words), int(sz.device_words)
    sizes = oracle.batch_sizes(int(opt.photons or spec.photons), int(opt.batches))
    bufs = torch.empty((len(sizes), dwords), dtype=torch.int64, device="cuda:0")
    stream = torch.cuda.current_stream().cuda_stream
    first = 0
    for b, n in enumerate(sizes):
        tmc.run_device_range(spec, opt, first, int(n), bufs[b].data_ptr(), stream)
        first += int(n)
    raw = bufs[:, :words].cpu().numpy().view(np.uint64)
    del bufs
    out = {k: np.empty((len(sizes), int(sz.a_rz if k == "a_rz" else sz.ra))) for k in PROFILES_2D}
    for b in range(len(sizes)):
        d = tmc.decode(spec, opt, raw[b])
        for k in PROFILES_2D:
            out[k][b] = getattr(d, k).ravel()
    return sizes, out


@pytest.fixture(scope="module")
def skin_f64(skin):
    """The float64 CPU engine on the five-layer stack: 2e6 photons, 100 batches, seed 7, with per-bin
    score counts and per-batch 2-D bins."""
    return oracle.run(_ospec(skin), 2_000_000, 100, 7, 64, threads=0, counts=True, per_batch_bins=True)


def _totals_within_3_se(res: tmc.RunResult, o) -> None:
    pairs = [("rd", res.rd, o.rd), ("tt", res.tt, o.tt)]
    pairs += [(f"absorbed[{l}]", res.absorbed[:, l], o.absorbed[:, l]) for l in range(o.absorbed.shape[1])]
    for key, sg, so in pairs:
        m, se = batch_estimate(sg, res.photons)
        mo, seo = batch_estimate(so, o.photons)
        z, ok = compare(m, se, mo, seo)
        assert ok and abs(z) < 3, (key, m, mo, z)


def test_skin5_every_profile_bin_vs_float64_engine_same_photons(skin, skin_f64):
    """The GPU's float32 walk against the float64 CPU engine on the same 2e6 photons (seed 7, 100
    batches): |z| < 3 on R_d, T_t, the absorption of every layer, and every A(r,z), R_d(r,a) and
    T_t(r,a) bin with at least FLOOR contributing scores; each side's standard error from its own
    per-batch bins."""
    o = skin_f64
    opt = tmc.options(photons=2_000_000, batches=100, seed=7)
    sizes, gpu = _gpu_batch_bins(skin, opt)
    assert np.array_equal(sizes, o.photons)
    whole = tmc.run(skin, opt)
    for k in PROFILES_2D:  # the shards are the run
        assert np.allclose(gpu[k].sum(axis=0), getattr(whole, k).ravel(), rtol=1e-12, atol=0)
    _totals_within_3_se(whole, o)
    tested = {}
    for k in PROFILES_2D:
        z, n = bin_z_two_runs(gpu[k], sizes, getattr(o, "b_" + k).reshape(len(o.photons), -1), o.photons,
                              getattr(o, "n_" + k).ravel(), FLOOR)
        tested[k] = n
        assert z.size == 0 or z.max() < 3, (k, float(z.max()), n)
    assert tested["a_rz"] > 10_000, tested
    print("skin5 same-photon bins tested:", tested)


def test_skin5_profile_bins_vs_an_independent_float64_run(skin, skin_f64):
    """The GPU at 1e7 photons (seed 101, 100 batches) against the float64 engine's independent 2e6
    photons (seed 7): totals within |z| < 3, and the |z| of every bin with at least FLOOR scores in the
    float64 run judged as a family of independent tests (family_check: the count above 3 near its
    null expectation, the largest below the Bonferroni bound), which a fixed |z| < 3 on each of
    ~10^4-10^5 independent bins cannot be."""
    o = skin_f64
    opt = tmc.options(photons=10_000_000, batches=100, seed=101)
    sizes, gpu = _gpu_batch_bins(skin, opt)
    _totals_within_3_se(tmc.run(skin, opt), o)
    for k in PROFILES_2D:
        z, n = bin_z_two_runs(gpu[k], sizes, getattr(o, "b_" + k).reshape(len(o.photons), -1), o.photons,
                              getattr(o, "n_" + k).ravel(), FLOOR)
        fam = family_check(z, dof=99)
        print(f"skin5 independent {k}: {fam}")
        assert fam.passed, (k, str(fam))


def test_autotuned_plan_gives_the_same_tallies(skin):
    """tmc_b200_autotune searches blocks per SM, block size and the shared tile shapes on a sample of
    the run; whatever it picks, the run's integer tallies are the same bits (only where they are
    summed changes), and the chosen plan is never slower on the sample than the planner's default."""
    opt = tmc.options(photons=2_000_000, batches=20, seed=4)
    tuned, plan, t_default, t_best = tmc.autotune(skin, opt, sample_photons=2_000_000)
    assert t_best <= t_default
    assert plan["smem_bytes"] > 0 and plan["grid"] > 0
    a = tmc.run(skin, opt)
    b = tmc.run(skin, tuned)
    assert np.array_equal(a.raw, b.raw)
    # the tile options on their own, each away from the planner's choice
    for kw in ({"tile_cross": -1}, {"tile_ra_rows": -1}, {"tile_tz": 399}, {"tile_tz": -1},
               {"tile_tz": -1, "tile_cross": -1}, {"blocks_per_sm": 2}, {"threads_per_block": 128}):
        o = tmc.options(photons=300_000, batches=20, seed=4, **kw)
        assert np.array_equal(tmc.run(skin, o).raw, tmc.run(skin, photons=300_000, batches=20, seed=4).raw), kw


# ---------------------------------------------------------------- failure paths and errors
def test_step_cap_turns_endless_packets_into_anomalies(slab):
    """The per-photon step cap (tmc_options.step_cap) ends a packet that is still alive after that
    many steps and counts one anomaly for it, instead of looping: with a cap of 3 steps nearly every
    slab packet (about 20 interactions each) is cut; without a cap none is."""
    cut = tmc.run(slab, photons=50_000, batches=5, seed=1, step_cap=3)
    full = tmc.run(slab, photons=50_000, batches=5, seed=1)
    assert int(full.anomalies.sum()) == 0
    n_cut = int(cut.anomalies.sum())
    assert 0.5 * 50_000 < n_cut <= 50_000
    # a cut packet ran exactly 3 steps: at most 3 absorption events each
    assert int(cut.events.sum()) <= 3 * 50_000 < int(full.events.sum())



def test_bad_config_raises_config_error(slab):
    with pytest.raises(tmc.ConfigError, match="batches cannot exceed the number of photons"):
        tmc.run(slab, photons=5, batches=6)


def test_bad_device_ordinal_is_no_device(slab):
    with pytest.raises(tmc.EngineError) as e:
        tmc.run(slab, photons=100, batches=1, device=63)
    assert e.value.code == tmc.NO_DEVICE


REF_CUDA = Path(__file__).resolve().parents[1] / "baseline" / "_ref" / "tissuemc_cuda"


@pytest.mark.skipif(not REF_CUDA.exists(),
                    reason="the reference's CUDA engine is not built here (make -C baseline)")
@pytest.mark.parametrize("rung", [7, 8])
def test_slab_identical_photons_vs_the_reference_cuda_engine(slab, slab_gpu, tmp_path, rung):
    """The reference's own GPU engine (its rungs 7 and 8, float32 transport) on the same device,
    same seed and batches: the reference's identical-photon limits on totals, per batch, events,
    a_z and rd_r."""
    import json
    import subprocess

    out = tmp_path / "ref.json"
    p = subprocess.run([str(REF_CUDA), "run", str(tmc.CONFIGS / "slab_n14.mci"), "--engine", "cuda", "--rung",
                        str(rung), "--photons", "1000000", "--batches", "80", "--seed", "1", "--output", str(out)],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    ref = from_reference_json(json.loads(out.read_text())["runs"][0])
    _assert_gaps(identical_photon_gaps(ref, from_engine(slab_gpu), profiles=("a_z", "rd_r")))


# ---- the walk's device physics in isolation (tmc_b200_probe_physics), checked the way the
# reference checks its CPU physics (tests/cpp/test_physics.cpp:91-160)

@pytest.mark.parametrize("fast", [True, False])
@pytest.mark.parametrize("g", [0.0, 0.5, 0.9, -0.3])
def test_device_hg_sampler_reproduces_its_first_two_moments(g, fast):
    r = tmc.probe_physics("hg", g, samples=1_000_000, seed=7, fast_math=fast)
    assert r["samples"] >= 1_000_000
    assert -1.0 <= r["min"] and r["max"] <= 1.0
    # E[cos] = g and E[cos^2] = (1 + 2 g^2) / 3; the standard error is below 5.8e-4: ~5 sigma
    assert abs(r["mean"] - g) < 3e-3
    assert abs(r["mean_square"] - (1 + 2 * g * g) / 3) < 3e-3


@pytest.mark.parametrize("fast", [True, False])
@pytest.mark.parametrize("g", [0.0, 0.99])
def test_device_direction_stays_unit_over_millions_of_scatterings(g, fast):
    """32 directions each turned 4e6 times in a row (g = 0.99 keeps consecutive directions close,
    where an unnormalised rotation would drift); the reference's float32 limit is 5e-7."""
    r = tmc.probe_physics("rotate", g, samples=32 * 4_000_000, seed=11, fast_math=fast)
    assert r["worst_norm_error"] < 5e-7


@pytest.mark.parametrize("fast", [True, False])
def test_device_free_paths_are_exponential_with_mean_one_over_mu_t(fast):
    mu_t = 10.0
    r = tmc.probe_physics("step", 0.75, mu_t=mu_t, samples=2_000_000, seed=3, fast_math=fast)
    se = (1 / mu_t) / math.sqrt(r["samples"])
    assert abs(r["mean"] - 1 / mu_t) < 5 * se
    assert abs(r["mean_square"] - 2 / mu_t ** 2) < 5 * math.sqrt(20) * se / mu_t

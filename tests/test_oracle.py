"""The oracle is pinned before it is trusted: known-answer vectors, bit-for-bit agreement with the
reference's own CPU engine, and closed-form / analytic physics checks (CPU only)."""

from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
from gates import batch_estimate, compare

SLAB = oracle.Spec(layers=[(1.4, 5, 95, 0.8, 0.05)], dz=0.0025, dr=0.005, nz=20, nr=50, na=30)


def test_philox_known_answer_vectors(golden):
    # tests/cpp/test_philox.cpp:24-30 of the reference (Random123 kat_vectors)
    for v in golden["kat"]:
        assert oracle.philox(v["ctr"], v["key"]) == v["out"]


@pytest.mark.parametrize("seed,pid", [(0, 0), (1, 7), (42, 1_000_003), (0xDEADBEEFCAFEF00D, 5),
                                      (7, 0x1_0000_0005), (2**64 - 1, 2**64 - 1)])
def test_photon_stream_is_counter_mode_philox(seed, pid):
    # philox.hpp:59-83: counter {id lo, id hi, block, 0}, key = seed; words in block order
    words = oracle.stream(seed, pid, 4 * 5)
    key = [seed & 0xFFFFFFFF, seed >> 32]
    for blk in range(5):
        assert list(words[4 * blk:4 * blk + 4]) == oracle.philox([pid & 0xFFFFFFFF, pid >> 32, blk, 0], key)


def test_streams_are_distinct_across_photons_and_seeds():
    a = set(oracle.stream(1234, 99, 64).tolist())
    assert not a & set(oracle.stream(1234, 100, 64).tolist())
    assert not a & set(oracle.stream(1235, 99, 64).tolist())


@pytest.mark.parametrize("case", ["slab_n14", "slab_n14_full", "skin5", "v1_slab", "v2_semi_infinite",
                                  "v3_three_layer", "o1_semi_infinite_matched", "tissue_g09"])
@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_restatement_equals_reference_engine_bit_for_bit(golden, case, precision):
    """The oracle's per-batch sums, events and 1-D profiles equal the reference CPU engine's
    (oracle/_ref/tissuemc, outputs committed in tests/golden/ref_runs.json) exactly."""
    g = golden["runs"][f"{case}/{precision}"]
    ref = g["result"]
    spec = _spec_from_json(ref)
    o = oracle.run(spec, g["photons"], g["batches"], g["seed"], 64 if precision == "float64" else 32, threads=0)
    b = ref["batches"]
    assert o.rd.tolist() == [x["rd"] for x in b]
    assert o.tt.tolist() == [x["tt"] for x in b]
    assert o.absorbed.tolist() == [x["absorbed"] for x in b]
    assert o.events.tolist() == [x["events"] for x in b]
    assert o.anomalies.tolist() == [x["anomalies"] for x in b]
    assert o.a_z.tolist() == ref["a_z"]
    assert o.rd_r.tolist() == ref["rd_r"]
    assert o.specular == ref["specular"]


def _spec_from_json(r: dict) -> oracle.Spec:
    g = r["grid"]
    return oracle.Spec(layers=[(L["n"], L["mua"], L["mus"], L["g"], L["d"]) for L in r["layers"]],
                       dz=g["dz"], dr=g["dr"], nz=g["nz"], nr=g["nr"], na=1,
                       n_above=r["n_above"], n_below=r["n_below"])


def test_two_dimensional_tallies_project_onto_the_reference_profiles():
    o = oracle.run(SLAB, 20000, 10, 1, 64, threads=0, counts=True, per_batch_bins=True)
    assert np.allclose(o.a_rz.sum(axis=0), o.a_z, rtol=1e-12, atol=0)
    assert np.allclose(o.rd_ra.sum(axis=1), o.rd_r, rtol=1e-12, atol=0)
    assert math.isclose(o.rd_ra.sum(), o.rd.sum(), rel_tol=1e-12)
    assert math.isclose(o.tt_ra.sum(), o.tt.sum(), rel_tol=1e-12)
    assert math.isclose(o.a_rz.sum(), o.absorbed.sum(), rel_tol=1e-12)
    assert np.allclose(o.b_a_rz.sum(axis=0), o.a_rz, rtol=1e-12, atol=1e-12)
    assert int(o.n_a_rz.sum()) == int(o.events.sum())  # one score per absorption event


def _textbook_fresnel(n1, n2, ci):
    st = n1 / n2 * math.sqrt(1 - ci * ci)
    if st >= 1:
        return 1.0
    ct = math.sqrt(1 - st * st)
    rs = (n1 * ci - n2 * ct) / (n1 * ci + n2 * ct)
    rp = (n2 * ci - n1 * ct) / (n2 * ci + n1 * ct)
    return 0.5 * (rs * rs + rp * rp)


@pytest.mark.parametrize("n1,n2", [(1.0, 1.5), (1.5, 1.0), (1.37, 1.0), (1.33, 1.37)])
def test_fresnel_matches_textbook_s_p_formulas(n1, n2):
    # test_physics.cpp:60-77 of the reference
    for ci in np.arange(0.05, 0.999, 0.05):
        r, ca2 = oracle.fresnel(n1, n2, float(ci))
        assert r == pytest.approx(_textbook_fresnel(n1, n2, ci), rel=1e-10)
        if r < 1.0:
            assert n1 * math.sqrt(1 - ci * ci) == pytest.approx(n2 * math.sqrt(1 - ca2 * ca2), rel=1e-10)


def test_fresnel_edge_cases():
    assert oracle.fresnel(1.37, 1.37, 0.3) == (0.0, 0.3)
    assert oracle.fresnel(1.0, 1.5, 1.0)[0] == pytest.approx(0.04)
    assert oracle.fresnel(1.5, 1.0, 0.70) == (1.0, 0.0)  # beyond the critical angle


@pytest.mark.parametrize("precision", [64, 32])
def test_absorbing_slab_closed_form(precision):
    """mu_s = 0: straight down and back with Fresnel reflections at both faces; the geometric
    series gives R_d and T_t exactly (test_physics.cpp:175-214 of the reference)."""
    n, mua, d = 1.5, 5.0, 0.1
    tau = mua * d
    spec = oracle.Spec(layers=[(n, mua, 0.0, 0.0, d)])
    photons = 400_000
    o = oracle.run(spec, photons, 20, 99, precision, threads=0)
    rsp = 0.04
    loop = 1 / (1 - 0.04 * 0.04 * math.exp(-2 * tau))
    t_exact = (1 - rsp) * math.exp(-tau) * (1 - 0.04) * loop
    r_exact = (1 - rsp) * math.exp(-2 * tau) * 0.04 * (1 - 0.04) * loop

    def se(x):
        p = x / (1 - rsp)
        return (1 - rsp) * math.sqrt(p * (1 - p) / photons)

    assert abs(o.tt.sum() / photons - t_exact) < 5 * se(t_exact)
    assert abs(o.rd.sum() / photons - r_exact) < 5 * se(r_exact)
    total = (o.rd.sum() + o.tt.sum() + o.absorbed.sum()) / photons + o.specular
    assert abs(total - 1) < (1e-13 if precision == 64 else 1e-5)


@pytest.mark.parametrize("case,key", [("o1", "rd"), ("v2", "rd")])
def test_semi_infinite_matches_h_function_oracle(golden, case, key):
    """The reference's independent H-function solution (oracle.py:84-105) for a semi-infinite
    isotropic medium; |z| < 3 on R_d."""
    hf = golden["hf"][case]
    spec = oracle.Spec(layers=[(hf["n_medium"], hf["mua"], hf["mus"], 0.0, 1e8)])
    o = oracle.run(spec, 200_000, 20, 11, 64, threads=0)
    mean, se = batch_estimate(o.rd, o.photons)
    z, ok = compare(mean, se, hf[key])
    assert ok, (mean, se, hf[key], z)


@pytest.mark.parametrize("case", ["v1_slab", "v3_three_layer"])
def test_published_validation_values(golden, case):
    """MCML-manual values as quoted by the reference's references.json (rd, tt)."""
    cfg = golden["refs"]["cases"][case]
    text = (golden["dir"] / "validation" / f"{case}.mci").read_text()
    spec = _spec_from_mci(text)
    photons = 200_000
    o = oracle.run(spec, photons, 20, 1, 64, threads=0)
    est = {"rd": batch_estimate(o.rd, o.photons), "tt": batch_estimate(o.tt, o.photons)}
    for chk in cfg["checks"]:
        q = chk["quantity"]
        if q not in est:
            continue
        mean, se = est[q]
        rounding = 0.5 * 10 ** (-chk["decimals"]) if "decimals" in chk else 0.0
        se_ref = chk.get("se", se * math.sqrt(photons / chk["n_photons"]) if "n_photons" in chk else 0.0)
        z, ok = compare(mean, se, chk["value"], se_ref, rounding)
        assert ok, (case, chk, mean, se, z)


def _spec_from_mci(text: str) -> oracle.Spec:
    rows = [ln.split("#")[0].split() for ln in text.splitlines()]
    rows = [r for r in rows if r]
    dz, dr = map(float, rows[4])
    nz, nr, na = map(int, rows[5])
    nl = int(rows[6][0])
    layers = [tuple(map(float, rows[8 + i])) for i in range(nl)]
    return oracle.Spec(layers=layers, dz=dz, dr=dr, nz=nz, nr=nr, na=na, n_above=float(rows[7][0]),
                       n_below=float(rows[8 + nl][0]), photons=int(rows[3][0]))

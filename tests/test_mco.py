"""The MCML .mco writer (tmc_b200_write_mco, pure host code): sections, scaling and integrals,
checked on tallies from the oracle (CPU), and the CLI's --mco option on the GPU."""

from __future__ import annotations

import subprocess

import numpy as np
import pytest

import oracle
import tissuemc_b200 as tmc
from tissuemc_b200.mco import bin_measures, read_mco

TWO = oracle.Spec(layers=[(1.37, 1.0, 100.0, 0.9, 0.1), (1.37, 1.0, 10.0, 0.0, 0.1)], dz=0.01, dr=0.01, nz=40,
                  nr=50, na=30, n_above=1.0, n_below=1.0)


def _result_from_oracle(spec: oracle.Spec, photons: int, batches: int, seed: int) -> tmc.RunResult:
    o = oracle.run(spec, photons, batches, seed, 64, threads=0)
    first = np.concatenate([[0], np.cumsum(o.photons)[:-1]]).astype(np.uint64)
    rs = tmc.RunSpec(layers=list(spec.layers), photons=photons, dz=spec.dz, dr=spec.dr, nz=spec.nz, nr=spec.nr,
                     na=spec.na, n_above=spec.n_above, n_below=spec.n_below)
    return tmc.RunResult(spec=rs, seed=seed, first_photon=first, photons=o.photons.astype(np.uint64), rd=o.rd,
                         tt=o.tt, absorbed=o.absorbed, events=o.events, anomalies=o.anomalies, a_z=o.a_z,
                         rd_r=o.rd_r, tt_r=o.tt_ra.sum(1), a_rz=o.a_rz, rd_ra=o.rd_ra, tt_ra=o.tt_ra,
                         raw=np.zeros(0, np.uint64), specular=o.specular, kernel_seconds=0.0, wall_seconds=0.0,
                         device="oracle")


@pytest.fixture(scope="module")
def written(tmp_path_factory):
    res = _result_from_oracle(TWO, 20_000, 10, 5)
    path = tmp_path_factory.mktemp("mco") / "two.mco"
    tmc.write_mco(res, path)
    return res, read_mco(path), path


def test_input_parameters_round_trip(written):
    res, m, path = written
    assert m["file"] == "two.mco" and m["photons"] == 20_000
    assert (m["dz"], m["dr"], m["nz"], m["nr"], m["na"]) == (0.01, 0.01, 40, 50, 30)
    assert m["n_above"] == 1.0 and m["n_below"] == 1.0
    np.testing.assert_allclose(m["layers"], np.array(TWO.layers))
    text = path.read_text()
    for key in ("InParm", "RAT", "A_l", "A_z", "Rd_r", "Rd_a", "Tt_r", "Tt_a", "A_rz", "Rd_ra", "Tt_ra"):
        assert f"\n{key}" in text, key


def test_scaling_follows_the_mcml_definitions(written):
    res, m, _ = written
    N = float(res.photons.sum())
    area, omega, cosa = bin_measures(TWO.nr, TWO.dr, TWO.na)
    rtol = 1e-4  # five significant digits in the file
    assert m["specular"] == pytest.approx(res.specular, rel=1e-5)
    assert m["rd"] == pytest.approx(res.rd.sum() / N, rel=1e-5)
    assert m["tt"] == pytest.approx(res.tt.sum() / N, rel=1e-5)
    assert m["a"] == pytest.approx(res.absorbed.sum() / N, rel=1e-5)
    np.testing.assert_allclose(m["A_l"], res.absorbed.sum(0) / N, rtol=rtol)
    np.testing.assert_allclose(m["A_z"], res.a_rz.sum(0) / (N * TWO.dz), rtol=rtol)
    np.testing.assert_allclose(m["A_rz"], res.a_rz / (N * area[:, None] * TWO.dz), rtol=rtol)
    np.testing.assert_allclose(m["Rd_r"], res.rd_ra.sum(1) / (N * area), rtol=rtol)
    np.testing.assert_allclose(m["Rd_a"], res.rd_ra.sum(0) / (N * omega), rtol=rtol)
    np.testing.assert_allclose(m["Rd_ra"], res.rd_ra / (N * area[:, None] * omega * cosa), rtol=rtol)
    np.testing.assert_allclose(m["Tt_r"], res.tt_ra.sum(1) / (N * area), rtol=rtol)
    np.testing.assert_allclose(m["Tt_ra"], res.tt_ra / (N * area[:, None] * omega * cosa), rtol=rtol)
    # A_z is also the reference's own 1-D depth profile, per photon and per cm
    np.testing.assert_allclose(m["A_z"], res.a_z / (N * TWO.dz), rtol=rtol)


def test_every_profile_integrates_to_its_total(written):
    _, m, _ = written
    area, omega, cosa = bin_measures(TWO.nr, TWO.dr, TWO.na)
    tol = dict(rel=5e-4)
    assert (m["Rd_r"] * area).sum() == pytest.approx(m["rd"], **tol)
    assert (m["Rd_a"] * omega).sum() == pytest.approx(m["rd"], **tol)
    assert (m["Rd_ra"] * area[:, None] * omega * cosa).sum() == pytest.approx(m["rd"], **tol)
    assert (m["Tt_r"] * area).sum() == pytest.approx(m["tt"], **tol)
    assert (m["Tt_a"] * omega).sum() == pytest.approx(m["tt"], **tol)
    assert (m["A_z"] * TWO.dz).sum() == pytest.approx(m["a"], **tol)
    assert (m["A_rz"] * area[:, None] * TWO.dz).sum() == pytest.approx(m["a"], **tol)
    assert m["A_l"].sum() == pytest.approx(m["a"], **tol)
    # energy balance, to the six significant digits of the RAT lines
    assert m["specular"] + m["rd"] + m["a"] + m["tt"] == pytest.approx(1.0, abs=3e-6)


def test_ring_solid_angles_cover_the_hemisphere():
    _, omega, _ = bin_measures(1, 0.01, 30)
    assert omega.sum() == pytest.approx(2 * np.pi, rel=1e-12)  # sum of 4 pi sin(a) sin(da/2) over the rings


def test_writer_rejects_missing_arrays_and_bad_paths(written, tmp_path):
    res, _, _ = written
    import ctypes

    opt = tmc.options(seed=1, batches=10)
    r = tmc.CResult()
    st = tmc.CStatus()
    c = res.spec.to_c()
    rc = tmc.lib().tmc_b200_write_mco(ctypes.byref(c), ctypes.byref(opt), ctypes.byref(r),
                                      str(tmp_path / "x.mco").encode(), ctypes.byref(st))
    assert rc == 5 and b"a_rz" in st.message  # TMC_BAD_ARGUMENT
    with pytest.raises(tmc.EngineError, match="cannot open"):
        tmc.write_mco(res, tmp_path / "no" / "such" / "dir" / "x.mco")


@pytest.mark.gpu
def test_cli_writes_an_mco_that_matches_its_json(tmp_path):
    import json

    from tissuemc_b200 import build as b

    mci = tmp_path / "slab.mci"
    mci.write_text(oracle.Spec(layers=[(1.4, 5.0, 95.0, 0.8, 0.05)], dz=0.0025, dr=0.005, nz=20, nr=50, na=30,
                               photons=100_000).to_mci())
    out, mco = tmp_path / "out.json", tmp_path / "slab.mco"
    p = subprocess.run([str(b.CLI), "run", str(mci), "--output", str(out), "--mco", str(mco)], capture_output=True,
                       text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    run = json.loads(out.read_text())["runs"][0]
    m = read_mco(mco)
    N = sum(bt["photons"] for bt in run["batches"])
    assert m["photons"] == N == 100_000
    assert m["rd"] == pytest.approx(sum(bt["rd"] for bt in run["batches"]) / N, rel=1e-5)
    area, omega, cosa = bin_measures(50, 0.005, 30)
    np.testing.assert_allclose(m["Rd_r"], np.array(run["rd_r"]) / (N * area), rtol=1e-4)
    np.testing.assert_allclose(m["A_z"], np.array(run["a_z"]) / (N * 0.0025), rtol=1e-4)

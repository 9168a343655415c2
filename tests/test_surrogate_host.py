"""Host logic of the surrogate on the CPU: the feature encoding and its inverse, the targets and the
diffuse-reflectance total that the gate reads, the gate's spread, and the Levenberg-Marquardt fit
driven through a stand-in model with a known answer. The network's kernels are covered on the GPU
by test_surrogate.py."""

from __future__ import annotations

import numpy as np
import pytest

import tissuemc_b200 as tmc
from tissuemc_b200 import surrogate as S


def test_features_and_configurations_round_trip():
    cfgs = tmc.sweep_sample(5, 256)
    X = S.features(cfgs)
    assert X.shape == (256, S.N_FEAT) and np.isfinite(X).all()
    for i, c in enumerate(cfgs):
        nl = c.num_layers
        for l in range(3):
            assert bool(S.present(X[i:i + 1], l)[0]) == (l < nl)
            if l < nl:
                L = c.layers[l]
                assert X[i, 4 * l] == pytest.approx(np.log10(L.mua), abs=1e-12)
                assert X[i, 4 * l + 1] == pytest.approx(np.log10(L.mus * (1 - L.g)), abs=1e-12)
                assert X[i, 4 * l + 2] == L.g
                assert S.thickness(X[i:i + 1], l)[0] == pytest.approx(L.d, rel=1e-12)
            else:  # an absent slot: zero optics and the absent-thickness marker
                assert (X[i, 4 * l:4 * l + 3] == 0).all()
                assert X[i, 4 * l + 3] == S.ABSENT_LOG_D
                assert S.thickness(X[i:i + 1], l)[0] == 0.0
        assert X[i, 12] == c.layers[0].n
        back = S.config_from_features(X[i], int(c.photons), int(c.seed))
        assert back.num_layers == nl and back.photons == c.photons and back.seed == c.seed
        for l in range(nl):
            a, b = back.layers[l], c.layers[l]
            for k in ("n", "mua", "mus", "g", "d"):
                assert getattr(a, k) == pytest.approx(getattr(b, k), rel=1e-12), (i, l, k)
        np.testing.assert_allclose(S.features([back])[0], X[i], rtol=0, atol=1e-12)


def test_targets_profile_and_reflectance_total():
    rng = np.random.default_rng(3)
    n = 32
    area = S.annulus_areas()
    summary = np.zeros((n, S.N_RD + 3))
    # R_d(r) per photon in each annulus, decaying with r, above the floor per unit area
    r = np.arange(S.N_RD)
    summary[:, :S.N_RD] = area * 10.0 ** (1.5 - 0.05 * r[None, :] - rng.uniform(0, 0.5, (n, 1)))
    summary[:, S.N_RD] = summary[:, :S.N_RD].sum(1)
    summary[:, S.N_RD + 1:] = rng.uniform(0, 0.5, (n, 2))  # T_t, A
    Y = S.targets(summary)
    assert Y.shape == (n, S.N_OUT)
    np.testing.assert_allclose(S.rd_profile(Y) * area, summary[:, :S.N_RD], rtol=1e-12)
    np.testing.assert_array_equal(Y[:, S.N_RD:], summary[:, S.N_RD + 1:])
    np.testing.assert_allclose(S.rd_total(Y), summary[:, S.N_RD], rtol=1e-12)
    # an empty bin is floored, not -inf
    summary[0, 10] = 0.0
    assert S.targets(summary)[0, 10] == np.log10(S.RD_FLOOR)
    # the annuli tile the disc of radius nr dr
    assert area.sum() == pytest.approx(np.pi * (S.N_RD * 0.01) ** 2, rel=1e-12)


def test_spread_and_gate():
    rng = np.random.default_rng(4)
    n = 16
    base = rng.normal(0.0, 0.3, (n, S.N_OUT))
    same = np.repeat(base[None], 4, 0)
    assert np.allclose(S.spread(same), 0.0) and not S.gate(same).any()
    # members whose profiles differ by a factor (1 + e_k): their totals differ by the same factor
    e = np.array([-0.02, 0.0, 0.005, 0.03])
    scaled = same.copy()
    scaled[:, :, :S.N_RD] += np.log10(1 + e)[:, None, None]
    f = 1 + e
    expect = f.std(ddof=1) / f.mean()
    np.testing.assert_allclose(S.spread(scaled), expect, rtol=1e-10)
    assert S.gate(scaled, threshold=expect * 0.99).all()
    assert not S.gate(scaled, threshold=expect * 1.01).any()
    # T_t and A do not enter the gate
    other = same.copy()
    other[:, :, S.N_RD:] += rng.normal(0, 1, (4, n, 2))
    assert np.allclose(S.spread(other), 0.0)


class _KnownModel:
    """A smooth stand-in for the ensemble: log10 R_d(r) as a non-linear function of features 0
    and 4 (log10 mu_a of two layers), the other columns ignored."""

    def __init__(self):
        r = np.linspace(0, 1, S.N_RD)
        self.w, self.v, self.u = 1.0 - r, -0.5 - r ** 2, np.sin(3 * r)

    def predict(self, th: np.ndarray) -> np.ndarray:
        a, b = th[:, 0:1], th[:, 4:5]
        y = np.zeros((len(th), S.N_OUT))
        y[:, :S.N_RD] = a * self.w + b * self.v + 0.3 * np.tanh(a * b) * self.u
        return y


def test_levenberg_marquardt_recovers_a_known_answer():
    rng = np.random.default_rng(5)
    model = _KnownModel()
    n = 64
    truth = np.zeros((n, S.N_FEAT))
    truth[:, [0, 4]] = rng.uniform(-1, 1, (n, 2))
    truth[:, 12] = 1.4
    obs = model.predict(truth)[:, :S.N_RD]
    mask = np.ones(S.N_RD)
    mask[50:] = 0.0  # bins left out of the fit
    obs[:, 50:] += 10.0  # ...so what they hold cannot matter
    start = truth.copy()
    start[:, [0, 4]] += rng.uniform(-0.4, 0.4, (n, 2))
    fit, res = S.lm_fit(model, start, obs, mask, free=[0, 4], iters=40)
    np.testing.assert_allclose(fit[:, [0, 4]], truth[:, [0, 4]], atol=1e-6)
    assert (res < 1e-6).all()
    keep = [c for c in range(S.N_FEAT) if c not in (0, 4)]
    np.testing.assert_array_equal(fit[:, keep], start[:, keep])  # fixed features stay put


def test_fit_uncertainty_is_calibrated_and_flags_what_the_data_cannot_fix():
    """lm_uncertainty on the known model: with 1 % noise on the observations the recovered
    parameters lie within 3 standard errors of the truth in nearly every fit; a parameter the model
    ignores (feature 1) has no curvature and every fit that frees it is flagged."""
    rng = np.random.default_rng(7)
    model = _KnownModel()
    n = 200
    truth = np.zeros((n, S.N_FEAT))
    truth[:, [0, 4]] = rng.uniform(-1, 1, (n, 2))
    obs = model.predict(truth)[:, :S.N_RD] + rng.normal(0, 0.01, (n, S.N_RD))
    mask = np.ones((n, S.N_RD))
    start = truth.copy()
    start[:, [0, 4]] += rng.uniform(-0.3, 0.3, (n, 2))
    fit, _ = S.lm_fit(model, start, obs, mask, free=[0, 4], iters=40)
    se, flag = S.lm_uncertainty(model, fit, obs, mask, [0, 4])
    assert not flag.any() and np.isfinite(se).all()
    z = np.abs(fit[:, [0, 4]] - truth[:, [0, 4]]) / se
    assert (z < 3).mean() > 0.97
    se2, flag2 = S.lm_uncertainty(model, fit, obs, mask, [0, 1, 4])  # feature 1 does not enter the model
    assert flag2.all()

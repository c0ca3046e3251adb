"""Conductivity Monte Carlo host logic (cunibs_b200.uq): sampling, sensitivity shares, result files."""

from __future__ import annotations

import numpy as np
import pytest

from cunibs_b200 import Placement
from cunibs_b200.fem import TISSUE_CONDUCTIVITY
from cunibs_b200.uq import (ConductivityUQConfig, ConductivityUQResult, sample_conductivities,
                            tissue_sensitivity)


def test_lognormal_draws_are_positive_with_the_nominal_mean():
    tags = (1, 2, 3, 4, 5)
    cfg = ConductivityUQConfig(n_samples=40000, seed=3)
    s = sample_conductivities(cfg, tags)
    assert s.shape == (40000, 5) and (s > 0).all()
    nominal = np.array([TISSUE_CONDUCTIVITY[t] for t in tags])
    np.testing.assert_allclose(s.mean(0), nominal, rtol=0.01)
    covs = np.array([cfg.cov_for(t) for t in tags])
    np.testing.assert_allclose(s.std(0) / s.mean(0), covs, rtol=0.05)
    again = sample_conductivities(cfg, tags)
    np.testing.assert_array_equal(s, again)  # seeded


def test_normal_draws_are_clamped_and_overrides_apply():
    cfg = ConductivityUQConfig(n_samples=5000, seed=1, distribution="normal", tissue_cov={4: 3.0})
    s = sample_conductivities(cfg, (4,))
    assert (s >= 1e-6 * TISSUE_CONDUCTIVITY[4]).all() and (s == 1e-6 * TISSUE_CONDUCTIVITY[4]).any()
    with pytest.raises(ValueError):
        sample_conductivities(ConductivityUQConfig(distribution="uniform"), (1,))


def test_tissue_sensitivity_recovers_log_linear_shares():
    rng = np.random.default_rng(0)
    sig = np.exp(rng.normal(0.0, [0.1, 0.3, 0.2], size=(20000, 3)))
    y = np.exp(0.5 * np.log(sig[:, 0]) - 1.0 * np.log(sig[:, 1]) + 0.0 * np.log(sig[:, 2]))
    share = tissue_sensitivity(sig, y, (1, 2, 3))
    total = 0.25 * 0.01 + 1.0 * 0.09
    assert share[1] == pytest.approx(0.25 * 0.01 / total, rel=0.05)
    assert share[2] == pytest.approx(0.09 / total, rel=0.05)
    assert share[3] == pytest.approx(0.0, abs=1e-6)


def test_result_round_trip(tmp_path):
    rng = np.random.default_rng(2)
    n_tets = 50
    tags = np.full(n_tets, 2, np.int32)
    res = ConductivityUQResult(
        mean_magnE=rng.random(n_tets), std_magnE=rng.random(n_tets) * 0.1, cov_magnE=rng.random(n_tets) * 0.2,
        n_samples=4, perturbed_tags=(2, 3), sigma_samples=rng.random((4, 2)) + 0.1,
        vols=rng.random(n_tets).astype(np.float32) + 0.1, tet_tags=tags, barycenters_mm=rng.random((n_tets, 3)),
        placement=Placement([0, 0, 90.0], [0, 50, 90.0]), coil_name="fig8", didt=1e6,
        peak_samples=rng.random(4) + 1, focality_samples=rng.random(4), peak_location_samples=rng.random((4, 3)),
        iteration_samples=np.arange(4, dtype=np.int32), recovery="raw")
    res.summary = res.compute_summary()
    res.save(tmp_path / "u.npz")
    back = ConductivityUQResult.load(tmp_path / "u.npz")
    np.testing.assert_array_equal(back.mean_magnE, res.mean_magnE)
    np.testing.assert_array_equal(back.peak_samples, res.peak_samples)
    assert back.perturbed_tags == (2, 3) and back.placement.distance_mm == 4.0
    assert back.peak_mean_magnE() == res.peak_mean_magnE()
    assert back.max_local_cov() == pytest.approx(float(res.cov_magnE.max()))
    assert set(back.tissue_sensitivity("focality")) == {2, 3}
    with pytest.raises(ValueError, match="Unknown output"):
        back.tissue_sensitivity("roi")


def test_zero_cov_draws_are_the_nominal_conductivity():
    tags = (2, 3)
    for dist in ("lognormal", "normal"):
        cfg = ConductivityUQConfig(n_samples=16, seed=5, tissue_cov={2: 0.0, 3: 0.0}, distribution=dist)
        s = sample_conductivities(cfg, tags)
        np.testing.assert_allclose(s, np.tile([TISSUE_CONDUCTIVITY[2], TISSUE_CONDUCTIVITY[3]], (16, 1)), rtol=1e-15)


def test_draws_of_a_smaller_ensemble_are_a_prefix():
    tags = (1, 2, 3)
    small = sample_conductivities(ConductivityUQConfig(n_samples=3, seed=4), tags)
    large = sample_conductivities(ConductivityUQConfig(n_samples=9, seed=4), tags)
    np.testing.assert_array_equal(large[:3], small)


def test_roi_samples_round_trip_and_feed_the_sensitivity(tmp_path):
    rng = np.random.default_rng(3)
    n, tags = 64, (2, 3)
    sig = np.exp(rng.normal(0.0, 0.2, size=(n, 2)))
    roi = np.exp(0.8 * np.log(sig[:, 1]))  # driven by tag 3 alone
    res = ConductivityUQResult(
        mean_magnE=None, std_magnE=None, cov_magnE=None, n_samples=n, perturbed_tags=tags, sigma_samples=sig,
        vols=None, tet_tags=None, barycenters_mm=None, placement=Placement([0, 0, 90.0], [0, 50, 90.0]),
        coil_name="fig8", didt=1e6, peak_samples=np.ones(n), focality_samples=np.ones(n),
        peak_location_samples=np.zeros((n, 3)), iteration_samples=np.zeros(n, np.int32),
        roi_samples={"M1": roi})
    share = res.tissue_sensitivity("M1")
    assert share[3] == pytest.approx(1.0, abs=1e-9) and share[2] == pytest.approx(0.0, abs=1e-9)
    assert res.tissue_sensitivity("peak") == {2: 0.0, 3: 0.0}
    with pytest.raises(ValueError, match="available"):
        res.tissue_sensitivity("V1")
    res.save(tmp_path / "r.npz")
    back = ConductivityUQResult.load(tmp_path / "r.npz")
    assert list(back.roi_samples) == ["M1"]
    np.testing.assert_array_equal(back.roi_samples["M1"], roi)

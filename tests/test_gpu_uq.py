"""Conductivity Monte Carlo on the GPU (Subject.simulate_conductivity_uq, cunibs_sigma_*). Needs a B200.

Each draw is solved with the nominal coarse AMG levels kept, from the sensitivity-subspace guess;
its gray-matter peak must match a solve after a full re-setup for that draw, the moments must be
the draws' mean and spread, and the subject must be back at the nominal conductivities afterwards,
bit for bit.
"""

from __future__ import annotations

import numpy as np
import pytest

from cunibs_b200 import Placement, Subject
from cunibs_b200.synthetic import figure8_coil, sphere_head
from cunibs_b200.uq import ConductivityUQConfig, nominal_sigma_table, sample_conductivities

pytestmark = pytest.mark.gpu


def test_conductivity_uq_matches_per_draw_full_resetup():
    mesh = sphere_head(6.0, 90.0, jitter_mm=0.3, seed=1)
    coil = figure8_coil(64)
    top = np.array([0.0, 0.0, 90.0])
    site = Placement(top, top + [0, 50, 0])
    cfg = ConductivityUQConfig(n_samples=5, seed=4)
    subj = Subject(mesh, tolerance=1e-10)
    before = subj.simulate(coil, site, magnitude=True, recovery="raw").magnE
    res = subj.simulate_conductivity_uq(coil, site, cfg, moments=True, recovery="raw")
    after = subj.simulate(coil, site, magnitude=True, recovery="raw").magnE
    np.testing.assert_array_equal(after, before)
    assert res.n_samples == 5 and res.full_resetups == 0
    tags = res.perturbed_tags
    np.testing.assert_array_equal(res.sigma_samples, sample_conductivities(cfg, tags))
    ref = Subject(mesh, tolerance=1e-10)
    fields = []
    for i in range(cfg.n_samples):
        sigma = nominal_sigma_table()
        sigma[list(tags)] = res.sigma_samples[i]
        ref.context.set_conductivity(sigma)
        r = ref.simulate(coil, site, magnitude=True, recovery="raw")
        assert res.peak_samples[i] == pytest.approx(r.peak_magnE(), rel=1e-6)
        assert res.focality_samples[i] == pytest.approx(r.summary["focality_m3"]["0.5"], rel=1e-4)
        fields.append(r.magnE.astype(np.float64))
    f = np.stack(fields)
    gm = res.tet_tags == 2
    np.testing.assert_allclose(res.mean_magnE[gm], f.mean(0)[gm], rtol=1e-5)
    np.testing.assert_allclose(res.std_magnE[gm], f.std(0)[gm], rtol=1e-3, atol=1e-6 * f.max())
    assert res.summary is not None and res.max_local_cov() > 0
    assert res.peak_mean_magnE() == pytest.approx(float(f.mean(0)[gm].max()), rel=1e-5)
    assert np.isclose(sum(res.tissue_sensitivity().values()), 1.0, atol=0.5)
    subj.free()
    ref.free()


def test_a_draw_the_kept_hierarchy_cannot_finish_gets_a_full_resetup():
    """With a tight iteration budget and wide draws, the kept coarse levels miss it on some draws
    (even after the solver's own FP64 retry, which grants a second budget): those are solved again
    after a full re-setup, and the subject ends on its nominal hierarchy (the same field as
    before, bit for bit)."""
    mesh = sphere_head(6.0, 90.0, jitter_mm=0.3, seed=1)
    coil = figure8_coil(64)
    top = np.array([0.0, 0.0, 90.0])
    site = Placement(top, top + [0, 50, 0])
    probe = Subject(mesh, tolerance=1e-8)
    nominal_iters = probe.simulate(coil, site, recovery="raw").iterations
    probe.free()
    budget = nominal_iters // 2 + 2  # solve plus retry: about nominal + 3 iterations in all
    subj = Subject(mesh, tolerance=1e-8, max_iters=budget)
    before = subj.simulate(coil, site, magnitude=True, recovery="raw").magnE
    cfg = ConductivityUQConfig(n_samples=6, seed=9, tissue_cov={t: 1.5 for t in range(1, 11)})
    res = subj.simulate_conductivity_uq(coil, site, cfg, recovery="raw")
    assert res.full_resetups >= 1
    assert (res.iteration_samples <= 2 * budget).all()
    np.testing.assert_array_equal(subj.simulate(coil, site, magnitude=True, recovery="raw").magnE, before)
    subj.free()


def test_placements_batched_per_draw_match_single_runs():
    """A sequence of placements shares every draw's re-setup and one block solve; each result is
    the one a run of that placement alone gives, bit for bit."""
    mesh = sphere_head(6.0, 90.0, jitter_mm=0.3, seed=1)
    coil = figure8_coil(64)
    sites = [Placement([0.0, 0.0, 90.0], [0.0, 50.0, 90.0]), Placement([25.0, 0.0, 86.4], [25.0, 50.0, 86.4]),
             Placement([0.0, -25.0, 86.4], [50.0, -25.0, 86.4])]
    cfg = ConductivityUQConfig(n_samples=4, seed=2)
    subj = Subject(mesh, tolerance=1e-8)
    together = list(subj.iter_simulate_conductivity_uq(coil, sites, cfg, moments=True, recovery="harmonic"))
    for site, r in zip(sites, together):
        alone = subj.simulate_conductivity_uq(coil, site, cfg, moments=True, recovery="harmonic")
        np.testing.assert_array_equal(r.peak_samples, alone.peak_samples)
        np.testing.assert_array_equal(r.iteration_samples, alone.iteration_samples)
        np.testing.assert_array_equal(r.mean_magnE, alone.mean_magnE)
        assert r.placement is site
    subj.free()


def test_study_guess_cuts_iterations_against_the_zero_guess_on_the_same_hierarchy():
    """cunibs_sigma_draw against cunibs_context_set_conductivity_keep_coarse + a zero-guess block
    solve of the same draw: the same operator and coarse levels, so the same field to the solve
    tolerance; the sensitivity-subspace guess starts well below the zero guess's residual and
    needs fewer iterations."""
    mesh = sphere_head(6.0, 90.0, jitter_mm=0.3, seed=1)
    coil = figure8_coil(64)
    centers = np.array([[0.0, 0.0, 90.0], [25.0, 0.0, 86.4]])
    handles = centers + [0.0, 50.0, 0.0]
    dists = [4.0, 4.0]
    subj = Subject(mesh, tolerance=1e-8)
    ctx = subj.context
    nominal = nominal_sigma_table()
    tags = tuple(int(t) for t in np.unique(mesh.tet_tags))
    draws = sample_conductivities(ConductivityUQConfig(n_samples=3, seed=5), tags)
    ranks = ctx.sigma_begin(coil, centers, handles, dists, 1e6, nominal, tags, magnitude=True, recovery="raw")
    assert (ranks >= 1).all() and (ranks <= len(tags)).all()
    with pytest.raises(ValueError, match="conductivity study is open"):
        ctx.solve_block(coil, centers, handles, dists, 1e6)
    with pytest.raises(ValueError, match="conductivity study is open"):
        ctx.set_conductivity(nominal)
    outs = [ctx.sigma_draw(d) for d in draws]
    ctx.sigma_end()
    with pytest.raises(ValueError, match="no conductivity study"):
        ctx.sigma_draw(draws[0])
    for d, o in zip(draws, outs):
        sigma = nominal.copy()
        sigma[list(tags)] = d
        ctx.set_conductivity(sigma, keep_coarse=True)
        ref = ctx.solve_block(coil, centers, handles, dists, 1e6, magnitude=True, recovery="raw")
        assert o["resetup"] == 0
        assert (o["init_relres"] < 0.2).all(), o["init_relres"]
        assert (o["iterations"] <= ref["iterations"]).all() and o["iterations"].sum() < ref["iterations"].sum()
        np.testing.assert_allclose(o["summary"][:, 0], ref["summary"][:, 0], rtol=1e-6)
        diff = np.linalg.norm(o["magnE"] - ref["magnE"], axis=1) / np.linalg.norm(ref["magnE"], axis=1)
        assert (diff < 1e-6).all(), diff
    ctx.set_conductivity(nominal, keep_coarse=True)
    subj.free()


def test_study_properties_homogeneous_small_perturbation_subset_and_ensemble_size():
    """Four properties of the reference's test_uq.py on the native study:
    * a one-tissue head: scaling its only conductivity leaves the field as it was (and the nominal
      solution is already the draw's, so the guess starts at the nominal solve's residual);
    * a small perturbation: the first-order guess is nearly exact;
    * a subset of perturbed tissues;
    * draw i's result does not depend on how many draws the ensemble has."""
    coil = figure8_coil(64)
    top = np.array([0.0, 0.0, 90.0])
    site = Placement(top, top + [0, 50, 0])
    homog = Subject(sphere_head(8.0, 90.0, shells=((1.0, 2),), jitter_mm=0.3, seed=2), tolerance=1e-10)
    res = homog.simulate_conductivity_uq(coil, site, ConductivityUQConfig(n_samples=3, seed=1), recovery="raw")
    assert res.perturbed_tags == (2,)
    np.testing.assert_allclose(res.peak_samples, res.peak_samples[0], rtol=1e-7)
    homog.free()

    subj = Subject(sphere_head(6.0, 90.0, jitter_mm=0.3, seed=1), tolerance=1e-8)
    ctx = subj.context
    nominal = nominal_sigma_table()
    c, h = top[None], (top + [0.0, 50.0, 0.0])[None]
    tags = tuple(int(t) for t in np.unique(subj.mesh.tet_tags))
    ctx.sigma_begin(coil, c, h, [4.0], 1e6, nominal, tags, recovery="raw")
    try:
        small = ctx.sigma_draw(nominal[list(tags)] * (1.0 + 1e-4 * np.arange(1, len(tags) + 1)))
    finally:
        ctx.sigma_end()
    assert small["init_relres"][0] < 1e-5, small["init_relres"]

    ctx.sigma_begin(coil, c, h, [4.0], 1e6, nominal, (3,), magnitude=True, recovery="raw")
    try:
        csf = ctx.sigma_draw([2.5])
    finally:
        ctx.sigma_end()
    sigma = nominal.copy()
    sigma[3] = 2.5
    ctx.set_conductivity(sigma, keep_coarse=True)
    ref = ctx.solve_block(coil, c, h, [4.0], 1e6, magnitude=True, recovery="raw")
    ctx.set_conductivity(nominal, keep_coarse=True)
    assert np.linalg.norm(csf["magnE"] - ref["magnE"]) / np.linalg.norm(ref["magnE"]) < 1e-6

    three = subj.simulate_conductivity_uq(coil, site, ConductivityUQConfig(n_samples=3, seed=8), recovery="raw")
    five = subj.simulate_conductivity_uq(coil, site, ConductivityUQConfig(n_samples=5, seed=8), recovery="raw")
    np.testing.assert_array_equal(five.peak_samples[:3], three.peak_samples)
    np.testing.assert_array_equal(five.iteration_samples[:3], three.iteration_samples)
    subj.free()


def test_record_rois_and_depth_probes():
    """Per-draw ROI means (record_rois) are the volume-weighted |E| of the ROI in each draw: their
    ensemble mean is the ROI's weighted mean of the per-element mean field."""
    mesh = sphere_head(6.0, 90.0, jitter_mm=0.3, seed=1)
    coil = figure8_coil(64)
    top = np.array([0.0, 0.0, 90.0])
    site = Placement(top, top + [0, 50, 0])
    subj = Subject(mesh, tolerance=1e-8)
    rois = {"vertex": subj.roi([0.0, 0.0, 72.0], radius_mm=8.0), "one": subj.roi([10.0, 0.0, 70.0])}
    probes = subj.depth_probes([0.0, 0.0, 76.0], [0.0, 0.0, -1.0], [0.0, 10.0, 20.0], radius_mm=5.0)
    assert len(probes) == 3 and len({tuple(p.elem_idx[:3]) for p in probes}) == 3
    with pytest.raises(ValueError, match="non-zero"):
        subj.depth_probes([0.0, 0.0, 76.0], [0.0, 0.0, 0.0], [0.0])
    res = subj.simulate_conductivity_uq(coil, site, ConductivityUQConfig(n_samples=4, seed=6), moments=True,
                                        recovery="raw", record_rois=rois)
    for name, r in rois.items():
        s = res.roi_samples[name]
        assert s.shape == (4,) and (s > 0).all()
        assert s.mean() == pytest.approx(float(res.mean_magnE[r.elem_idx] @ r.weights), rel=1e-9)
    assert set(res.tissue_sensitivity("vertex")) == set(res.perturbed_tags)
    subj.free()


def test_conductivity_draws_match_the_fp64_oracle_with_the_draws_table():
    """Each draw of the study (nominal coarse levels kept, subspace guess) against the FP64 oracle
    assembled and solved from scratch with that draw's conductivity table: gray-matter |E| relative
    L2 and peak |E| within the product's 1e-5."""
    from oracle import Oracle, OracleParams

    mesh = sphere_head(6.0, 90.0, jitter_mm=0.3, seed=2)
    coil = figure8_coil(64)
    top = np.array([0.0, 0.0, 90.0])
    sites = [Placement(top, top + [0, 50, 0]), Placement([20.0, 0.0, 87.7], [20.0, 50.0, 87.7])]
    subj = Subject(mesh, tolerance=1e-10)
    ctx = subj.context
    nominal = nominal_sigma_table()
    tags = tuple(int(t) for t in np.unique(mesh.tet_tags))
    rng = np.random.default_rng(3)
    draws = nominal[list(tags)] * np.exp(0.25 * rng.standard_normal((3, len(tags))))
    c = np.stack([s.center_mm for s in sites])
    h = np.stack([s.handle_mm for s in sites])
    ctx.sigma_begin(coil, c, h, [4.0, 4.0], 1e6, nominal, tags, magnitude=True, recovery="raw")
    try:
        got = [ctx.sigma_draw(d) for d in draws]
    finally:
        ctx.sigma_end()
    gm = subj.mesh.tet_tags == 2
    for d, g in zip(draws, got):
        table = nominal.copy()
        table[list(tags)] = d
        ref = Oracle(mesh, OracleParams(sigma_by_tag=tuple(table))).solve(coil, c, h, [4.0, 4.0], 1e6, tolerance=1e-12)
        for i in range(2):
            a, b = g["magnE"][i].astype(np.float64)[gm], ref["magnE"][i].astype(np.float64)[gm]
            assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-5
            assert abs(g["summary"][i][0] - ref["summary"][i][0]) <= 1e-5 * ref["summary"][i][0]
    subj.free()


def test_draw_guess_modes_agree_and_rank():
    """The draws from the subspace guess, from the nominal potential alone and from zero reach the
    same field to the tolerance; the subspace guess starts closest and needs the fewest iterations."""
    mesh = sphere_head(6.0, 90.0, jitter_mm=0.3, seed=1)
    coil = figure8_coil(64)
    top = np.array([0.0, 0.0, 90.0])
    c = np.stack([top, top + [15.0, 0.0, -1.3]])
    h = c + [0.0, 50.0, 0.0]
    subj = Subject(mesh, tolerance=1e-10)
    ctx = subj.context
    nominal = nominal_sigma_table()
    tags = tuple(int(t) for t in np.unique(mesh.tet_tags))
    draw = nominal[list(tags)] * np.exp(0.25 * np.random.default_rng(8).standard_normal(len(tags)))
    ctx.sigma_begin(coil, c, h, [4.0, 4.0], 1e6, nominal, tags, magnitude=True, recovery="raw")
    out = {}
    try:
        for mode in ("subspace", "nominal", "zero"):
            ctx.sigma_set_guess(mode)
            out[mode] = ctx.sigma_draw(draw)
    finally:
        ctx.sigma_end()
    base = out["zero"]["magnE"].astype(np.float64)
    for mode in ("subspace", "nominal"):
        m = out[mode]["magnE"].astype(np.float64)
        assert np.linalg.norm(m - base) / np.linalg.norm(base) <= 1e-7
    assert (out["subspace"]["init_relres"] < out["nominal"]["init_relres"]).all()
    assert (out["zero"]["init_relres"] == 1.0).all()
    assert out["subspace"]["iterations"].sum() <= out["nominal"]["iterations"].sum() <= out["zero"]["iterations"].sum()
    subj.free()

"""The sweep-setting autotuner on the GPU (cunibs_b200.tune). Needs a B200.

It times block widths and dA/dt overlaps on the caller's placements and keeps the fastest; the
settings it may change leave every result bit as it was.
"""

from __future__ import annotations

import numpy as np
import pytest

from cunibs_b200 import Placement, Subject
from cunibs_b200.synthetic import figure8_coil, sphere_head

pytestmark = pytest.mark.gpu


def test_autotune_picks_a_measured_setting_and_changes_no_result():
    subj = Subject(sphere_head(6.0, 90.0, jitter_mm=0.3, seed=1), tolerance=1e-8)
    coil = figure8_coil(64)
    rng = np.random.default_rng(3)
    sites = []
    for _ in range(8):
        th, ph = rng.uniform(0.0, 0.5), rng.uniform(0.0, 2 * np.pi)
        c = 90.0 * np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
        sites.append(Placement(c, c + [-50.0 * np.sin(ph), 50.0 * np.cos(ph), 0.0]))
    before = [r.magnE for r in subj.iter_simulate(coil, sites, magnitude=True)]
    res = subj.autotune(coil, sites, widths=(2, 4), overlaps=(1, 3), repeats=1)
    assert set(res.placements_per_s) == {(2, 1), (4, 1), (2, 3), (4, 3)}
    assert all(v > 0 for v in res.placements_per_s.values())
    assert res.placements_per_s[(res.block_k, res.overlap_blocks_per_sm)] == max(res.placements_per_s.values())
    assert subj.block_k_default == res.block_k and subj.overlap_blocks_per_sm == res.overlap_blocks_per_sm
    after = [r.magnE for r in subj.iter_simulate(coil, sites, magnitude=True)]
    for a, b in zip(after, before):
        np.testing.assert_array_equal(a, b)
    subj.free()


def test_sweep_sixteen_wide_matches_eight_wide_bitwise():
    """A block_k=None sweep may run 16 placements per block (the native solver's widest), wider
    than an explicit block_k may ask; every result is bitwise the 8-wide sweep's."""
    subj = Subject(sphere_head(6.0, 90.0, jitter_mm=0.3, seed=1), tolerance=1e-8)
    coil = figure8_coil(64)
    rng = np.random.default_rng(5)
    sites = []
    for _ in range(20):
        th, ph = rng.uniform(0.0, 0.5), rng.uniform(0.0, 2 * np.pi)
        c = 90.0 * np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
        sites.append(Placement(c, c + [-50.0 * np.sin(ph), 50.0 * np.cos(ph), 0.0]))
    eight = list(subj.iter_simulate(coil, sites, magnitude=True))
    subj.set_sweep_defaults(block_k=16)
    sixteen = list(subj.iter_simulate(coil, sites, magnitude=True))
    for a, b in zip(sixteen, eight):
        np.testing.assert_array_equal(a.magnE, b.magnE)
        assert a.summary["distribution"] == b.summary["distribution"]
    subj.free()

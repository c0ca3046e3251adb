"""Field parity at the benchmark workloads' full sizes, CUDA path vs the FP64 oracle. Needs a B200.

Two workloads, both seeded synthetic sphere heads:

* the small plain-method case: a 64^3 lattice at 3 mm clipped to r <= 90 mm (679,044 tets), five
  shells, a figure-8 of 2 x 512 z-dipoles 4 mm above the vertex, dI/dt = 1e6, one placement per
  block (block_k = 1), relative residual 1e-10;
* the 1M-tet ten-tissue head (eight shells with an eye and a muscle cap, 2.63 mm lattice, +-0.2 mm
  jitter), a figure-8 of 2 x 2048 dipoles, 8 placements on a 15-degree grid solved as one block
  (block_k = 8) to relative residual 1e-8.

The oracle solves to 1e-12 and stands as the exact discrete solution; the bar is the one stated for
the product: gray-matter |E| relative L2 <= 1e-5 and peak |E| <= 1e-5 relative.
"""

from __future__ import annotations

import numpy as np
import pytest

from cunibs_b200 import Placement, Subject
from cunibs_b200.synthetic import EIGHT_SHELLS, EYE_CAP, FIVE_SHELLS, MUSCLE_CAP, figure8_coil, sphere_head
from oracle import Oracle

pytestmark = pytest.mark.gpu

GM_REL_L2 = 1e-5  # relative L2 of |E| over gray matter (tag 2), GPU vs FP64 oracle
PEAK_REL = 1e-5   # peak |E| relative
ORACLE_TOL = 1e-12


def _gm_errors(res, ref, tags):
    gm = tags == 2
    out = []
    for i, r in enumerate(res):
        a, b = r.magnE.astype(np.float64)[gm], ref["magnE"][i].astype(np.float64)[gm]
        rel = float(np.linalg.norm(a - b) / np.linalg.norm(b))
        peak = float(abs(r.peak_magnE() - ref["summary"][i][0]) / ref["summary"][i][0])
        out.append((rel, peak))
    return out


@pytest.fixture(scope="module")
def small_head():
    return sphere_head(3.0, 90.0, FIVE_SHELLS, cells=64)


@pytest.fixture(scope="module")
def small_oracle(small_head):
    return Oracle(small_head)


@pytest.mark.parametrize("precision", ["plain", "split"])
@pytest.mark.parametrize("recovery", ["raw", "harmonic"])
def test_small_head_single_placement_vs_oracle(small_head, small_oracle, precision, recovery):
    assert small_head.n_tets == 679044
    coil = figure8_coil(512)
    top = np.array([0.0, 0.0, 90.0])
    site = Placement(top, top + [0.0, 50.0, 0.0], distance_mm=4.0)
    subj = Subject(small_head, tolerance=1e-10, precision=precision)
    res = list(subj.iter_simulate(coil, [site], magnitude=True, block_k=1, recovery=recovery))
    ref = small_oracle.solve(coil, site.center_mm[None], site.handle_mm[None], [4.0], 1e6, tolerance=ORACLE_TOL,
                             recovery=recovery)
    assert res[0].relative_residual <= 1e-10
    (rel, peak), = _gm_errors(res, ref, subj.mesh.tet_tags)
    assert rel <= GM_REL_L2, f"GM rel-L2 {rel:.2e}"
    assert peak <= PEAK_REL, f"peak rel {peak:.2e}"
    subj.free()


@pytest.fixture(scope="module")
def head_1m():
    return sphere_head(2.63, 90.0, EIGHT_SHELLS, (EYE_CAP, MUSCLE_CAP), jitter_mm=0.2, seed=0)


def _grid_sites():
    sites = []
    for th, ph in [(0, 0), (15, 0), (15, 90), (15, 180), (15, 270), (30, 45), (30, 135), (30, 225)]:
        t, f = np.radians(th), np.radians(ph)
        c = 90.0 * np.array([np.sin(t) * np.cos(f), np.sin(t) * np.sin(f), np.cos(t)])
        sites.append(Placement(c, c + 50.0 * np.array([-np.sin(f), np.cos(f), 0.0])))
    return sites


@pytest.mark.parametrize("precision", ["split", "mixed"])
def test_1m_head_block_of_8_vs_oracle(head_1m, precision):
    """The benchmark's block (default harmonic recovery) at relative residual 1e-8."""
    assert head_1m.n_tets == 1007532
    coil = figure8_coil(2048)
    sites = _grid_sites()
    subj = Subject(head_1m, tolerance=1e-8, precision=precision)
    res = list(subj.iter_simulate(coil, sites, magnitude=True, block_k=8))
    orc = Oracle(head_1m)
    ref = orc.solve(coil, np.stack([s.center_mm for s in sites]), np.stack([s.handle_mm for s in sites]),
                    [4.0] * 8, 1e6, tolerance=ORACLE_TOL, recovery=res[0].recovery)
    errs = _gm_errors(res, ref, subj.mesh.tet_tags)
    for i, (rel, peak) in enumerate(errs):
        assert rel <= GM_REL_L2, f"placement {i}: GM rel-L2 {rel:.2e}"
        assert peak <= PEAK_REL, f"placement {i}: peak rel {peak:.2e}"
    subj.free()


def test_summary_percentiles_at_full_size_vs_oracle(head_1m):
    """The gray-matter summary (radix-selected percentiles, focality) on the 1M-tet head's ~330k
    gray-matter elements, three fields in one call: continuous values, values rounded to 1/64
    (long runs of ties, kept in element order), and a constant field."""
    from cunibs_b200 import _native
    from oracle import oracle_summary

    m = head_1m
    ctx = _native.Context(m.nodes_mm, m.tet_nodes, m.tet_tags, m.skin_tris)
    orc = Oracle(m)
    rng = np.random.default_rng(9)
    f = np.empty((3, ctx.n_tets), np.float32)
    f[0] = rng.gamma(2.0, 0.3, ctx.n_tets)
    f[1] = np.round(rng.gamma(2.0, 0.3, ctx.n_tets) * 64.0) / 64.0
    f[2] = 0.25
    got = ctx.summary(f)
    vols32 = orc.f64("vols").astype(np.float32)
    bary, tags = orc.f64("bary").reshape(-1, 3), orc.i32("tet_tags")
    for i in range(3):
        want = oracle_summary(f[i], vols32, bary, tags)
        np.testing.assert_allclose(got[i], want, rtol=1e-10, atol=0, err_msg=f"field {i}")
    again = ctx.summary(f)
    np.testing.assert_array_equal(again, got)  # reproducible run to run
    ctx.close()

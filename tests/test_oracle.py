"""The CPU oracle, pinned against the reference's own golden values and known answers.

These run without a GPU. They establish that the restatement in oracle/ reproduces the
reference's published behaviour before any CUDA result is compared with it.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import (
    Oracle,
    oracle_dadt,
    oracle_l1_dinv_f32,
    oracle_select_size4,
    oracle_summary,
    oracle_weighted_quantiles,
)


@pytest.fixture(scope="module")
def patch_oracle(patch_mesh):
    return Oracle(patch_mesh)


def test_patch_fixture_counts(patch_mesh, pins):
    c = pins["patch_counts"]
    assert patch_mesh.n_nodes == c["n_nodes"]
    assert patch_mesh.n_tets == c["n_tets"]
    assert patch_mesh.skin_tris.shape[0] == c["n_skin_tris"]
    tags, counts = np.unique(patch_mesh.tet_tags, return_counts=True)
    assert dict(zip(tags.tolist(), counts.tolist())) == {1: 1781, 2: 5805, 3: 8105, 5: 4122, 7: 13533, 8: 5530, 9: 2263}


def test_patch_hierarchy_sizes_match_reference_pin(patch_oracle, pins):
    """tests/test_solver_kernels.py:615-637 pins [8403, 465] on this fixture."""
    assert patch_oracle.i32("level_sizes").tolist() == pins["patch_hierarchy_sizes"]["value"]


def test_patch_peak_matches_reference_pin(patch_oracle, d70_coil, patch_placement, pins):
    """End-to-end pin of the raw field (tests/test_realmesh.py:115-134)."""
    p = patch_placement
    r = patch_oracle.solve(d70_coil, p.center_mm, p.handle_mm, [p.distance_mm], 1e6, tolerance=1e-10)
    s = r["summary"][0]
    assert s[0] == pytest.approx(pins["patch_peak_magnE_raw"]["value"], rel=pins["patch_peak_magnE_raw"]["rel"])
    np.testing.assert_allclose(s[1:4], pins["patch_peak_location_mm"]["value"], atol=2.0)
    assert r["relative_residual"][0] <= 1e-10


def test_patch_iteration_count_at_reference_tolerance(patch_oracle, d70_coil, patch_placement, pins):
    """The reference documents 11 iterations at rel.res 1e-6 on this patch (test_block_solve.py:284-287)."""
    p = patch_placement
    r = patch_oracle.solve(d70_coil, p.center_mm, p.handle_mm, [p.distance_mm], 1e6, tolerance=1e-6)
    assert int(r["iterations"][0]) == pins["patch_iterations_tol_1e-6"]["value"]


def test_reference_tet_gradients(cube_mesh):
    """tests/test_solver.py:18-31: unit tet in mm -> 1e3/m gradients, (1/6) mm^3 volume."""
    from cunibs_b200.mesh import HeadMesh

    m = HeadMesh([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], [[0, 1, 2, 3]], [2], np.zeros((0, 3), np.int32))
    o = Oracle(m)
    g = o.f64("g").reshape(-1, 4, 3)
    # Morton order may permute the four nodes; undo it to read the gradients per original node.
    perm = o.i32("node_perm")
    tets = o.i32("tet_nodes").reshape(-1, 4)
    orig = perm[tets[0]]
    by_orig = np.empty((4, 3))
    by_orig[orig] = g[0]
    np.testing.assert_allclose(by_orig, [[-1e3, -1e3, -1e3], [1e3, 0, 0], [0, 1e3, 0], [0, 0, 1e3]], atol=1e-9)
    assert o.f64("vols")[0] == pytest.approx(1e-9 / 6)


def test_zero_volume_is_rejected():
    from cunibs_b200.mesh import HeadMesh

    m = HeadMesh([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]], [[0, 1, 2, 3]], [2], np.zeros((0, 3), np.int32))
    with pytest.raises(ValueError, match="volume"):
        Oracle(m)


def test_unknown_tag_is_rejected(cube_mesh):
    from cunibs_b200.mesh import HeadMesh

    m = HeadMesh(cube_mesh.nodes_mm, cube_mesh.tet_nodes, [2, 2, 2, 2, 2, 99], cube_mesh.skin_tris)
    with pytest.raises(ValueError, match="tag"):
        Oracle(m)


def test_stiffness_symmetric_zero_rowsum(patch_oracle):
    ptr, col, val = patch_oracle.i32("stiff_ptr"), patch_oracle.i32("stiff_col"), patch_oracle.f64("stiff_val")
    n = ptr.shape[0] - 1
    rows = np.repeat(np.arange(n), np.diff(ptr))
    a = {(int(r), int(c)): v for r, c, v in zip(rows, col, val)}
    for (r, c), v in list(a.items())[:5000]:
        assert a[(c, r)] == pytest.approx(v, rel=1e-12, abs=1e-18)
    rowsum = np.zeros(n)
    np.add.at(rowsum, rows, val)
    assert np.abs(rowsum).max() <= 1e-12 * np.abs(val).max()


def test_l1_dinv_known_rows():
    """tests/test_solver_kernels.py:518-540 known answer."""
    rows = [[(0, 2.0), (1, -1.0), (3, 0.5)], [(0, -1.0), (1, -4.0), (2, 1.0)], [(2, 0.0)], [], [(0, 3.0), (2, -1.0)]]
    ptr = np.cumsum([0] + [len(r) for r in rows]).astype(np.int32)
    col = np.array([c for r in rows for c, _ in r], np.int32)
    val = np.array([v for r in rows for _, v in r], np.float32)
    np.testing.assert_allclose(oracle_l1_dinv_f32(ptr, col, val), [1 / 3.5, -1 / 6, 1, 1, 0.25], rtol=1e-6)


def test_aggregation_partition_and_determinism(patch_oracle):
    for lev in range(patch_oracle.n_levels):
        agg = patch_oracle.i32("agg", lev)
        nc = patch_oracle.i32("level_sizes")[lev + 1]
        assert agg.min() == 0 and agg.max() == nc - 1
        assert np.unique(agg).size == nc
    a_ptr, a_col, a_val = patch_oracle.i32("a_ptr", 0), patch_oracle.i32("a_col", 0), patch_oracle.f64("a_val", 0)
    first, nc1 = oracle_select_size4(a_ptr, a_col, a_val.astype(np.float32))
    again, nc2 = oracle_select_size4(a_ptr, a_col, a_val.astype(np.float32))
    assert nc1 == nc2
    np.testing.assert_array_equal(first, again)


def test_dadt_matches_closed_form_dipoles():
    """tests/test_solver_kernels.py:389-416 closed form, identity transform."""
    from cunibs_b200.coil import Coil

    rng = np.random.default_rng(7)
    s = rng.uniform(-0.05, 0.05, size=(16, 3))
    m = rng.standard_normal((16, 3))
    r = rng.uniform(0.1, 0.2, size=(40, 3))
    out = oracle_dadt(Coil(s, m), np.eye(4), 1e6, r * 1e3)
    diff = r[:, None, :] - s[None, :, :]
    ref = 1e6 * 1e-7 * (np.cross(m[None], diff) / np.linalg.norm(diff, axis=2)[:, :, None] ** 3).sum(1)
    assert np.linalg.norm(out - ref) / np.linalg.norm(ref) <= 1e-12


def test_weighted_quantiles_hazen_under_uniform_weights():
    """tests/test_metrics.py:89-95."""
    rng = np.random.default_rng(0)
    v = rng.random(1001)
    qs = np.array([0.01, 0.1, 0.5, 0.95, 0.99, 0.999])
    np.testing.assert_allclose(oracle_weighted_quantiles(v, np.ones_like(v), qs), np.quantile(v, qs, method="hazen"), atol=1e-9)


def test_weighted_quantiles_weights_and_scale():
    """tests/test_metrics.py:98-115."""
    light = oracle_weighted_quantiles(np.array([1.0, 2.0]), np.array([1.0, 9.0]), np.array([0.5]))
    heavy = oracle_weighted_quantiles(np.array([1.0, 2.0]), np.array([9.0, 1.0]), np.array([0.5]))
    assert light[0] > 1.8 and heavy[0] < 1.2
    rng = np.random.default_rng(1)
    v, w = rng.random(50), rng.random(50) + 0.1
    qs = np.array([0.25, 0.5, 0.9])
    np.testing.assert_allclose(oracle_weighted_quantiles(v, w, qs), oracle_weighted_quantiles(v, w * 1e6, qs), rtol=1e-12)


def test_summary_center_of_gravity_analytic():
    """tests/test_metrics.py:118-127: equal vol*|E| weights put the CoG at the midpoint."""
    s = oracle_summary(np.array([2.0, 1.0], np.float32), np.array([1.0, 2.0], np.float32),
                       np.array([[0.0, 0, 0], [4.0, 0, 0]]), np.array([2, 2], np.int32))
    np.testing.assert_allclose(s[4:7], [2.0, 0.0, 0.0])
    assert s[0] == 2.0 and s[7] == 3.0


def test_bf16_restatement_matches_torch():
    """The network checker's BF16 rounding (oracle/mlp.py) is round-to-nearest-even, as torch's."""
    import torch

    from oracle.mlp import bf16_round

    rng = np.random.default_rng(0)
    a = rng.standard_normal(10000) * 10.0 ** rng.integers(-5, 5, 10000)
    want = torch.tensor(a, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(bf16_round(a), want)


def test_mlp_restatement_gradients_match_finite_differences():
    """The FP64 network restatement's backward pass against central differences (no BF16 rounding
    in play: weights and inputs already BF16, perturbations along one weight)."""
    from oracle.mlp import bf16_round, forward_backward

    rng = np.random.default_rng(1)
    W = [bf16_round(rng.standard_normal((16, 8)) * 0.5), bf16_round(rng.standard_normal((8, 16)) * 0.3)]
    b = [rng.standard_normal(16) * 0.1, rng.standard_normal(8) * 0.1]
    x = bf16_round(rng.standard_normal((12, 8)))
    t = rng.standard_normal((12, 8))
    _, _, dW, _ = forward_backward(W, b, x, t, 8)
    i, j, h = 3, 2, 1e-6
    Wp = [W[0], W[1].copy()]
    Wm = [W[0], W[1].copy()]
    Wp[1][i, j] += h
    Wm[1][i, j] -= h
    lp, *_ = forward_backward(Wp, b, x, t, 8)
    lm, *_ = forward_backward(Wm, b, x, t, 8)
    assert dW[1][i, j] == pytest.approx((lp - lm) / (2 * h), rel=1e-3)


def test_oracle_conductivity_table_parameter():
    """The oracle's conductivity table: the default table given explicitly changes nothing bit for
    bit; every conductivity scaled by one factor leaves |E| unchanged (it depends on ratios only);
    one tissue changed moves it."""
    from cunibs_b200.fem import TISSUE_CONDUCTIVITY
    from cunibs_b200.synthetic import figure8_coil, sphere_head
    from oracle import Oracle, OracleParams

    mesh = sphere_head(10.0, 90.0, jitter_mm=0.3, seed=1)
    coil = figure8_coil(32)
    c = np.array([[0.0, 0.0, 90.0]])
    h = c + [0.0, 50.0, 0.0]
    table = [0.0] * 11
    for tag, s in TISSUE_CONDUCTIVITY.items():
        table[tag] = s
    base = Oracle(mesh).solve(coil, c, h, [4.0], 1e6, tolerance=1e-12)["magnE"][0].astype(np.float64)
    same = Oracle(mesh, OracleParams(sigma_by_tag=tuple(table))).solve(coil, c, h, [4.0], 1e6, tolerance=1e-12)
    np.testing.assert_array_equal(same["magnE"][0], base)
    scaled = Oracle(mesh, OracleParams(sigma_by_tag=tuple(2.5 * s for s in table))).solve(coil, c, h, [4.0], 1e6,
                                                                                            tolerance=1e-12)
    assert np.linalg.norm(scaled["magnE"][0] - base) / np.linalg.norm(base) <= 1e-8
    bumped = list(table)
    bumped[3] *= 3.0
    moved = Oracle(mesh, OracleParams(sigma_by_tag=tuple(bumped))).solve(coil, c, h, [4.0], 1e6, tolerance=1e-12)
    assert np.linalg.norm(moved["magnE"][0] - base) / np.linalg.norm(base) >= 1e-3

"""CUDA path vs the CPU oracle, through the C ABI. Needs a B200.

Integer stages (Morton layout, CSR pattern, aggregation) must match bit for bit; the setup
stages compiled without FMA contraction (gradients, stiffness, hierarchy operators, placement) must
match exactly too; the field must match the FP64 oracle within the stated tolerances.
"""

from __future__ import annotations

import numpy as np
import pytest

from cunibs_b200 import Placement, Subject, _native
from cunibs_b200.synthetic import figure8_coil, sphere_head
from oracle import Oracle, oracle_dadt, oracle_select_size4, oracle_summary

pytestmark = pytest.mark.gpu

GM_REL_L2 = 1e-5  # relative L2 of |E| over gray matter, GPU vs FP64 oracle
PEAK_REL = 1e-5   # peak |E| relative


@pytest.fixture(scope="module")
def patch_pair(patch_mesh):
    m = patch_mesh
    return _native.Context(m.nodes_mm, m.tet_nodes, m.tet_tags, m.skin_tris), Oracle(m)


@pytest.fixture(scope="module")
def sphere_mesh():
    return sphere_head(6.0, 90.0, jitter_mm=0.3, seed=1)


@pytest.fixture(scope="module")
def sphere_pair(sphere_mesh):
    m = sphere_mesh
    return _native.Context(m.nodes_mm, m.tet_nodes, m.tet_tags, m.skin_tris), Oracle(m)


@pytest.mark.parametrize("which", ["patch_pair", "sphere_pair"])
def test_layout_and_operator_bit_exact(which, request):
    ctx, orc = request.getfixturevalue(which)
    for name in ("node_perm", "tet_perm", "tet_nodes", "tet_tags", "skin_tris", "n2c_ptr", "n2c_idx", "stiff_ptr",
                 "stiff_col"):
        np.testing.assert_array_equal(ctx.array(name), orc.i32(name), err_msg=name)
    for name in ("nodes_mm", "g", "vols", "bary", "stiff_val", "skin_normals"):
        np.testing.assert_array_equal(ctx.array(name), orc.f64(name), err_msg=name)
    assert ctx.ground_node == int(orc.i32("ground")[0])


@pytest.mark.parametrize("which", ["patch_pair", "sphere_pair"])
def test_hierarchy_bit_exact(which, request):
    ctx, orc = request.getfixturevalue(which)
    assert ctx.levels() == orc.i32("level_sizes").tolist()
    for lev in range(ctx.n_levels):
        for name in ("a_ptr", "a_col", "agg", "p_ptr", "p_col"):
            np.testing.assert_array_equal(ctx.array(name, lev), orc.i32(name, lev), err_msg=f"{name}[{lev}]")
        for name in ("a_val", "p_val", "dinv"):
            np.testing.assert_array_equal(ctx.array(name, lev), orc.f64(name, lev), err_msg=f"{name}[{lev}]")
    np.testing.assert_array_equal(ctx.array("coarse_col"), orc.i32("coarse_col"))
    np.testing.assert_array_equal(ctx.array("coarse_val"), orc.f64("coarse_val"))
    inv_g, inv_o = ctx.array("coarse_inv"), orc.f64("coarse_inv")
    assert np.abs(inv_g - inv_o).max() <= 1e-12 * np.abs(inv_o).max()


def test_patch_hierarchy_matches_reference_pin(patch_pair, pins):
    ctx, _ = patch_pair
    assert ctx.levels() == pins["patch_hierarchy_sizes"]["value"]


def test_select_size4_bit_exact_on_level_operators(patch_pair):
    ctx, orc = patch_pair
    ptr, col, val = orc.i32("a_ptr", 0), orc.i32("a_col", 0), orc.f64("a_val", 0).astype(np.float32)
    agg_g, nc_g = _native.select_size4(ptr, col, val)
    agg_o, nc_o = oracle_select_size4(ptr, col, val)
    assert nc_g == nc_o
    np.testing.assert_array_equal(agg_g, agg_o)


@pytest.fixture(scope="module")
def sphere_ref_cycle(sphere_mesh):
    """A context whose V-cycle descends to the coarsest level, as the reference's does."""
    m = sphere_mesh
    p = _native.default_params()
    p.dense_max_rows = 0
    ctx = _native.Context(m.nodes_mm, m.tet_nodes, m.tet_tags, m.skin_tris, p)
    yield ctx
    ctx.close()


@pytest.mark.parametrize("fp32,tol", [(False, 1e-11), (True, 2e-5)])
def test_vcycle_matches_oracle(sphere_ref_cycle, sphere_pair, fp32, tol):
    ctx, orc = sphere_ref_cycle, sphere_pair[1]
    assert ctx.vcycle_levels == ctx.n_levels and ctx.bottom_rows == ctx.coarse_rows
    rng = np.random.default_rng(0)
    r = rng.standard_normal((ctx.n_nodes - 1, 4))
    z_g = ctx.vcycle(r, fp32=fp32)
    z_o = orc.vcycle(r)
    for c in range(4):
        assert np.linalg.norm(z_g[:, c] - z_o[:, c]) / np.linalg.norm(z_o[:, c]) <= tol


def test_dense_bottom_vcycle_is_a_symmetric_preconditioner(sphere_pair, sphere_ref_cycle):
    """The default V-cycle stops at the first level below the finest with at most 12,288 rows and
    solves it exactly: the preconditioner stays symmetric positive definite (FP64), and PCG with it
    needs no more iterations than with the full descent."""
    ctx = sphere_pair[0]
    assert 1 <= ctx.vcycle_levels < ctx.n_levels and ctx.bottom_rows <= 12288
    rng = np.random.default_rng(3)
    r = rng.standard_normal((ctx.n_nodes - 1, 2))
    z = ctx.vcycle(r)
    assert abs(r[:, 0] @ z[:, 1] - r[:, 1] @ z[:, 0]) <= 1e-10 * abs(r[:, 0] @ z[:, 1])
    assert (np.einsum("ij,ij->j", r, z) > 0).all()
    B = rng.standard_normal((ctx.n_nodes - 1, 4))
    _, it_dense, rel = ctx.solve(B, 4, 4, tolerance=1e-10, max_iters=500)
    _, it_full, _ = sphere_ref_cycle.solve(B, 4, 4, tolerance=1e-10, max_iters=500)
    assert (rel <= 1e-10).all() and (it_dense <= it_full).all()


def test_placement_matches_oracle(patch_pair, patch_placement):
    ctx, orc = patch_pair
    p = patch_placement
    centers = np.stack([p.center_mm, p.center_mm + [3.0, -2.0, 0.0]])
    handles = centers + [0.0, 50.0, 0.0]
    T_g, deg_g = ctx.place(centers, handles, [4.0, 6.0])
    T_o, deg_o = orc.place(centers, handles, [4.0, 6.0])
    np.testing.assert_array_equal(T_g, T_o)
    np.testing.assert_array_equal(deg_g, deg_o)
    # A handle straight along the outward normal leaves the frame undefined.
    normal = -T_g[0, :3, 2]
    proj = T_g[0, :3, 3] - 4.0 * normal
    _, deg = ctx.place(centers[:1], (proj + 30 * normal)[None], [4.0])
    assert deg[0] == 1


@pytest.mark.parametrize("general", [False, True])
def test_dadt_matches_fp64_oracle(patch_pair, d70_coil, patch_placement, general):
    """Both dipole paths: the D70's z-moments (coil-frame path) and a tilted copy (general path)."""
    from cunibs_b200.coil import Coil

    ctx, orc = patch_pair
    p = patch_placement
    coil = d70_coil
    if general:
        c, s_ = np.cos(0.3), np.sin(0.3)
        rot = np.array([[c, 0, s_], [0, 1, 0], [-s_, 0, c]])
        coil = Coil(d70_coil.positions_m, d70_coil.moments @ rot.T)
    T, _ = ctx.place(np.stack([p.center_mm, p.center_mm + [4.0, 0, 0]]), np.stack([p.handle_mm, p.handle_mm + [4.0, 0, 0]]),
                     [p.distance_mm, 6.0])
    got = ctx.dadt(coil, T, 1e6).astype(np.float64)
    for i in range(2):
        want = oracle_dadt(coil, T[i], 1e6, ctx.array("nodes_mm").reshape(-1, 3))
        assert np.linalg.norm(got[i] - want) / np.linalg.norm(want) <= 2e-6
        assert np.abs(got[i] - want).max() <= 1e-5 * np.abs(want).max()


@pytest.mark.parametrize("precision", [_native.PREC_PLAIN_FP64, _native.PREC_MIXED, _native.PREC_SPLIT])
def test_linear_solve_matches_oracle_direct(sphere_pair, precision):
    ctx, orc = sphere_pair
    n = ctx.n_nodes - 1
    rng = np.random.default_rng(5)
    B = rng.standard_normal((n, 4))
    X, it, rel = ctx.solve(B, 4, 4, precision=precision, tolerance=1e-10, max_iters=500)
    assert (rel <= 1e-10).all() and (it > 0).all()
    # Residual in FP64 against the oracle's assembled operator.
    ptr, col, val = orc.i32("a_ptr", 0), orc.i32("a_col", 0), orc.f64("a_val", 0)
    rows = np.repeat(np.arange(n), np.diff(ptr))
    for c in range(4):
        ax = np.zeros(n)
        np.add.at(ax, rows, val * X[col, c])
        assert np.linalg.norm(B[:, c] - ax) / np.linalg.norm(B[:, c]) <= 2e-10


def _compare_block(subject, orc, coil, sites, tol=1e-10, recovery="raw"):
    res = list(subject.iter_simulate(coil, sites, magnitude=True, block_k=8, recovery=recovery))
    ref = orc.solve(coil, np.stack([s.center_mm for s in sites]), np.stack([s.handle_mm for s in sites]),
                    [s.distance_mm for s in sites], 1e6, tolerance=tol, recovery=recovery)
    tags = subject.mesh.tet_tags
    gm = tags == 2
    for i, r in enumerate(res):
        a, b = r.magnE.astype(np.float64)[gm], ref["magnE"][i].astype(np.float64)[gm]
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert rel <= GM_REL_L2, f"placement {i}: GM rel-L2 {rel:.2e}"
        assert abs(r.peak_magnE() - ref["summary"][i][0]) <= PEAK_REL * ref["summary"][i][0]
        np.testing.assert_allclose(r.transform, ref["transform"][i], rtol=0, atol=1e-12)
    return res, ref


@pytest.mark.parametrize("precision", ["mixed", "split", "plain"])
def test_patch_end_to_end_vs_oracle_and_reference_pin(patch_mesh, d70_coil, patch_placement, pins, precision):
    subj = Subject(patch_mesh, tolerance=1e-10, precision=precision)
    orc = Oracle(patch_mesh)
    p = patch_placement
    sites = [p, Placement(p.center_mm + [5.0, 3.0, -1.0], p.handle_mm + [5.0, 3.0, -1.0])]
    res, _ = _compare_block(subj, orc, d70_coil, sites)
    pin = pins["patch_peak_magnE_raw"]
    assert res[0].peak_magnE() == pytest.approx(pin["value"], rel=pin["rel"])
    np.testing.assert_allclose(res[0].peak_location_mm(), pins["patch_peak_location_mm"]["value"], atol=2.0)
    subj.free()


def test_sphere_block_vs_oracle(sphere_mesh):
    subj = Subject(sphere_mesh, tolerance=1e-10)
    coil = figure8_coil(128)
    sites = []
    for th, ph in [(0, 0), (15, 0), (15, 90), (30, 180), (30, 270)]:
        t, f = np.radians(th), np.radians(ph)
        c = 90 * np.array([np.sin(t) * np.cos(f), np.sin(t) * np.sin(f), np.cos(t)])
        sites.append(Placement(c, c + 50 * np.array([-np.sin(f), np.cos(f), 0.0])))
    _compare_block(subj, Oracle(sphere_mesh), coil, sites)
    subj.free()


@pytest.mark.parametrize("recovery,precision", [("raw", "mixed"), ("harmonic", "mixed"), ("spr_tissue", "mixed"),
                                                ("harmonic", "split")])
def test_block_width_and_batch_invariance_bitwise(sphere_mesh, recovery, precision):
    """A placement's result is bitwise independent of block_k and of its block-mates."""
    subj = Subject(sphere_mesh, tolerance=1e-8, precision=precision)
    coil = figure8_coil(64)
    top = np.array([0.0, 0.0, 90.0])
    sites = [Placement(top + [dx, 0, 0], top + [dx, 50, 0]) for dx in (0.0, 10.0, -12.0)]
    kw = dict(magnitude=True, recovery=recovery)
    runs = {bk: list(subj.iter_simulate(coil, sites, potential=True, block_k=bk, **kw)) for bk in (1, 2, 4, 8)}
    for bk in (2, 4, 8):
        for i in range(3):
            np.testing.assert_array_equal(runs[bk][i].magnE, runs[1][i].magnE)
            np.testing.assert_array_equal(runs[bk][i].v, runs[1][i].v)
            assert runs[bk][i].summary["peak_magnE"] == runs[1][i].summary["peak_magnE"]
    alone = subj.simulate(coil, sites[2], **kw)
    np.testing.assert_array_equal(alone.magnE, runs[8][2].magnE)
    again = list(subj.iter_simulate(coil, sites, block_k=8, **kw))
    for i in range(3):
        np.testing.assert_array_equal(again[i].magnE, runs[8][i].magnE)
    subj.free()


def test_gpu_summary_matches_oracle_summary(sphere_pair):
    ctx, orc = sphere_pair
    rng = np.random.default_rng(2)
    m = rng.gamma(2.0, 0.3, size=(2, ctx.n_tets)).astype(np.float32)
    m[1, :50] = m[1].max()  # ties at the top
    got = ctx.summary(m)
    vols32 = orc.f64("vols").astype(np.float32)
    for i in range(2):
        want = oracle_summary(m[i], vols32, orc.f64("bary").reshape(-1, 3), orc.i32("tet_tags"))
        np.testing.assert_allclose(got[i], want, rtol=1e-10, atol=0)


def test_invalid_inputs_raise(sphere_mesh):
    subj = Subject(sphere_mesh)
    coil = figure8_coil(16)
    top = np.array([0.0, 0.0, 90.0])
    with pytest.raises(ValueError, match="zero right-hand side"):
        subj.simulate(coil, Placement(top, top + [0, 50, 0]), didt=0.0)
    T, _ = subj.context.place(top[None], (top + [0, 50, 0])[None], [4.0])
    normal = -T[0, :3, 2]
    proj = T[0, :3, 3] - 4.0 * normal
    with pytest.raises(ValueError, match="degenerate"):
        subj.simulate(coil, Placement(top, proj + 30.0 * normal))
    subj.free()
    with pytest.raises(ValueError, match="volume"):
        from cunibs_b200.mesh import HeadMesh

        bad = HeadMesh([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]], [[0, 1, 2, 3]], [2], [[0, 1, 2]])
        _native.Context(bad.nodes_mm, bad.tet_nodes, bad.tet_tags, bad.skin_tris)


def test_conductivity_resetup_scale_invariance(sphere_mesh):
    """cunibs_context_set_conductivity (the per-sample step of a conductivity Monte Carlo): E depends
    on conductivity ratios only, so scaling every tissue leaves the field unchanged, while changing
    one tissue changes it; the default table restores the original field."""
    from cunibs_b200.fem import TISSUE_CONDUCTIVITY

    subj = Subject(sphere_mesh, tolerance=1e-10, precision="plain")
    coil = figure8_coil(64)
    top = np.array([0.0, 0.0, 90.0])
    site = Placement(top, top + [0, 50, 0])
    base = subj.simulate(coil, site, magnitude=True, recovery="raw").magnE.astype(np.float64)
    sigma = np.zeros(11)
    for tag, s in TISSUE_CONDUCTIVITY.items():
        sigma[tag] = s
    gm = subj.mesh.tet_tags == 2

    def rel(a):
        return np.linalg.norm(a[gm] - base[gm]) / np.linalg.norm(base[gm])

    subj.context.set_conductivity(2.5 * sigma)
    assert rel(subj.simulate(coil, site, magnitude=True, recovery="raw").magnE.astype(np.float64)) <= 1e-6
    bumped = sigma.copy()
    bumped[3] *= 3.0  # CSF
    subj.context.set_conductivity(bumped)
    assert rel(subj.simulate(coil, site, magnitude=True, recovery="raw").magnE.astype(np.float64)) >= 1e-3
    subj.context.set_conductivity(sigma)
    assert rel(subj.simulate(coil, site, magnitude=True, recovery="raw").magnE.astype(np.float64)) <= 1e-6
    subj.free()


def test_conductivity_keep_coarse_matches_full_resetup(sphere_mesh):
    """cunibs_context_set_conductivity_keep_coarse (finest level refreshed, coarse levels kept)
    solves the same operator as a full re-setup: the fields agree to the solve tolerance, at a
    modest iteration cost, and the nominal table restores the original field."""
    from cunibs_b200.fem import TISSUE_CONDUCTIVITY

    sigma = np.zeros(11)
    for tag, s in TISSUE_CONDUCTIVITY.items():
        sigma[tag] = s
    rng = np.random.default_rng(11)
    draw = sigma.copy()
    draw[1:] *= np.exp(0.25 * rng.standard_normal(10))  # lognormal, log-sd 0.25
    coil = figure8_coil(64)
    top = np.array([0.0, 0.0, 90.0])
    sites = [Placement(top, top + [0, 50, 0]), Placement([30.0, 0, 84.8], [30.0, 50, 84.8])]
    full = Subject(sphere_mesh, tolerance=1e-10)
    kept = Subject(sphere_mesh, tolerance=1e-10)
    base = [r.magnE.astype(np.float64) for r in kept.iter_simulate(coil, sites, magnitude=True, recovery="raw")]
    full.context.set_conductivity(draw)
    kept.context.set_conductivity(draw, keep_coarse=True)
    gm = full.mesh.tet_tags == 2
    a = list(full.iter_simulate(coil, sites, magnitude=True, recovery="raw"))
    b = list(kept.iter_simulate(coil, sites, magnitude=True, recovery="raw"))
    for ra, rb, r0 in zip(a, b, base):
        x, y = ra.magnE.astype(np.float64)[gm], rb.magnE.astype(np.float64)[gm]
        assert np.linalg.norm(x - y) / np.linalg.norm(x) <= 1e-7
        assert np.linalg.norm(x - r0[gm]) / np.linalg.norm(r0[gm]) >= 1e-3  # the draw changed the field
        assert rb.iterations <= 2 * ra.iterations
    kept.context.set_conductivity(sigma, keep_coarse=True)
    back = [r.magnE.astype(np.float64) for r in kept.iter_simulate(coil, sites, magnitude=True, recovery="raw")]
    for r, r0 in zip(back, base):
        assert np.linalg.norm(r[gm] - r0[gm]) / np.linalg.norm(r0[gm]) <= 1e-7
    full.free()
    kept.free()


def test_hierarchy_rebuild_and_plain_solve_are_bit_reproducible(sphere_mesh):
    """A full re-setup at unchanged conductivities rebuilds the same hierarchy bit for bit, and a
    plain FP64 block solve gives the same field before it, twice in a row, and after it."""
    from cunibs_b200.fem import TISSUE_CONDUCTIVITY

    m = sphere_mesh
    p = _native.default_params()
    p.precision = _native.PREC_PLAIN_FP64
    p.tolerance = 1e-8
    ctx = _native.Context(m.nodes_mm, m.tet_nodes, m.tet_tags, m.skin_tris, p)
    coil = figure8_coil(64)
    c = np.array([[0.0, 0.0, 90.0], [10.0, 0.0, 89.4]])
    h = c + [0.0, 50.0, 0.0]

    def arrays():
        out = {}
        for lev in range(ctx.n_levels):
            for name in ("a_val", "p_val", "dinv", "a_col", "agg"):
                out[(name, lev)] = ctx.array(name, lev).copy()
        return out

    def field():
        return ctx.solve_block(coil, c, h, [4.0, 4.0], 1e6, magnitude=True, recovery="harmonic")["magnE"].copy()

    before, f0, f1 = arrays(), field(), field()
    np.testing.assert_array_equal(f1, f0)
    sigma = np.zeros(11)
    for tag, s in TISSUE_CONDUCTIVITY.items():
        sigma[tag] = s
    ctx.set_conductivity(sigma)  # full rebuild at the same values
    after = arrays()
    for key in before:
        np.testing.assert_array_equal(after[key], before[key], err_msg=str(key))
    np.testing.assert_array_equal(field(), f0)
    ctx.close()


@pytest.mark.parametrize("precision", ["split", "plain"])
def test_per_call_tolerance_is_honoured_by_the_cached_loop_graph(sphere_mesh, precision):
    """The PCG loop is captured once per block width and replayed; each call's own tolerance must
    still govern it: loose, then tight, then loose again on one context, each stopping at its own."""
    subj = Subject(sphere_mesh, tolerance=1e-8, precision=precision)
    ctx = subj.context
    coil = figure8_coil(64)
    c = np.array([[0.0, 0.0, 90.0], [10.0, 0.0, 89.4]])
    h = c + [0.0, 50.0, 0.0]
    runs = {}
    for tol in (1e-3, 1e-11, 1e-3):
        r = ctx.solve_block(coil, c, h, [4.0, 4.0], 1e6, tolerance=tol, max_iters=500)
        assert (r["relative_residual"] <= tol).all(), (tol, r["relative_residual"])
        runs.setdefault(tol, []).append(r["iterations"].copy())
    loose, tight = runs[1e-3][0], runs[1e-11][0]
    assert (tight > loose + 5).all()
    np.testing.assert_array_equal(runs[1e-3][1], loose)
    subj.free()

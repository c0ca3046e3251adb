"""Field recovery on the GPU vs the CPU oracle, through the C ABI. Needs a B200.

The recovery operators (slots, patches, boundary marks, rungs, FP32 weights) must match the oracle
bit for bit, and so must the apply kernels given the same inputs; the end-to-end recovered field
must match the FP64 oracle within the field tolerances, and the default (harmonic) path must hit
the reference's pinned peak on its head patch (tests/test_realmesh.py:25,137-141).
"""

from __future__ import annotations

import numpy as np
import pytest

from cunibs_b200 import Placement, Subject, _native
from cunibs_b200.synthetic import figure8_coil, sphere_head
from oracle import Oracle

pytestmark = pytest.mark.gpu

MODES = ("spr_global", "spr_tissue", "harmonic")
GM_REL_L2 = 1e-5
PEAK_REL = 1e-5


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


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("which", ["patch_pair", "sphere_pair"])
def test_operator_bit_exact(which, mode, request):
    ctx, orc = request.getfixturevalue(which)
    g = ctx.recovery(mode)
    o = orc.recovery(mode)
    assert (g["n_slots"], g["n_fallback"], g["n_undetermined"]) == (o["n_slots"], o["n_fallback"], o["n_undetermined"])
    for name in ("ptr", "idx", "slot_of_corner", "slot_node", "slot_tag", "status", "is_boundary"):
        np.testing.assert_array_equal(ctx.recovery_array(mode, name), o[name], err_msg=name)
    wg, wo = ctx.recovery_array(mode, "w"), o["w"]
    assert wg.shape == wo.shape
    np.testing.assert_array_equal(wg.view(np.uint32), wo.view(np.uint32))


@pytest.mark.parametrize("mode", MODES)
def test_apply_bit_exact(sphere_pair, mode):
    """The apply kernels against the oracle's mirror of their arithmetic, on the same inputs."""
    ctx, orc = sphere_pair
    rng = np.random.default_rng(7)
    k = 3
    if mode == "harmonic":
        x = orc.f64("nodes_mm").reshape(-1, 3) * 1e-3
        v = np.stack([np.sin(40 * x[:, 0] + c) * x[:, 1] + 3.0 * x[:, 2] for c in range(k)])
        v += 1e-6 * rng.standard_normal(v.shape)
        v[:, ctx.ground_node] = 0.0
        dadt = rng.standard_normal((k, ctx.n_nodes, 3)).astype(np.float32)
        got = ctx.recover(mode, v=v, dadt_nodes=dadt)
        want = orc.recovery_apply(mode, v=v, dadt_nodes=dadt)
    else:
        e = rng.standard_normal((k, ctx.n_tets, 3)).astype(np.float32)
        got = ctx.recover(mode, elements=e)
        want = orc.recovery_apply(mode, elements=e)
    for a, b, name in zip(got, want, ("E_slots", "E", "magnE")):
        np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32), err_msg=name)


def _compare_block(subject, orc, coil, sites, recovery, tol=1e-10):
    res = list(subject.iter_simulate(coil, sites, magnitude=True, block_k=8, recovery=recovery))
    ref = orc.solve(coil, np.stack([s.center_mm for s in sites]), np.stack([s.handle_mm for s in sites]),
                    [s.distance_mm for s in sites], 1e6, tolerance=tol, recovery=recovery)
    gm = subject.mesh.tet_tags == 2
    for i, r in enumerate(res):
        assert r.recovery == recovery
        a, b = r.magnE.astype(np.float64)[gm], ref["magnE"][i].astype(np.float64)[gm]
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert rel <= GM_REL_L2, f"placement {i}: GM rel-L2 {rel:.2e}"
        assert abs(r.peak_magnE() - ref["summary"][i][0]) <= PEAK_REL * ref["summary"][i][0]
    return res, ref


@pytest.mark.parametrize("precision", ["mixed", "plain"])
def test_patch_default_recovery_vs_oracle_and_reference_pin(patch_mesh, d70_coil, patch_placement, pins, precision):
    subj = Subject(patch_mesh, tolerance=1e-10, precision=precision)
    p = patch_placement
    default = subj.simulate(d70_coil, p, magnitude=True)
    assert default.recovery == "harmonic"
    pin = pins["patch_peak_magnE_harmonic"]
    assert default.peak_magnE() == pytest.approx(pin["value"], rel=pin["rel"])
    sites = [p, Placement(p.center_mm + [5.0, 3.0, -1.0], p.handle_mm + [5.0, 3.0, -1.0])]
    res, _ = _compare_block(subj, Oracle(patch_mesh), d70_coil, sites, "harmonic")
    np.testing.assert_array_equal(res[0].magnE, default.magnE)
    subj.free()


@pytest.mark.parametrize("mode", ["spr_global", "spr_tissue"])
def test_sphere_spr_vs_oracle(sphere_mesh, mode):
    subj = Subject(sphere_mesh, tolerance=1e-10)
    coil = figure8_coil(128)
    top = np.array([0.0, 0.0, 90.0])
    sites = [Placement(top, top + [0, 50, 0]), Placement([30.0, 0, 84.8], [30.0, 50, 84.8])]
    _compare_block(subj, Oracle(sphere_mesh), coil, sites, mode)
    subj.free()


def test_recovery_lowers_or_keeps_the_peak(patch_mesh, d70_coil, patch_placement):
    subj = Subject(patch_mesh, tolerance=1e-8)
    raw = subj.simulate(d70_coil, patch_placement, recovery="raw").peak_magnE()
    for mode in MODES:
        assert 0 < subj.simulate(d70_coil, patch_placement, recovery=mode).peak_magnE() <= raw
    subj.free()


def test_nodal_field(patch_mesh, d70_coil, patch_placement, tmp_path):
    """FieldResult.nodal_field (reference simulation.py:709-747) on the recovered slots."""
    subj = Subject(patch_mesh, tolerance=1e-8)
    r = subj.simulate(d70_coil, patch_placement, nodal=True, magnitude=True)
    assert r.E_slots.shape == (subj.recovery_operator("harmonic")["n_slots"], 3)
    nf = r.nodal_field("gray_matter")
    assert nf.shape == (subj.mesh.n_nodes, 3)
    gm_slots = r.slot_tag == 2
    np.testing.assert_array_equal(nf[r.slot_node[gm_slots]], r.E_slots[gm_slots])
    assert np.isnan(nf).any(axis=1).sum() == subj.mesh.n_nodes - np.unique(r.slot_node[gm_slots]).size
    with pytest.raises(ValueError, match="ambiguous"):
        r.nodal_field("all")
    r.save(tmp_path / "r.npz")
    back = type(r).load(tmp_path / "r.npz")
    np.testing.assert_array_equal(back.nodal_field("gray_matter"), nf)
    g = subj.simulate(d70_coil, patch_placement, nodal=True, recovery="spr_global")
    assert g.nodal_field("all").shape == (subj.mesh.n_nodes, 3)
    assert not np.isnan(g.nodal_field("all")).any()
    with pytest.raises(ValueError, match="nodal=True needs a recovery mode"):
        subj.simulate(d70_coil, patch_placement, nodal=True, recovery="raw")
    subj.free()


def test_gpu_field_matches_the_closed_form_sphere():
    """The GPU path (default harmonic recovery, mixed precision) on a 678k-tet five-shell sphere
    against the closed-form field (oracle/analytic_sphere.py): measured 0.027 GM relative L2."""
    from oracle.analytic_sphere import head_frame_dipoles, sphere_efield

    mesh = sphere_head(3.0, 90.0, jitter_mm=0.0, seed=0)
    subj = Subject(mesh, tolerance=1e-8)
    coil = figure8_coil(256)
    top = np.array([0.0, 0.0, 90.0])
    r = subj.simulate(coil, Placement(top, top + [0, 50, 0]), vectors=True)
    pos, mom = head_frame_dipoles(coil, r.transform)
    ordered = subj.mesh
    gm = ordered.tet_tags == 2
    bary = ordered.tet_barycenters_mm[gm] * 1e-3
    Ea = sphere_efield(bary, pos, mom)
    Ef = r.E[gm].astype(np.float64)
    assert np.linalg.norm(Ef - Ea) / np.linalg.norm(Ea) <= 0.05
    subj.free()

"""Field recovery in the CPU oracle, pinned against the reference's golden value and the properties
its own recovery tests hold (tests/test_recovery.py, tests/test_realmesh.py:137-141).

No GPU: these establish that the restatement reproduces the reference before the CUDA operator is
compared with it bit for bit.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import Oracle

MODES = ("spr_global", "spr_tissue", "harmonic")


@pytest.fixture(scope="module")
def patch_oracle(patch_mesh):
    return Oracle(patch_mesh)


@pytest.fixture(scope="module")
def sphere_oracle(small_sphere):
    return Oracle(small_sphere)


def _solve(orc, coil, placement, recovery, tol=1e-10):
    p = placement
    return orc.solve(coil, p.center_mm, p.handle_mm, [p.distance_mm], 1e6, tolerance=tol, recovery=recovery)


def test_harmonic_peak_matches_reference_pin(patch_oracle, d70_coil, patch_placement, pins):
    """The default path's end-to-end pin (tests/test_realmesh.py:25,137-141)."""
    pin = pins["patch_peak_magnE_harmonic"]
    r = _solve(patch_oracle, d70_coil, patch_placement, "harmonic")
    assert r["summary"][0][0] == pytest.approx(pin["value"], rel=pin["rel"])


@pytest.mark.parametrize("mode", MODES)
def test_recovery_does_not_raise_the_peak(patch_oracle, d70_coil, patch_placement, mode):
    """tests/test_recovery.py:1089-1100: smoothing never reports a higher gray-matter peak than raw."""
    raw = _solve(patch_oracle, d70_coil, patch_placement, "raw")["summary"][0][0]
    rec = _solve(patch_oracle, d70_coil, patch_placement, mode)["summary"][0][0]
    assert 0 < rec <= raw


@pytest.mark.parametrize("mode", ["spr_global", "spr_tissue"])
def test_spr_weights_are_a_partition_of_unity(patch_oracle, mode):
    """tests/test_recovery.py:72-81."""
    op = patch_oracle.recovery(mode)
    sums = np.add.reduceat(op["w"].astype(np.float64), op["ptr"][:-1])
    np.testing.assert_allclose(sums, 1.0, atol=1e-6)


@pytest.mark.parametrize("mode", ["spr_global", "spr_tissue"])
def test_spr_reproduces_a_linear_field(sphere_oracle, mode):
    """tests/test_recovery.py:84-110: a field linear in space is recovered exactly where the fit ran."""
    orc = sphere_oracle
    op = orc.recovery(mode)
    nodes = orc.f64("nodes_mm").reshape(-1, 3)
    bary = orc.f64("bary").reshape(-1, 3)
    slope = np.array([[0.3, -0.2, 0.1], [0.05, 0.4, -0.1], [-0.2, 0.1, 0.25]])
    offset = np.array([1.0, -2.0, 0.5])
    elements = (offset + bary @ slope.T).astype(np.float32)
    slots, _, _ = orc.recovery_apply(mode, elements=elements[None])
    fitted = ~op["is_boundary"][op["slot_node"]].astype(bool)
    want = offset + nodes[op["slot_node"][fitted]] @ slope.T
    scale = np.abs(want).max()
    np.testing.assert_allclose(slots[0][fitted], want, atol=1e-5 * scale)


def test_spr_boundary_nodes_take_the_volume_average(patch_oracle):
    """tests/test_recovery.py:128-144."""
    op = patch_oracle.recovery("spr_global")
    vols = patch_oracle.f64("vols").astype(np.float32).astype(np.float64)
    ptr, idx, w = op["ptr"], op["idx"], op["w"]
    for node in np.flatnonzero(op["is_boundary"])[:200]:
        seg = slice(ptr[node], ptr[node + 1])
        v = vols[idx[seg] >> 2]
        np.testing.assert_allclose(w[seg], v / v.sum(), rtol=1e-6)


def test_outer_boundary_covers_the_skin(patch_oracle, patch_mesh):
    """tests/test_recovery.py:237-246: every scalp node is on the outer boundary."""
    op = patch_oracle.recovery("spr_global")
    skin = np.unique(patch_oracle.i32("skin_tris"))
    assert op["is_boundary"][skin].all()


def test_tissue_boundary_contains_the_outer_boundary(patch_oracle):
    """tests/test_recovery.py:462-474, plus every node carrying two tissues."""
    outer = patch_oracle.recovery("spr_global")["is_boundary"].astype(bool)
    tissue = patch_oracle.recovery("spr_tissue")
    tb = tissue["is_boundary"].astype(bool)
    assert (tb | ~outer).all()
    sn = tissue["slot_node"]
    mixed = np.unique(sn[1:][sn[1:] == sn[:-1]])
    assert tb[mixed].all()
    assert (tb & ~outer).sum() == mixed.size - (outer[mixed]).sum()


def test_tissue_slots_split_each_node_by_tissue(patch_oracle):
    """tests/test_recovery.py:370-393."""
    op = patch_oracle.recovery("spr_tissue")
    tets = patch_oracle.i32("tet_nodes")
    tags = np.repeat(patch_oracle.i32("tet_tags"), 4)
    soc = op["slot_of_corner"]
    assert np.array_equal(op["slot_node"][soc], tets)
    assert np.array_equal(op["slot_tag"][soc], tags)
    key = op["slot_node"].astype(np.int64) * 16 + op["slot_tag"]
    assert (np.diff(key) > 0).all()


def test_spr_tissue_equals_spr_global_on_a_single_tissue_mesh(single_tissue_ball):
    """tests/test_recovery.py:396-439: with one tag the two modes are the same operator."""
    orc = Oracle(single_tissue_ball)
    g = orc.recovery("spr_global")
    t = orc.recovery("spr_tissue")
    assert np.array_equal(g["ptr"], t["ptr"]) and np.array_equal(g["idx"], t["idx"])
    assert np.array_equal(g["w"], t["w"])


def test_harmonic_ladder_covers_every_slot(patch_oracle):
    """tests/test_recovery.py:733-762: every slot takes a rung; on the head patch nearly all the cubic."""
    op = patch_oracle.recovery("harmonic")
    st = op["status"]
    assert st.shape[0] == op["n_slots"] and set(np.unique(st)) <= {0, 1, 2, 3}
    assert op["n_fallback"] == int((st >= 2).sum()) and op["n_undetermined"] == int((st == 3).sum()) == 0
    assert (st == 0).mean() > 0.9


def test_harmonic_patches_hold_their_first_ring(patch_oracle):
    """A patch is sorted, distinct, holds its own node and is at least the 16-node floor where the
    same-tissue component allows (recovery.py:246-312)."""
    op = patch_oracle.recovery("harmonic")
    ptr, idx = op["ptr"], op["idx"]
    sizes = np.diff(ptr)
    for s in range(0, op["n_slots"], 97):
        seg = idx[ptr[s] : ptr[s + 1]]
        assert (np.diff(seg) > 0).all()
        assert op["slot_node"][s] in seg
    assert np.median(sizes) >= 16


def test_harmonic_reproduces_its_own_fit_space(sphere_oracle):
    """tests/test_recovery.py:664-690: a harmonic cubic potential is differentiated exactly on
    cubic-rung slots; with dA/dt = 0 the recovered E is -grad v."""
    orc = sphere_oracle
    op = orc.recovery("harmonic")
    x = orc.f64("nodes_mm").reshape(-1, 3) * 1e-3
    u, v, t = x[:, 0], x[:, 1], x[:, 2]
    pot = u * v * t + 2.0 * (u * u - v * v) + 0.5 * t * (2 * t * t - 3 * u * u - 3 * v * v) + 3.0 * u
    grad = np.stack([v * t + 4 * u - 3 * t * u + 3.0, u * t - 4 * v - 3 * t * v,
                     u * v + 3 * t * t - 1.5 * (u * u + v * v)], axis=1)
    slots, _, _ = orc.recovery_apply("harmonic", v=pot[None], dadt_nodes=np.zeros((1, x.shape[0], 3), np.float32))
    cubic = op["status"] == 0
    want = -grad[op["slot_node"][cubic]]
    np.testing.assert_allclose(slots[0][cubic], want, rtol=1e-4, atol=1e-4 * np.abs(want).max())


def test_harmonic_adds_dadt_exactly_at_the_nodes(sphere_oracle):
    """tests/test_recovery.py:715-730: with v = 0 the recovered field is exactly -dA/dt(node)."""
    orc = sphere_oracle
    op = orc.recovery("harmonic")
    n = orc.n_nodes
    rng = np.random.default_rng(3)
    dadt = rng.standard_normal((1, n, 3)).astype(np.float32)
    slots, _, _ = orc.recovery_apply("harmonic", v=np.zeros((1, n)), dadt_nodes=dadt)
    assert np.array_equal(slots[0], -dadt[0][op["slot_node"]])


def test_harmonic_weights_cannot_amplify(patch_oracle):
    """tests/test_recovery.py:788-805: h * max_c sum_p |w_pc| <= 50 on every accepted rung."""
    op = patch_oracle.recovery("harmonic")
    x = patch_oracle.f64("nodes_mm").reshape(-1, 3) * 1e-3
    ptr, idx, w = op["ptr"], op["idx"], op["w"].astype(np.float64)
    for s in range(0, op["n_slots"], 13):
        if op["status"][s] == 3:
            continue
        seg = slice(ptr[s], ptr[s + 1])
        h = np.abs(x[idx[seg]] - x[op["slot_node"][s]]).max()
        assert h * np.abs(w[seg]).sum(axis=0).max() <= 50.0 * (1 + 1e-5)


def test_recovery_operator_is_reproducible(patch_mesh):
    """tests/test_recovery.py:147-154: two builds give the same bits."""
    a = Oracle(patch_mesh).recovery("harmonic")
    b = Oracle(patch_mesh).recovery("harmonic")
    for key in ("ptr", "idx", "status"):
        assert np.array_equal(a[key], b[key])
    assert np.array_equal(a["w"].view(np.uint32), b["w"].view(np.uint32))

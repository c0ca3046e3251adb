"""Auxiliary dipole method on the GPU (cunibs_b200.adm, cunibs_adm_*). Needs a B200.

The self-consistent ladder of the reference's tests (test_adm.py): every layer is checked against
the forward solve or the layer below it, on a multi-tissue sphere.
  1. The adjoint functional J_d = sum_n W_n . dA/dt_n equals dir . E of the forward solve.
  2. Q evaluated exactly at the placed dipoles gives J to FP32 N-body accuracy; Q on a grid gives
     it to the interpolation error, which falls as the grid refines.
  3. The optimiser's optimum is what a forward solve at that placement gives, and the closed-form
     rotation agrees with a brute-force angle sweep.
"""

from __future__ import annotations

import numpy as np
import pytest

from cunibs_b200 import Placement, Subject, adm
from cunibs_b200.synthetic import figure8_coil, sphere_head

pytestmark = pytest.mark.gpu

TOP = np.array([0.0, 0.0, 90.0])
HANDLE = TOP + [0.0, 50.0, 0.0]
DIST = 4.0
DIDT = 1e6


@pytest.fixture(scope="module")
def setup():
    mesh = sphere_head(6.0, 90.0, jitter_mm=0.3, seed=1)
    subj = Subject(mesh, tolerance=1e-10)
    coil = figure8_coil(64)
    ctx = subj.context
    res = ctx.solve_block(coil, TOP[None], HANDLE[None], [DIST], DIDT, vectors=True, magnitude=True, recovery="raw")
    dadt = ctx.dadt(coil, res["transform"], DIDT)[0]
    tags = ctx.array("tet_tags")
    bary = ctx.array("bary").reshape(-1, 3)
    gm = np.flatnonzero(tags == 2)
    tgt = int(gm[np.argmax(res["magnE"][0][gm])])
    yield subj, coil, res, dadt, tgt, bary
    subj.free()


@pytest.fixture(scope="module")
def recip(setup):
    subj, coil, _, _, tgt, bary = setup
    return adm.build_reciprocity(subj, coil, adm.Target(bary[tgt]), TOP[None])


def test_adjoint_functional_matches_forward_directional(setup):
    subj, _, res, dadt, tgt, bary = setup
    E = res["E"][0][tgt].astype(np.float64)
    for direction in ([1, 0, 0], [0, 0, 1], [0.3, -0.7, 0.6]):
        rt = adm.resolve_target(subj, adm.Target(bary[tgt], direction))
        assert rt.elem_idx.tolist() == [tgt] and not rt.magnitude
        adj = adm.solve_adjoint(subj, rt)
        assert adj.relative_residual[0] <= adm.ADJOINT_TOLERANCE and adj.iterations[0] > 0
        j = float(adm.exact_functional(adj.node_weights, dadt)[0])
        ehat = np.asarray(direction, float) / np.linalg.norm(direction)
        assert j == pytest.approx(float(E @ ehat), rel=1e-4, abs=1e-5 * np.linalg.norm(E))


def test_adjoint_functional_magnitude_recovers_the_field_vector(setup):
    subj, _, res, dadt, tgt, bary = setup
    rt = adm.resolve_target(subj, adm.Target(bary[tgt]))
    assert rt.magnitude and rt.directions.shape == (3, 3)
    adj = adm.solve_adjoint(subj, rt)
    j = adm.exact_functional(adj.node_weights, dadt)
    E = res["E"][0][tgt].astype(np.float64)
    np.testing.assert_allclose(j, E, rtol=1e-4, atol=1e-5 * np.linalg.norm(E))


def test_qfield_exact_and_grid_interpolation_converge_to_the_functional(setup):
    subj, coil, _, dadt, tgt, bary = setup
    adj = adm.solve_adjoint(subj, adm.resolve_target(subj, adm.Target(bary[tgt])))
    j = adm.exact_functional(adj.node_weights, dadt)
    pl = Placement(TOP, HANDLE, DIST)
    errors = []
    for spacing in (4.0, 2.0, 1.0):
        grid = adm.grid_for_placements(subj, coil, [pl], spacing_mm=spacing, margin_mm=8.0)
        exact = adm.evaluate_exact(adj, coil, pl, DIDT, center_m=grid.center_m)
        np.testing.assert_allclose(exact, j, rtol=1e-3, atol=1e-3 * np.linalg.norm(j))
        approx = adm.evaluate(adm.sample_qfield(adj, grid), coil, pl, DIDT)
        errors.append(float(np.linalg.norm(approx - exact) / np.linalg.norm(exact)))
    assert errors[0] > errors[1] > errors[2], errors
    assert errors[1] <= 5e-3 and errors[2] <= 3e-3, errors


def test_qfield_directions_from_one_pass_equal_each_direction_alone(setup):
    """A magnitude target's three Q fields come from one pass over the sources, each pair's
    geometry shared by the directions; each equals the field of its direction's target alone,
    bitwise where the two adjoints' node weights are bitwise equal."""
    subj, coil, _, _, tgt, bary = setup
    grid = adm.grid_for_placements(subj, coil, [Placement(TOP, HANDLE, DIST)], spacing_mm=4.0, margin_mm=8.0)
    mag = adm.solve_adjoint(subj, adm.resolve_target(subj, adm.Target(bary[tgt])))
    assert np.array_equal(mag.target.directions, np.eye(3))
    w3, q3 = mag.node_weights, adm.sample_qfield(mag, grid).q
    assert q3.shape == (3, *grid.shape, 3) and np.isfinite(q3).all()
    for d in range(3):
        one = adm.solve_adjoint(subj, adm.resolve_target(subj, adm.Target(bary[tgt], np.eye(3)[d])))
        w1, q1 = one.node_weights, adm.sample_qfield(one, grid).q
        np.testing.assert_allclose(w1[0], w3[d], rtol=1e-9, atol=1e-12 * np.abs(w3[d]).max())
        if np.array_equal(w1[0], w3[d]):
            np.testing.assert_array_equal(q1[0], q3[d])
        else:
            np.testing.assert_allclose(q1[0], q3[d], rtol=1e-5, atol=1e-6 * np.abs(q3[d]).max())


def test_optimum_matches_a_forward_solve_there(setup):
    subj, coil, res, _, tgt, bary = setup
    T = res["transform"][0]
    x0, y0 = T[:3, 0], T[:3, 1]
    centers = np.array([TOP + dx * x0 + dy * y0 for dx in (-10, 0, 10) for dy in (-10, 0, 10)])
    result = adm.optimize(subj, coil, adm.Target(bary[tgt]), centers)
    assert result.center_objective.shape == (9,)
    assert result.best_objective == pytest.approx(float(result.center_objective.max()), rel=1e-12)
    fwd = subj.context.solve_block(coil, result.best_center_mm[None], result.best_handle_mm[None], [DIST], DIDT,
                                   vectors=True, recovery="raw")
    assert result.best_objective == pytest.approx(float(np.linalg.norm(fwd["E"][0][tgt])), rel=5e-3)


def test_closed_form_rotation_matches_a_brute_force_sweep(setup, recip):
    _, coil, res, _, _, _ = setup
    result = adm.optimize_placement(recip, coil, TOP[None], n_samples=17)
    T = res["transform"][0]
    x0, y0 = T[:3, 0], T[:3, 1]
    proj = result.best_center_mm
    angles = np.linspace(0, 2 * np.pi, 720, endpoint=False)
    sweep = [Placement(proj, proj + 50 * (np.cos(a) * y0 + np.sin(a) * x0), DIST) for a in angles]
    brute = np.linalg.norm(adm.evaluate(recip, coil, sweep, DIDT), axis=1)
    assert result.best_objective == pytest.approx(float(brute.max()), rel=5e-3)


def test_evaluate_contracts(setup, recip):
    subj, coil, _, _, _, _ = setup
    pls = [Placement(TOP, HANDLE, 4.0), Placement(TOP + [5.0, -5.0, 0.0], TOP + [45.0, 50.0, 0.0], 4.0),
           Placement(TOP + [-5.0, 5.0, 0.0], TOP + [-40.0, 50.0, 0.0], 6.0)]
    batched = adm.evaluate(recip, coil, pls, DIDT)
    assert batched.shape == (3, 3)
    for i, pl in enumerate(pls):  # one block per placement: the batch changes nothing
        np.testing.assert_array_equal(batched[i], adm.evaluate(recip, coil, pl, DIDT))
    T, _ = subj.context.place(np.stack([p.center_mm for p in pls]), np.stack([p.handle_mm for p in pls]),
                              [p.distance_mm for p in pls])
    np.testing.assert_array_equal(adm.evaluate_frames(recip, coil, T, DIDT), batched)
    np.testing.assert_array_equal(adm.evaluate(recip, coil, pls[0], 2e6), 2.0 * batched[0])
    lifted = T[:1].copy()
    lifted[0, :3, 3] -= 6.0 * T[0, :3, 2]  # 6 mm further out along the scalp normal
    assert np.linalg.norm(adm.evaluate_frames(recip, coil, lifted, DIDT)) < np.linalg.norm(batched[0])
    far = Placement(TOP, HANDLE, 200.0)
    with pytest.raises(ValueError, match="outside the reciprocity grid"):
        adm.evaluate(recip, coil, far, DIDT)
    with pytest.raises(ValueError, match=r"sample 2 of 3"):
        adm.evaluate(recip, coil, [pls[0], pls[0], far], DIDT)
    q = recip.q
    assert q.shape == (3, *recip.grid.shape, 3) and np.isfinite(q).all()


def test_resolve_target(setup):
    subj, _, _, _, _, bary = setup
    ctx = subj.context
    tags = ctx.array("tet_tags")
    vols = ctx.array("vols")
    gm = np.flatnonzero(tags == 2)
    point = np.array([10.0, 20.0, 75.0])
    rt = adm.resolve_target(subj, adm.Target(point))
    assert rt.elem_idx.tolist() == [int(gm[np.argmin(np.linalg.norm(bary[gm] - point, axis=1))])]
    np.testing.assert_array_equal(rt.weights, [1.0])
    inside = bary[rt.elem_idx[0]]  # a gray-matter barycentre: the ball around it holds its neighbours
    rt = adm.resolve_target(subj, adm.Target(inside, radius_mm=8.0))
    assert rt.elem_idx.size > 1 and (tags[rt.elem_idx] == 2).all()
    np.testing.assert_allclose(rt.weights, vols[rt.elem_idx] / vols[rt.elem_idx].sum(), rtol=1e-14)
    np.testing.assert_allclose(rt.barycenter_mm, rt.weights @ bary[rt.elem_idx], rtol=1e-12)
    tiny = adm.resolve_target(subj, adm.Target(point, radius_mm=1e-6))
    assert tiny.elem_idx.tolist() == adm.resolve_target(subj, adm.Target(point)).elem_idx.tolist()
    with pytest.raises(ValueError, match="contains no elements"):
        adm.resolve_target(subj, adm.Target(point, region="eye_balls"))


def test_coverage_grid_holds_the_coil_at_every_rotation(setup):
    subj, coil, _, _, tgt, bary = setup
    centers = np.array([TOP, [20.0, 0.0, 87.7], [0.0, -20.0, 87.7]])
    recip = adm.build_reciprocity(subj, coil, adm.Target(bary[tgt]), centers)
    T, _ = subj.context.place(centers, None, np.full(3, DIST))
    u, v = T[:, :3, 0], T[:, :3, 1]
    for a in np.radians(np.arange(0.0, 360.0, 15.0)):
        handles = centers + 50.0 * (np.cos(a) * v + np.sin(a) * u)
        e = adm.evaluate(recip, coil, [Placement(c, hd, DIST) for c, hd in zip(centers, handles)], DIDT)
        assert np.isfinite(e).all()

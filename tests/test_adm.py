"""Host logic of the auxiliary dipole method (cunibs_b200.adm): targets, grids, the angle search.

The GPU ladder (adjoint functional against forward solves, the Q reformulation and its grid,
the optimiser against forward solves and a brute-force sweep) is tests/test_gpu_adm.py.
"""

from __future__ import annotations

import numpy as np
import pytest

from cunibs_b200 import adm


def test_target_direction_is_normalised_and_copied():
    d = np.array([0.0, 0.0, -7.5])
    t = adm.Target([0, 0, 0], d)
    np.testing.assert_allclose(t.direction, [0.0, 0.0, -1.0])
    assert not np.shares_memory(t.direction, d)
    assert adm.Target([1, 2, 3]).direction is None


def test_target_rejects_zero_direction_and_bad_points():
    with pytest.raises(ValueError, match="non-zero"):
        adm.Target([0, 0, 0], [0.0, 0.0, 0.0])
    with pytest.raises(ValueError, match="3-vector"):
        adm.Target([0, 0], None)


def test_build_grid_covers_the_points_with_margin():
    pts = np.array([[0.0, 0.0, 0.0], [0.01, 0.02, 0.005]])
    g = adm.build_grid(pts, spacing_mm=2.0, margin_mm=8.0)
    np.testing.assert_allclose(g.origin_m, [-0.008, -0.008, -0.008])
    assert g.shape == (int(np.ceil(0.026 / 0.002)) + 1, int(np.ceil(0.036 / 0.002)) + 1, int(np.ceil(0.021 / 0.002)) + 1)
    assert (g.upper_m >= pts.max(0) + 0.008 - 1e-12).all()
    p = g.points_m()
    assert p.shape == (g.n_points, 3)
    # C order, x slowest: the flat index (ix * ny + iy) * nz + iz.
    ix, iy, iz = 2, 3, 4
    np.testing.assert_allclose(p[(ix * g.shape[1] + iy) * g.shape[2] + iz], g.origin_m + g.spacing_m * [ix, iy, iz])
    np.testing.assert_allclose(g.world_to_index(p[[0, -1]]).T, [[0, 0, 0], g.max_index], atol=1e-9)


def test_fourier_kernel_reproduces_band_limited_functions():
    n = 9
    theta_s = np.linspace(0.0, 2 * np.pi, n, endpoint=False)
    theta_f = np.linspace(0.0, 2 * np.pi, 512, endpoint=False)
    f = lambda t: 0.3 + np.cos(t) - 0.4 * np.sin(2 * t) + 0.2 * np.cos(4 * t + 0.3)  # noqa: E731  degree 4
    got = adm.fourier_kernel(theta_f, theta_s, n) @ f(theta_s)
    np.testing.assert_allclose(got, f(theta_f), atol=1e-12)


def test_parabolic_refine_finds_the_vertex():
    thetas = np.linspace(0.0, 2 * np.pi, 64, endpoint=False)
    true = thetas[10] + 0.3 * (thetas[1] - thetas[0])
    obj = -((thetas - true) ** 2)[None]
    got = adm._parabolic_refine(obj, np.argmax(obj, axis=1), thetas)
    assert got[0] == pytest.approx(true, abs=1e-12)


def test_inplane_basis_is_orthonormal_for_any_normal():
    rng = np.random.default_rng(0)
    n = rng.standard_normal((50, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    n[0] = [0.0, 0.0, 1.0]
    u, v = adm._inplane_basis(n)
    for a, b in ((u, v), (u, n), (v, n)):
        np.testing.assert_allclose((a * b).sum(1), 0.0, atol=1e-12)
    np.testing.assert_allclose(np.linalg.norm(u, axis=1), 1.0)
    np.testing.assert_allclose(np.linalg.norm(v, axis=1), 1.0)


def test_exact_functional_is_the_weighted_sum():
    rng = np.random.default_rng(1)
    w = rng.standard_normal((3, 20, 3))
    d = rng.standard_normal((20, 3)).astype(np.float32)
    np.testing.assert_allclose(adm.exact_functional(w, d), (w * d.astype(np.float64)).sum((1, 2)))


def test_optimize_placement_rejects_even_n_samples():
    with pytest.raises(ValueError, match="odd"):
        adm.optimize_placement(None, None, np.zeros((1, 3)), n_samples=8)

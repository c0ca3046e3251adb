"""The conductivity study's per-placement coefficient map (cunibs_sigma_coefficients, host only)
against the NumPy restatement of the reference's draw guess (oracle/sigma_guess.py).

The study never forms the reference's orthonormal basis W: it keeps the sensitivities S and maps a
draw's conductivity change to subspace coefficients through the pseudo-inverse of S^T A S, which
is the same A-Galerkin correction S G^+ S^T r0 = W E^-1 W^T r0 whenever W spans the columns of S.
"""

from __future__ import annotations

import numpy as np
import pytest

from cunibs_b200 import _native
from oracle.sigma_guess import galerkin_correction


def _system(n=80, p=4, seed=0):
    rng = np.random.default_rng(seed)
    m = rng.standard_normal((n, n))
    a = m @ m.T + n * np.eye(n)
    c = rng.standard_normal((n, p))
    sens = np.linalg.solve(a, c)
    sens = sens * (1.0 + 1e-3 * rng.standard_normal(sens.shape))  # a loose sensitivity solve
    dsig = rng.uniform(-0.3, 0.3, p)
    return a, c, sens, dsig


def _study_correction(a, c, sens, dsig, active=None):
    p = sens.shape[1]
    active = np.ones(p, np.int32) if active is None else np.asarray(active, np.int32)
    z, rank = _native.sigma_coefficients(sens.T @ a @ sens, sens.T @ c, active)
    return sens @ (z @ dsig), rank


def test_full_rank_matches_the_reference_correction():
    a, c, sens, dsig = _system()
    mine, rank = _study_correction(a, c, sens, dsig)
    ref = galerkin_correction(a, sens, c @ dsig)
    assert rank == 4
    np.testing.assert_allclose(mine, ref, rtol=1e-9, atol=1e-12 * np.abs(ref).max())


def test_exact_sensitivities_give_the_first_order_solution():
    a, c, _, dsig = _system(seed=1)
    sens = np.linalg.solve(a, c)
    mine, _ = _study_correction(a, c, sens, dsig)
    np.testing.assert_allclose(mine, sens @ dsig, rtol=1e-9, atol=1e-13)


def test_collinear_sensitivities_are_dropped_like_the_reference():
    a, c, sens, dsig = _system(seed=2)
    sens[:, 3] = 2.0 * sens[:, 1]
    c[:, 3] = 2.0 * c[:, 1]
    mine, rank = _study_correction(a, c, sens, dsig)
    ref = galerkin_correction(a, sens, c @ dsig)
    assert rank == 3
    np.testing.assert_allclose(mine, ref, rtol=1e-8, atol=1e-12 * np.abs(ref).max())


def test_a_tissue_without_sensitivity_contributes_nothing():
    a, c, sens, dsig = _system(seed=3)
    c[:, 2] = 0.0
    sens[:, 2] = 0.0
    mine, rank = _study_correction(a, c, sens, dsig, active=[1, 1, 0, 1])
    ref = galerkin_correction(a, sens, c @ dsig)
    assert rank == 3
    np.testing.assert_allclose(mine, ref, rtol=1e-9, atol=1e-12 * np.abs(ref).max())


def test_a_small_but_independent_sensitivity_keeps_its_direction():
    a, c, sens, dsig = _system(seed=4)
    sens[:, 0] *= 1e-6
    c[:, 0] *= 1e-6
    mine, rank = _study_correction(a, c, sens, dsig)
    ref = galerkin_correction(a, sens, c @ dsig)
    assert rank == 4
    np.testing.assert_allclose(mine, ref, rtol=1e-8, atol=1e-12 * np.abs(ref).max())


def test_no_active_tissue_and_bad_arguments():
    z, rank = _native.sigma_coefficients(np.eye(2), np.eye(2), [0, 0])
    assert rank == 0 and not z.any()
    with pytest.raises(ValueError):
        _native.sigma_coefficients(np.eye(2), np.eye(2), [1, 1], rtol=2.0)

"""The V-cycle's dense bottom at a level of a few thousand rows, through the C ABI. Needs a B200.

On a 3.5 mm sphere head (77k nodes) the hierarchy is 77,326 -> ~4,300 -> ...; the default V-cycle
smooths the finest level and solves level 1 exactly with its dense inverse. The inverse is built by
the blocked sweep (many 64-row pivot blocks) and applied by the streaming product (several column
blocks and row splits), so these checks cover the paths a 1M-tet head takes.
"""

from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp

from cunibs_b200 import _native
from cunibs_b200.synthetic import EIGHT_SHELLS, EYE_CAP, MUSCLE_CAP, sphere_head

pytestmark = pytest.mark.gpu

CHEBY_LOWER_RATIO = 12.0


@pytest.fixture(scope="module")
def mid_ctx():
    m = sphere_head(3.5, 90.0, EIGHT_SHELLS, (EYE_CAP, MUSCLE_CAP), jitter_mm=0.2, seed=0)
    ctx = _native.Context(m.nodes_mm, m.tet_nodes, m.tet_tags, m.skin_tris)
    yield ctx
    ctx.close()


def _csr(ctx, prefix, level, ncol=None):
    ptr, col, val = ctx.array(f"{prefix}_ptr", level), ctx.array(f"{prefix}_col", level), ctx.array(f"{prefix}_val", level)
    n = ptr.shape[0] - 1
    return sp.csr_matrix((val, col, ptr), shape=(n, ncol if ncol is not None else n))


def _cheby(A, dinv, b, x0=None):
    """The V-cycle's Chebyshev smoother on [lambda_max / 12, lambda_max], lambda_max = 1 for the l1
    scaling, degree 2: from zero when x0 is None (first step alpha0 D b), else from x0."""
    hi, lo = 1.0, 1.0 / CHEBY_LOWER_RATIO
    theta, delta = 0.5 * (hi + lo), 0.5 * (hi - lo)
    sigma = theta / delta
    alpha0 = 1.0 / theta
    rho = 1.0 / sigma
    rho_n = 1.0 / (2.0 * sigma - rho)
    c_cur, c_prev, alpha = 1.0 + rho_n * rho, -rho_n * rho, 2.0 * rho_n / delta
    D = dinv[:, None]
    if x0 is None:
        prev, cur = np.zeros_like(b), alpha0 * D * b
        c_p = 0.0
    else:
        prev, cur = x0, x0 + alpha0 * D * (b - A @ x0)
        c_p = c_prev
    return c_cur * cur + c_p * prev + alpha * D * (b - A @ cur)


def test_level_one_is_solved_by_its_dense_inverse(mid_ctx):
    ctx = mid_ctx
    sizes = ctx.levels()
    assert ctx.vcycle_levels == 1 and ctx.bottom_rows == sizes[1] and 2048 < sizes[1] <= 12288
    n1 = ctx.bottom_rows
    inv = ctx.array("bottom_inv").reshape(n1, n1)
    A1 = _csr(ctx, "a", 1)
    np.testing.assert_array_equal(inv, inv.T)  # stored from one triangle
    resid = A1 @ inv - np.eye(n1)
    assert np.abs(resid).max() <= 1e-9


def test_dense_bottom_vcycle_matches_two_level_cycle(mid_ctx):
    """z = post-smooth(x + P A1^-1 P^T (b - A0 x)) with x the pre-smoothed iterate, in FP64 to 1e-10
    and through the FP32 V-cycle (FP32 operators and inverse) to 2e-5."""
    ctx = mid_ctx
    A0 = _csr(ctx, "a", 0)
    P = _csr(ctx, "p", 0, ncol=ctx.bottom_rows)
    dinv = ctx.array("dinv", 0)
    n1 = ctx.bottom_rows
    inv = ctx.array("bottom_inv").reshape(n1, n1)
    rng = np.random.default_rng(5)
    b = rng.standard_normal((A0.shape[0], 4))
    x = _cheby(A0, dinv, b)
    x = x + P @ (inv @ (P.T @ (b - A0 @ x)))
    z_ref = _cheby(A0, dinv, b, x)
    for fp32, tol in ((False, 1e-10), (True, 2e-5)):
        z = ctx.vcycle(b, fp32=fp32)
        for c in range(b.shape[1]):
            assert np.linalg.norm(z[:, c] - z_ref[:, c]) / np.linalg.norm(z_ref[:, c]) <= tol, (fp32, c)


@pytest.mark.parametrize("fp32", [False, True])
def test_dense_bottom_vcycle_is_block_width_independent(mid_ctx, fp32):
    """A column's V-cycle output is bitwise the same alone and in blocks of 2, 8 and 16: the dense
    product's order of additions depends on the level's size and the GPU only."""
    ctx = mid_ctx
    rng = np.random.default_rng(7)
    b = rng.standard_normal((ctx.n_nodes - 1, 16))
    z16 = ctx.vcycle(b, fp32=fp32)
    z8 = ctx.vcycle(np.ascontiguousarray(b[:, :8]), fp32=fp32)
    z2 = ctx.vcycle(np.ascontiguousarray(b[:, 3:5]), fp32=fp32)
    z1 = ctx.vcycle(np.ascontiguousarray(b[:, 4]), fp32=fp32)
    np.testing.assert_array_equal(z8, z16[:, :8])
    np.testing.assert_array_equal(z2, z16[:, 3:5])
    np.testing.assert_array_equal(z1, z16[:, 4])

"""Lanes that carry 2 or 4 adjacent columns (the *_cols kernels of solve.cu, the harmonic recovery's
pair kernel). Needs a B200.

Such a lane adds each column's terms in the same order as a lane that carries one, so the results
must be bitwise those of the one-column kernels (CUNIBS_LANE_COLUMNS=1), for every precision and
block width.
"""

from __future__ import annotations

import numpy as np
import pytest

from cunibs_b200 import _native
from cunibs_b200.synthetic import figure8_coil, sphere_head

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def head():
    return sphere_head(5.0, 90.0, jitter_mm=0.3, seed=4)


def _ctx(m, lanes, monkeypatch):
    monkeypatch.setenv("CUNIBS_LANE_COLUMNS", str(lanes))
    ctx = _native.Context(m.nodes_mm, m.tet_nodes, m.tet_tags, m.skin_tris)
    monkeypatch.delenv("CUNIBS_LANE_COLUMNS", raising=False)
    return ctx


@pytest.mark.parametrize("lanes", [2, 4])
@pytest.mark.parametrize("precision", [_native.PREC_SPLIT, _native.PREC_PLAIN_FP64, _native.PREC_MIXED])
@pytest.mark.parametrize("k", [2, 5, 8, 16])
def test_column_lanes_bitwise_equal_one_column(head, precision, k, lanes, monkeypatch):
    rng = np.random.default_rng(k)
    th = rng.uniform(0.0, 0.6, k)
    ph = rng.uniform(0.0, 2 * np.pi, k)
    c = 90.0 * np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], axis=1)
    h = c + np.stack([-np.sin(ph), np.cos(ph), np.zeros(k)], axis=1) * 50.0
    d = np.full(k, 4.0)
    coil = figure8_coil(128)
    one = _ctx(head, 1, monkeypatch)
    two = _ctx(head, lanes, monkeypatch)
    try:
        kw = dict(magnitude=True, potential=True, recovery="harmonic", precision=precision, tolerance=1e-9)
        # The right-hand side and the recovery read the switch at each call, the solver at its build.
        monkeypatch.setenv("CUNIBS_LANE_COLUMNS", "1")
        a = one.solve_block(coil, c, h, d, 1e6, **kw)
        monkeypatch.setenv("CUNIBS_LANE_COLUMNS", str(lanes))
        b = two.solve_block(coil, c, h, d, 1e6, **kw)
        monkeypatch.delenv("CUNIBS_LANE_COLUMNS")
        for key in ("magnE", "v", "summary", "iterations", "relative_residual"):
            np.testing.assert_array_equal(a[key], b[key], err_msg=key)
    finally:
        one.close()
        two.close()

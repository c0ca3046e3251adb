"""The coil field table (cunibs_context_set_coil_table). Needs a B200.

The table samples the coil's dipole sum once per coil in its own frame and interpolates it at the
nodes deeper than the near depth; the rest keep the dipole sum. The block results must match the
dipole sum everywhere (fem/placement.py:279-317) to about 1e-7, follow a change of coil, fall back to
the dipole sum when the build check fails, and stay independent of the block they are solved in.
"""

from __future__ import annotations

import numpy as np
import pytest

from cunibs_b200 import Placement, Subject, _native
from cunibs_b200.coil import Coil
from cunibs_b200.synthetic import figure8_coil, sphere_head

pytestmark = pytest.mark.gpu

KW = dict(vectors=True, magnitude=True, potential=True, recovery="raw", tolerance=1e-10)


@pytest.fixture(scope="module")
def head():
    return sphere_head(4.0, 90.0, jitter_mm=0.3, seed=3)


def _block(k=4, seed=0, radius=90.0):
    rng = np.random.default_rng(seed)
    th = rng.uniform(0.0, 0.7, k)
    ph = rng.uniform(0.0, 2 * np.pi, k)
    c = radius * np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], axis=1)
    h = c + np.stack([-np.sin(ph), np.cos(ph), np.zeros(k)], axis=1) * 50.0
    return c, h, np.full(k, 4.0)


def _ctx(m, table=True, **kw):
    ctx = _native.Context(m.nodes_mm, m.tet_nodes, m.tet_tags, m.skin_tris)
    ctx.set_coil_table(table, **kw)
    return ctx


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _tilted_coil(n=256):
    """A figure-8 whose moments lean off the coil's z axis: the general (three-component) table."""
    base = figure8_coil(n)
    mom = base.moments.copy()
    mom[:, 0] = 0.3 * mom[:, 2]
    mom[:, 1] = -0.2 * mom[:, 2]
    return Coil(positions_m=base.positions_m, moments=np.ascontiguousarray(mom), name="tilted")


@pytest.mark.parametrize("coil_kind", ["z", "general"])
def test_table_matches_the_dipole_sum(head, coil_kind):
    coil = figure8_coil(1024) if coil_kind == "z" else _tilted_coil(512)
    blk = _block()
    direct = _ctx(head, table=False)
    table = _ctx(head, table=True)
    try:
        want = direct.solve_block(coil, *blk, 1e6, **KW)
        got = table.solve_block(coil, *blk, 1e6, **KW)
        info = table.coil_table_info()
        assert info["in_use"] and info["builds"] == 1
        assert info["check_rel_l2"] < 2e-6
        # Most nodes read the table; the near ones (within 15 mm of the coil) are a small share.
        assert 0 < info["last_near_nodes"] < 0.2 * info["last_node_placements"]
        assert direct.coil_table_info()["last_near_nodes"] == -1
        for p in range(blk[0].shape[0]):
            assert _rel(got["E"][p], want["E"][p]) < 1e-6, p
            assert _rel(got["magnE"][p], want["magnE"][p]) < 1e-6, p
            e = np.abs(got["E"][p] - want["E"][p]).max()
            assert e < 1e-5 * np.abs(want["E"][p]).max(), p
        np.testing.assert_allclose(got["summary"][:, 0], want["summary"][:, 0], rtol=1e-5)
    finally:
        direct.close()
        table.close()


def test_every_node_near_takes_the_split_dipole_sum(head):
    """A near depth beyond the head lists every node: the eight-warp split sum alone."""
    coil = figure8_coil(512)
    blk = _block(k=3, seed=5)
    direct = _ctx(head, table=False)
    near = _ctx(head, table=True, near_mm=400.0)
    try:
        want = direct.solve_block(coil, *blk, 1e6, **KW)
        got = near.solve_block(coil, *blk, 1e6, **KW)
        info = near.coil_table_info()
        if info["in_use"]:
            assert info["last_near_nodes"] == info["last_node_placements"]
        for p in range(3):
            assert _rel(got["E"][p], want["E"][p]) < 1e-6, p
    finally:
        direct.close()
        near.close()


def test_failed_check_falls_back_to_the_dipole_sum_bitwise(head):
    """A table too coarse to pass its build check is not used: the result is the dipole sum's."""
    coil = figure8_coil(256)
    blk = _block(k=2, seed=7)
    direct = _ctx(head, table=False)
    coarse = _ctx(head, table=True, step=0.5)
    try:
        want = direct.solve_block(coil, *blk, 1e6, **KW)
        got = coarse.solve_block(coil, *blk, 1e6, **KW)
        info = coarse.coil_table_info()
        assert info["builds"] == 1 and not info["in_use"]
        assert info["check_rel_l2"] > 2e-6
        assert info["last_near_nodes"] == -1
        for key in ("E", "magnE", "v", "summary"):
            np.testing.assert_array_equal(got[key], want[key], err_msg=key)
    finally:
        direct.close()
        coarse.close()


def test_table_follows_the_coil(head):
    a, b = figure8_coil(256), figure8_coil(384)
    shifted = Coil(positions_m=a.positions_m + np.array([0.0, 0.0, -0.002]), moments=a.moments, name="shifted")
    blk = _block(k=2, seed=9)
    ctx = _ctx(head)
    ref = _ctx(head)
    try:
        first = ctx.solve_block(a, *blk, 1e6, **KW)
        ctx.solve_block(a, *blk, 1e6, **KW)
        assert ctx.coil_table_info()["builds"] == 1
        ctx.solve_block(b, *blk, 1e6, **KW)
        assert ctx.coil_table_info()["builds"] == 2
        moved = ctx.solve_block(shifted, *blk, 1e6, **KW)
        assert ctx.coil_table_info()["builds"] == 3
        again = ctx.solve_block(a, *blk, 1e6, **KW)
        assert ctx.coil_table_info()["builds"] == 4
        # A rebuilt table is the same table: bit for bit the first block's result.
        for key in ("E", "magnE", "v"):
            np.testing.assert_array_equal(again[key], first[key], err_msg=key)
        # The moved coil's table is its own (a fresh context built for it agrees bit for bit).
        fresh = ref.solve_block(shifted, *blk, 1e6, **KW)
        np.testing.assert_array_equal(moved["E"], fresh["E"])
        # Parameters changed: rebuilt at the next block.
        ctx.set_coil_table(True, near_mm=20.0)
        ctx.solve_block(a, *blk, 1e6, **KW)
        assert ctx.coil_table_info()["builds"] == 5
    finally:
        ctx.close()
        ref.close()


def test_table_results_independent_of_block_and_pipeline(head):
    """Per node the table read and the near sum depend on nothing but the node and its placement."""
    coil = figure8_coil(512)
    c, h, d = _block(k=6, seed=11)
    ctx = _ctx(head)
    try:
        whole = ctx.solve_block(coil, c, h, d, 1e6, **KW)
        t1 = ctx.submit_block(coil, c[:2], h[:2], d[:2], 1e6, **KW)
        t2 = ctx.submit_block(coil, c[2:], h[2:], d[2:], 1e6, **KW)
        first = ctx.finish_block(t1)
        second = ctx.finish_block(t2)
        for key in ("E", "magnE"):
            np.testing.assert_array_equal(np.concatenate([first[key], second[key]]), whole[key], err_msg=key)
    finally:
        ctx.close()


def test_subject_coil_field_option(head):
    coil = figure8_coil(512)
    sites = [Placement(c, h) for c, h, _ in zip(*_block(k=2, seed=13))]
    with Subject(head, tolerance=1e-10) as s_tab, Subject(head, tolerance=1e-10, coil_field="direct") as s_dir:
        assert s_tab.coil_field == "table" and s_dir.coil_field == "direct"
        a = [r.magnE for r in s_tab.iter_simulate(coil, sites, magnitude=True)]
        b = [r.magnE for r in s_dir.iter_simulate(coil, sites, magnitude=True)]
        assert s_tab.context.coil_table_info()["in_use"]
        assert s_dir.context.coil_table_info()["mode"] == 0
        for x, y in zip(a, b):
            assert _rel(x, y) < 1e-6
    with pytest.raises(ValueError, match="coil_field"):
        Subject(head, coil_field="grid")

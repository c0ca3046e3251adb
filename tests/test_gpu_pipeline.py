"""Blocks submitted two deep (cunibs_submit_block / cunibs_finish_block and the device pair). Needs a B200.

A block's preparation (placement, dA/dt, right-hand side) runs on its own stream beside the
previous block's solve; the results must be bitwise those of the one-call entries, whatever the
order of finishing, the bounded dA/dt grid or the block's neighbours in the pipeline.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from cunibs_b200 import Placement, Subject, _native
from cunibs_b200.synthetic import figure8_coil, sphere_head

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sphere_ctx():
    m = sphere_head(6.0, 90.0, jitter_mm=0.3, seed=1)
    ctx = _native.Context(m.nodes_mm, m.tet_nodes, m.tet_tags, m.skin_tris)
    yield m, ctx
    ctx.close()


def _blocks(n, k=4, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        th = rng.uniform(0.0, 0.6, k)
        ph = rng.uniform(0.0, 2 * np.pi, k)
        c = 90.0 * np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], axis=1)
        h = c + np.stack([-np.sin(ph), np.cos(ph), np.zeros(k)], axis=1) * 50.0
        out.append((c, h, np.full(k, 4.0)))
    return out


KW = dict(magnitude=True, potential=True, recovery="harmonic")


def _same(a, b):
    for key in ("magnE", "v", "summary", "transform", "iterations", "relative_residual"):
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)


def test_pipelined_host_blocks_bitwise_equal_one_call(sphere_ctx):
    _, ctx = sphere_ctx
    coil = figure8_coil(128)
    blocks = _blocks(4)
    want = [ctx.solve_block(coil, c, h, d, 1e6, **KW) for c, h, d in blocks]
    tickets = [ctx.submit_block(coil, *blocks[0], 1e6, **KW)]
    got = []
    for b in range(1, len(blocks)):
        tickets.append(ctx.submit_block(coil, *blocks[b], 1e6, **KW))
        assert ctx.pending == 2
        got.append(ctx.finish_block(tickets.pop(0)))
    got.append(ctx.finish_block(tickets.pop(0)))
    assert ctx.pending == 0
    for a, b in zip(got, want):
        _same(a, b)


def test_finish_order_overlap_grid_and_one_call_in_between(sphere_ctx):
    _, ctx = sphere_ctx
    coil = figure8_coil(128)
    blocks = _blocks(3, seed=1)
    want = [ctx.solve_block(coil, c, h, d, 1e6, **KW) for c, h, d in blocks]
    for bps in (1, 5):
        ctx.set_overlap(bps)
        t0 = ctx.submit_block(coil, *blocks[0], 1e6, **KW)
        t1 = ctx.submit_block(coil, *blocks[1], 1e6, **KW)
        with pytest.raises(ValueError, match="two blocks are already submitted"):
            ctx.submit_block(coil, *blocks[2], 1e6, **KW)
        _same(ctx.finish_block(t1), want[1])  # the newer one first
        # A one-call solve while a block is submitted leaves that block intact.
        _same(ctx.solve_block(coil, *blocks[2], 1e6, **KW), want[2])
        _same(ctx.finish_block(t0), want[0])
    ctx.set_overlap(2)
    with pytest.raises(ValueError, match="no submitted block"):
        ctx.finish_block_device(12345, {"transforms": 1, "summary": 1})
    t = ctx.submit_block(coil, *blocks[0], 1e6, **KW)
    ctx.cancel_block(t)
    assert ctx.pending == 0


def test_device_pair_matches_device_one_call(sphere_ctx):
    _, ctx = sphere_ctx
    coil = figure8_coil(128)
    blocks = _blocks(3, seed=2)
    dev = torch.device("cuda", 0)
    pos = torch.tensor(coil.positions_m, dtype=torch.float64, device=dev)
    mom = torch.tensor(coil.moments, dtype=torch.float64, device=dev)
    ins = [[torch.tensor(a, dtype=torch.float64, device=dev) for a in blk] for blk in blocks]
    k = blocks[0][0].shape[0]

    def outs():
        o = {"transforms": torch.empty((k, 16), dtype=torch.float64, device=dev),
             "summary": torch.empty((k, 16), dtype=torch.float64, device=dev),
             "magnE": torch.empty((k, ctx.n_tets), dtype=torch.float32, device=dev),
             "iterations": torch.empty(k, dtype=torch.int32, device=dev)}
        return o, {key: t.data_ptr() for key, t in o.items()}

    args = lambda i: (pos.data_ptr(), mom.data_ptr(), coil.n_dipoles, ins[i][0].data_ptr(), ins[i][1].data_ptr(),
                      ins[i][2].data_ptr(), k, 1e6)
    want = []
    for i in range(3):
        o, ptrs = outs()
        ctx.solve_block_device(*args(i), ptrs, recovery="harmonic")
        want.append({key: t.cpu() for key, t in o.items()})
    got = []
    tickets = [ctx.submit_block_device(*args(0), recovery="harmonic")]
    for i in range(3):
        if i + 1 < 3:
            tickets.append(ctx.submit_block_device(*args(i + 1), recovery="harmonic"))
        o, ptrs = outs()
        ctx.finish_block_device(tickets.pop(0), ptrs)
        torch.cuda.synchronize()  # the outputs are complete when the context stream reaches them
        got.append({key: t.cpu() for key, t in o.items()})
    for a, b in zip(got, want):
        for key in a:
            assert torch.equal(a[key], b[key]), key


def test_degenerate_block_reported_at_its_finish(sphere_ctx):
    _, ctx = sphere_ctx
    coil = figure8_coil(64)
    good = _blocks(1, seed=3)[0]
    c = np.array([[0.0, 0.0, 90.0]])
    T, _ = ctx.place(c, c + [0.0, 50.0, 0.0], [4.0])
    normal = -T[0, :3, 2]
    proj = T[0, :3, 3] - 4.0 * normal
    bad = (c, (proj + 30.0 * normal)[None], np.array([4.0]))  # handle on the scalp normal
    tb = ctx.submit_block(coil, *bad, 1e6)
    tg = ctx.submit_block(coil, *good, 1e6)
    with pytest.raises(ValueError, match="degenerate coil placement at index 0"):
        ctx.finish_block(tb)
    _same(ctx.finish_block(tg), ctx.solve_block(coil, *good, 1e6))


def test_iter_simulate_pipelines_and_cleans_up(sphere_ctx):
    m, _ = sphere_ctx
    subj = Subject(m, tolerance=1e-8)
    coil = figure8_coil(64)
    rng = np.random.default_rng(4)
    sites = []
    for _ in range(7):
        th, ph = rng.uniform(0.0, 0.5), rng.uniform(0.0, 2 * np.pi)
        c = 90.0 * np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
        sites.append(Placement(c, c + [-50.0 * np.sin(ph), 50.0 * np.cos(ph), 0.0]))
    streamed = list(subj.iter_simulate(coil, sites, magnitude=True, block_k=2))
    for s, r in zip(sites, streamed):
        np.testing.assert_array_equal(r.magnE, subj.simulate(coil, s, magnitude=True).magnE)
    gen = subj.iter_simulate(coil, sites, magnitude=True, block_k=2)
    next(gen)
    assert subj.context.pending == 1
    gen.close()
    assert subj.context.pending == 0
    subj.free()

"""The library's device allocations are cached and reused. Needs a B200.

Contexts opened and closed one after another on the same mesh take their buffers from the blocks the
previous one freed: the cache does not grow round over round (the device's free memory stays put
after the first round, where it would fall by a context's footprint per round if freed blocks were
kept without reuse), and the answers do not change.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from cunibs_b200 import _native
from cunibs_b200.synthetic import sphere_head

pytestmark = pytest.mark.gpu


def _round(m, B):
    ctx = _native.Context(m.nodes_mm, m.tet_nodes, m.tet_tags, m.skin_tris)
    try:
        X, it, rel = ctx.solve(B, 4, 4, tolerance=1e-9, max_iters=500)
    finally:
        ctx.close()
    torch.cuda.synchronize()
    return X, it, torch.cuda.mem_get_info()[0]


def test_repeated_contexts_reuse_freed_blocks():
    m = sphere_head(4.0, 90.0, jitter_mm=0.3, seed=4)
    rng = np.random.default_rng(11)
    B = rng.standard_normal((m.n_nodes - 1, 4))
    X1, it1, _ = _round(m, B)
    X2, it2, free2 = _round(m, B)
    X3, it3, free3 = _round(m, B)
    np.testing.assert_array_equal(X1, X2)
    np.testing.assert_array_equal(X2, X3)
    np.testing.assert_array_equal(it1, it3)
    # The third round took its blocks from the cache (a little slack for the driver's own bookkeeping).
    assert free3 >= free2 - (2 << 20)

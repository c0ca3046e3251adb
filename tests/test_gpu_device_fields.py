"""Device-resident fields (cunibs_b200.fem.solve_placements_block). Needs a B200.

The CUDA tensors must hold bitwise what the host entry returns, and export through DLPack without
a copy.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from cunibs_b200 import Subject
from cunibs_b200.fem import solve_placements_block
from cunibs_b200.synthetic import figure8_coil, sphere_head

pytestmark = pytest.mark.gpu


def test_device_fields_match_host_entry_and_export_dlpack():
    mesh = sphere_head(6.0, 90.0, jitter_mm=0.3, seed=1)
    subj = Subject(mesh, tolerance=1e-8)
    ctx = subj.context
    coil = figure8_coil(64)
    c = np.array([[0.0, 0.0, 90.0], [20.0, 0.0, 87.7]])
    h = c + [0.0, 50.0, 0.0]
    sites = [(c[i], h[i], 4.0) for i in range(2)]
    got = solve_placements_block(ctx, coil.positions_m, coil.moments, sites, 1e6, recovery="harmonic", nodal=True)
    want = ctx.solve_block(coil, c, h, [4.0, 4.0], 1e6, magnitude=True, vectors=True, potential=True,
                           recovery="harmonic", nodal=True)
    for i, r in enumerate(got):
        assert r["magnE"].is_cuda and r["E"].shape == (ctx.n_tets, 3)
        np.testing.assert_array_equal(r["magnE"].cpu().numpy(), want["magnE"][i])
        np.testing.assert_array_equal(r["E"].cpu().numpy(), want["E"][i])
        np.testing.assert_array_equal(r["v"].cpu().numpy(), want["v"][i])
        np.testing.assert_array_equal(r["E_slots"].cpu().numpy(), want["E_slots"][i])
        np.testing.assert_array_equal(r["transform"], want["transform"][i])
        assert r["iterations"] == want["iterations"][i]
        shared = torch.utils.dlpack.from_dlpack(torch.utils.dlpack.to_dlpack(r["magnE"]))
        assert shared.data_ptr() == r["magnE"].data_ptr()
    with pytest.raises(ValueError, match="nodal=True needs a recovery mode"):
        solve_placements_block(ctx, coil.positions_m, coil.moments, sites, 1e6, nodal=True)
    subj.free()

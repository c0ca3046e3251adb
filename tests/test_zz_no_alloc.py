"""cunibs_dadt_noalloc: dA/dt for callers that cannot let the library allocate GPU memory.

Such a caller hands over device buffers for every input and output, and the library uses only the
fixed scratch array compiled into it. The result must equal the regular entry point's
(cunibs_context_dadt, same general-moment kernel) on two calls in a row, which also shows that the
shared scratch carries nothing over from one call to the next.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from cunibs_b200 import _native
from cunibs_b200.coil import Coil
from cunibs_b200.synthetic import figure8_coil, sphere_head

pytestmark = pytest.mark.gpu


def _tilted(coil: Coil, angle: float) -> Coil:
    c, s = np.cos(angle), np.sin(angle)
    rot = np.array([[c, 0.0, s], [0.0, 1.0, 0.0], [-s, 0.0, c]])
    return Coil(coil.positions_m, coil.moments @ rot.T)


def _noalloc(lib, torch, nodes, coil, transforms, didt):
    dev = torch.device("cuda", 0)
    d_nodes = torch.tensor(nodes, dtype=torch.float64, device=dev)
    d_pos = torch.tensor(coil.positions_m, dtype=torch.float64, device=dev)
    d_mom = torch.tensor(coil.moments, dtype=torch.float64, device=dev)
    d_T = torch.tensor(transforms.reshape(-1, 16), dtype=torch.float64, device=dev)
    k = transforms.shape[0]
    d_out = torch.full((k, nodes.shape[0], 3), float("nan"), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()
    rc = lib.cunibs_dadt_noalloc(
        C.c_void_p(d_nodes.data_ptr()), nodes.shape[0], C.c_void_p(d_pos.data_ptr()), C.c_void_p(d_mom.data_ptr()),
        coil.n_dipoles, C.c_void_p(d_T.data_ptr()), k, C.c_double(didt), C.c_void_p(d_out.data_ptr()),
        C.c_void_p(stream.cuda_stream))
    _native.check(rc)
    stream.synchronize()
    return d_out.cpu().numpy()


def test_noalloc_matches_regular_entry_point_on_two_calls():
    torch = pytest.importorskip("torch")
    lib = _native.load()
    lib.cunibs_dadt_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                        C.c_double, C.c_void_p, C.c_void_p]
    lib.cunibs_dadt_noalloc.restype = C.c_int
    mesh = sphere_head(8.0, 90.0, jitter_mm=0.3, seed=4)
    ctx = _native.Context(mesh.nodes_mm, mesh.tet_nodes, mesh.tet_tags, mesh.skin_tris)
    nodes = ctx.array("nodes_mm").reshape(-1, 3)
    top = np.array([0.0, 0.0, 90.0])
    calls = [
        (_tilted(figure8_coil(96), 0.4), np.stack([top, top + [20.0, 5.0, -2.0]]), 1e6),
        (_tilted(figure8_coil(160), -0.7), np.stack([top + [-15.0, 0.0, -1.0], top, top + [5.0, 12.0, -1.0]]), 2.5e6),
    ]
    for coil, centers, didt in calls:
        T, deg = ctx.place(centers, centers + [0.0, 50.0, 0.0], np.full(centers.shape[0], 4.0))
        assert not deg.any()
        want = ctx.dadt(coil, T, didt)
        got = _noalloc(lib, torch, nodes, coil, T, didt)
        assert np.isfinite(got).all()
        np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-6 * np.abs(want).max())
    ctx.close()


def test_noalloc_call_leaves_free_device_memory_unchanged():
    """After a first call (which, under lazy module loading, places the library's module on the
    device), further calls take no device memory: the device's free memory is the same before and
    after them."""
    torch = pytest.importorskip("torch")
    lib = _native.load()
    lib.cunibs_dadt_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                        C.c_double, C.c_void_p, C.c_void_p]
    lib.cunibs_dadt_noalloc.restype = C.c_int
    dev = torch.device("cuda", 0)
    coil = figure8_coil(128)
    n_nodes, k = 4096, 4
    rng = np.random.default_rng(7)
    d_nodes = torch.tensor(rng.uniform(-80.0, 80.0, (n_nodes, 3)), dtype=torch.float64, device=dev)
    d_pos = torch.tensor(coil.positions_m, dtype=torch.float64, device=dev)
    d_mom = torch.tensor(coil.moments, dtype=torch.float64, device=dev)
    T = np.tile(np.eye(4), (k, 1, 1))
    T[:, :3, 3] = [[0.0, 0.0, 94.0], [10.0, 0.0, 93.0], [0.0, 10.0, 93.0], [-10.0, 0.0, 93.0]]  # mm
    d_T = torch.tensor(T.reshape(-1, 16), dtype=torch.float64, device=dev)
    d_out = torch.empty((k, n_nodes, 3), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    def call():
        rc = lib.cunibs_dadt_noalloc(
            C.c_void_p(d_nodes.data_ptr()), n_nodes, C.c_void_p(d_pos.data_ptr()), C.c_void_p(d_mom.data_ptr()),
            coil.n_dipoles, C.c_void_p(d_T.data_ptr()), k, C.c_double(1e6), C.c_void_p(d_out.data_ptr()),
            C.c_void_p(stream.cuda_stream))
        _native.check(rc)
        stream.synchronize()

    call()
    free_before, _ = torch.cuda.mem_get_info(dev)
    for _ in range(3):
        call()
    free_after, _ = torch.cuda.mem_get_info(dev)
    assert free_after == free_before
    assert torch.isfinite(d_out).all()


def test_noalloc_rejects_more_records_than_its_scratch():
    torch = pytest.importorskip("torch")
    lib = _native.load()
    lib.cunibs_dadt_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                        C.c_double, C.c_void_p, C.c_void_p]
    lib.cunibs_dadt_noalloc.restype = C.c_int
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.float64, device=dev)
    out = torch.zeros(3, dtype=torch.float32, device=dev)
    p = C.c_void_p(buf.data_ptr())
    rc = lib.cunibs_dadt_noalloc(p, 1, p, p, 16385, p, 1, C.c_double(1e6), C.c_void_p(out.data_ptr()), None)
    with pytest.raises(ValueError, match="exceeds the fixed scratch"):
        _native.check(rc)

"""Failure contracts, made to happen on the host side or by a wait that runs out. Needs a B200.

* Forward non-convergence (reference tests/test_block_solve.py:321-376, contract at
  fem/solve.py:368-392,528-551): a tolerance out of reach of a small iteration budget makes every
  column of a block miss; the library rebuilds the hierarchy at the operator's current values, retries
  in FP64 from the failed iterate, and then raises SolverConvergenceError naming the column. The
  subject stays usable afterwards.
* The tensor-core GEMM's bounded mbarrier waits: with the loads withheld (a barrier that nothing
  completes) and a short wait limit, the kernel gives up, records the expiry in the device's status
  word and returns; cunibs_gemm_status reports CUNIBS_ETIMEOUT, and the next GEMM on the same context
  is correct.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from cunibs_b200 import Placement, SolverConvergenceError, Subject, _native
from cunibs_b200.synthetic import figure8_coil, sphere_head

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_sphere():
    return sphere_head(8.0, 90.0, jitter_mm=0.3, seed=5)


def _sites():
    top = np.array([0.0, 0.0, 90.0])
    return [Placement(top + [dx, 0.0, 0.0], top + [dx, 50.0, 0.0]) for dx in (0.0, 8.0, -6.0, 12.0)]


@pytest.mark.parametrize("precision", ["split", "plain"])
def test_unreachable_tolerance_rebuilds_then_raises_block(small_sphere, precision):
    coil = figure8_coil(64)
    sites = _sites()
    good = Subject(small_sphere, tolerance=1e-8, precision=precision)
    want = [r.magnE for r in good.iter_simulate(coil, sites, magnitude=True)]
    good.free()

    # Five iterations cannot reach 1e-12 (this head needs about 20), and neither can the FP64 retry's
    # five. (A tiny tolerance with a larger budget is not enough: on a small head the recursively
    # updated residual keeps falling far below machine precision, even to zero.)
    subj = Subject(small_sphere, tolerance=1e-12, max_iters=5, precision=precision)
    ctx = subj.context
    builds = ctx.hierarchy_builds
    assert builds == 1
    with pytest.raises(SolverConvergenceError) as excinfo:
        list(subj.iter_simulate(coil, sites, magnitude=True))
    err = excinfo.value
    assert ctx.hierarchy_builds == builds + 1, "the hierarchy was not rebuilt before the retry"
    assert err.column in range(len(sites)), "the failing column must be attributable"
    assert err.tolerance == 1e-12
    assert err.relative_residual > 1e-12
    assert err.iterations >= 5
    assert ctx.pending == 0  # nothing is left submitted

    # The subject still solves: a block at a reachable tolerance matches a fresh subject's.
    out = ctx.solve_block(coil, np.stack([s.center_mm for s in sites]), np.stack([s.handle_mm for s in sites]),
                          [4.0] * len(sites), 1e6, tolerance=1e-8, max_iters=2000, magnitude=True, recovery="harmonic",
                          precision={"split": _native.PREC_SPLIT, "plain": _native.PREC_PLAIN_FP64}[precision])
    assert (out["relative_residual"] <= 1e-8).all()
    for i in range(len(sites)):
        np.testing.assert_array_equal(out["magnE"][i], want[i])
    subj.free()


@pytest.mark.parametrize("M", [256, 16384])
def test_gemm_wait_runs_out_and_reports_timeout(M):
    torch = pytest.importorskip("torch")
    from cunibs_b200.warmstart import gemm

    lib = _native.load()
    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(3)
    # 256 rows: the tiled kernel; 16384 rows and 32 columns: the streamed one (persistent CTAs).
    N, K = (128 if M == 256 else 32), 512
    a = torch.randn(M, K, generator=g).to(torch.bfloat16).to(dev)
    b = torch.randn(N, K, generator=g).to(torch.bfloat16).to(dev)
    out = torch.zeros(M, N, dtype=torch.float32, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    flag = C.c_int(-1)
    _native.check(lib.cunibs_gemm_status(stream, C.byref(flag)))  # clears any earlier record
    assert flag.value == 0
    try:
        # At most 4096 polls or 1 ms per wait, and no loads issued: the MMA warp's first wait on a
        # stage that nothing fills runs out.
        _native.check(lib.cunibs_debug_gemm_waits(4096, 1_000_000, 1))
        gemm(a, b, out32=out)
        rc = lib.cunibs_gemm_status(stream, C.byref(flag))
        assert rc == _native.ETIMEOUT and flag.value == 1
        with pytest.raises(_native.NativeError, match="wait of a tensor-core GEMM expired"):
            _native.check(rc)
    finally:
        _native.check(lib.cunibs_debug_gemm_waits(0, 0, 0))
    # The record was cleared by the read, and the next GEMM with the default bounds is correct.
    _native.check(lib.cunibs_gemm_status(stream, C.byref(flag)))
    assert flag.value == 0
    gemm(a, b, out32=out)
    _native.check(lib.cunibs_gemm_status(stream, C.byref(flag)))
    want = a.double() @ b.double().T
    rel = float((out.double() - want).norm() / want.norm())
    assert rel <= 2e-6, rel

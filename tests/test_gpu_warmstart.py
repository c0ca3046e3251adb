"""The learned warm start on the GPU: the BF16 tcgen05 GEMM against FP64, the network's gradients
against the CPU restatement in oracle/mlp.py, training, and the gain over the zero guess.
Needs a B200."""

from __future__ import annotations

import numpy as np
import pytest

from oracle.mlp import forward_backward, silu

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _bf16(rng, *shape, scale=1.0):
    return torch.tensor(rng.standard_normal(shape) * scale, dtype=torch.float32, device="cuda").to(torch.bfloat16)


def _f64(t):
    return t.float().cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (300, 200, 136), (16, 16, 512), (1000, 32, 1024),
                                   (256, 512, 512), (77, 1030, 200)])
def test_gemm_matches_fp64(M, N, K):
    from cunibs_b200.warmstart import gemm

    rng = np.random.default_rng(M + N + K)
    a, b = _bf16(rng, M, K), _bf16(rng, N, K)
    out = torch.empty(M, N, device="cuda")
    gemm(a, b, out32=out)
    torch.cuda.synchronize()
    ref = _f64(a) @ _f64(b).T
    err = np.abs(out.cpu().numpy() - ref).max() / np.abs(ref).max()
    assert err <= 2e-6, err


def test_gemm_epilogue_bias_silu_transpose_and_gate():
    from cunibs_b200.warmstart import gemm

    rng = np.random.default_rng(5)
    M, N, K = 200, 192, 128
    a, b = _bf16(rng, M, K), _bf16(rng, N, K)
    bias = torch.tensor(rng.standard_normal(N), dtype=torch.float32, device="cuda")
    gate = torch.tensor(rng.standard_normal((M, N)), dtype=torch.float32, device="cuda")
    z32 = torch.empty(M, N, device="cuda")
    h16 = torch.empty(M, N, device="cuda", dtype=torch.bfloat16)
    h16t = torch.empty(N, M, device="cuda", dtype=torch.bfloat16)
    gemm(a, b, bias=bias, act=1, out32=z32, out16=h16, out16t=h16t)
    g32 = torch.empty(M, N, device="cuda")
    gemm(a, b, gate=gate, out32=g32)
    torch.cuda.synchronize()
    ref = _f64(a) @ _f64(b).T + bias.cpu().numpy()
    np.testing.assert_allclose(z32.cpu().numpy(), ref, rtol=0, atol=2e-6 * np.abs(ref).max())
    h = _f64(h16)
    np.testing.assert_allclose(h, silu(ref), rtol=1e-2, atol=1e-2)
    np.testing.assert_array_equal(_f64(h16t), h.T)
    gz = gate.cpu().numpy().astype(np.float64)
    s = 1.0 / (1.0 + np.exp(-gz))
    want = (_f64(a) @ _f64(b).T) * s * (1.0 + gz * (1.0 - s))
    np.testing.assert_allclose(g32.cpu().numpy(), want, rtol=1e-4, atol=1e-4 * np.abs(want).max())


def test_network_gradients_match_the_cpu_restatement():
    """One batch through the tensor-core forward and backward against FP64 NumPy (oracle/mlp.py)."""
    from cunibs_b200.warmstart import PoseMLP

    rng = np.random.default_rng(11)
    n_out, B = 100, 256
    mlp = PoseMLP(n_out, hidden=128, depth=3, seed=2)
    x = np.zeros((B, 64))
    x[:, :6] = rng.standard_normal((B, 6))
    x16 = torch.tensor(x, dtype=torch.float32, device="cuda").to(torch.bfloat16)
    target = torch.zeros(B, mlp.n_out_pad, device="cuda")
    target[:, :n_out] = torch.tensor(rng.standard_normal((B, n_out)), dtype=torch.float32)
    pred = mlp.forward(x16, x16.t().contiguous(), keep=True)
    loss, d32, d16, d16t = mlp.loss_and_grad(pred, target)
    mlp.backward(d32, d16, d16t)
    torch.cuda.synchronize()
    W = [_f64(w) for w in mlp.W16]
    bias = [b.cpu().numpy().astype(np.float64) for b in mlp.b]
    l_ref, p_ref, dW_ref, db_ref = forward_backward(W, bias, _f64(x16), target.cpu().numpy().astype(np.float64), n_out)
    np.testing.assert_allclose(pred.cpu().numpy(), p_ref, rtol=0, atol=2e-2 * np.abs(p_ref).max())
    assert float(loss.item()) == pytest.approx(l_ref, rel=1e-2)
    for l in range(len(W)):
        g = mlp.gW[l].cpu().numpy()
        rel = np.linalg.norm(g - dW_ref[l]) / np.linalg.norm(dW_ref[l])
        assert rel <= 2e-2, f"dW[{l}] relative error {rel:.3e}"
        gb = mlp.gb[l].cpu().numpy()
        relb = np.linalg.norm(gb - db_ref[l]) / np.linalg.norm(db_ref[l])
        assert relb <= 2e-2, f"db[{l}] relative error {relb:.3e}"


def test_training_fits_a_smooth_map():
    """A few hundred tensor-core Adam steps bring a smooth 6 -> 64 map to a tenth of its variance."""
    from cunibs_b200.warmstart import PoseMLP

    rng = np.random.default_rng(3)
    n, n_out, B = 2048, 64, 256
    f = rng.uniform(-1, 1, (n, 6))
    freq = rng.standard_normal((6, n_out))
    y = np.sin(f @ freq) + 0.5 * np.cos(2 * f @ freq)
    y = (y - y.mean(0)) / y.std(0)
    x = np.zeros((n, 64))
    x[:, :6] = f
    x16 = torch.tensor(x, dtype=torch.float32, device="cuda").to(torch.bfloat16)
    tgt = torch.zeros(n, 64, device="cuda")
    tgt[:, :n_out] = torch.tensor(y, dtype=torch.float32)
    mlp = PoseMLP(n_out, hidden=256, depth=3, seed=1)
    first = last = None
    for ep in range(60):
        perm = torch.randperm(n, device="cuda")
        for s in range(0, n, B):
            idx = perm[s:s + B]
            xb = x16[idx].contiguous()
            pred = mlp.forward(xb, xb.t().contiguous(), keep=True)
            loss, d32, d16, d16t = mlp.loss_and_grad(pred, tgt[idx].contiguous())
            mlp.backward(d32, d16, d16t)
            mlp.adam(2e-3 * (0.5 + 0.5 * np.cos(np.pi * ep / 60)))
            if first is None:
                first = float(loss.item())
        last = float(loss.item())
    assert last < 0.1 * first, (first, last)


@pytest.fixture(scope="module")
def ws_subject():
    from cunibs_b200 import Subject
    from cunibs_b200.synthetic import sphere_head

    return Subject(sphere_head(4.0, 90.0, jitter_mm=0.2, seed=5), tolerance=1e-8)


def test_warm_start_cuts_iterations_and_keeps_the_answer(ws_subject):
    """Trained on plain-method solves, the network's guess lowers the PCG iterations on held-out poses
    while the answer stays the zero-guess one to the solve tolerance."""
    from cunibs_b200 import _native
    from cunibs_b200.synthetic import figure8_coil
    from cunibs_b200.warmstart import cap_poses, train_warm_start

    ctx = ws_subject.context
    coil = figure8_coil(256)
    model = train_warm_start(ctx, coil, n_train=768, rank=192, hidden=256, depth=4, epochs=300, batch=64, seed=0)
    assert model.stats["heldout_mse"] < 0.05  # targets have unit mean square; the mean predictor scores 1
    centers, handles = cap_poses(16, seed=99)
    dists = np.full(8, 4.0)
    gain = {}
    for prec in (_native.PREC_PLAIN_FP64, _native.PREC_SPLIT, _native.PREC_MIXED):
        iters = {True: [], False: []}
        for s in range(0, 16, 8):
            outs = {}
            for warm in (False, True):
                outs[warm] = ctx.solve_block(coil, centers[s:s + 8], handles[s:s + 8], dists, 1e6, potential=True,
                                             magnitude=True, warm_start=warm, precision=prec)
                iters[warm] += list(outs[warm]["iterations"])
            assert outs[True]["warm_used"].all()
            assert (outs[True]["init_relres"] < 0.5).all()
            assert (outs[True]["relative_residual"] <= 1e-8).all()
            gm = ws_subject.mesh.tet_tags == 2
            a, b = outs[True]["magnE"][:, gm].astype(np.float64), outs[False]["magnE"][:, gm].astype(np.float64)
            assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-5
        gain[prec] = np.mean(iters[False]) - np.mean(iters[True])
        if prec == _native.PREC_SPLIT:
            # The Galerkin projection of the right-hand sides onto the same basis is the A-norm-best
            # guess it spans: it needs no more iterations than the network's and gives the same answer.
            proj = [ctx.solve_block(coil, centers[s:s + 8], handles[s:s + 8], dists, 1e6, magnitude=True,
                                    warm_start="projection", precision=prec) for s in (0, 8)]
            assert all(o["warm_used"].all() and (o["relative_residual"] <= 1e-8).all() for o in proj)
            assert np.mean([o["iterations"] for o in proj]) <= np.mean(iters[True])
            gm = ws_subject.mesh.tet_tags == 2
            a = proj[1]["magnE"][:, gm].astype(np.float64)
            assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-5
    # The guess must save the FP64 Krylov methods (plain, and FP64 PCG over the FP32 V-cycle)
    # iterations. Iterative refinement restarts its FP32 inner solve at every step with a target
    # relative to the current residual (and carries Ap by its FP32 recurrence), so a better start
    # shortens its sequence less; on this small mesh it may cost two or three iterations (measured
    # 2.5 of about 20).
    assert gain[_native.PREC_PLAIN_FP64] >= 1.0, gain
    assert gain[_native.PREC_SPLIT] >= 1.0, gain
    assert gain[_native.PREC_MIXED] >= -3.0, gain


def test_a_useless_guess_falls_back_to_the_zero_guess(ws_subject):
    """A network whose guess is no better than zero is dropped per column: the solve is then the
    zero-guess solve, bit for bit."""
    from cunibs_b200 import _native
    from cunibs_b200.synthetic import figure8_coil
    from cunibs_b200.warmstart import PoseMLP, WarmStartModel

    ctx = ws_subject.context
    n_red = ctx.n_nodes - 1
    r = 64
    mlp = PoseMLP(r, hidden=64, depth=2, seed=7)
    rng = np.random.default_rng(1)
    basis = torch.tensor(rng.standard_normal((n_red, 2 * r)), dtype=torch.float32, device="cuda").to(torch.bfloat16)
    ones6 = torch.ones(6, device="cuda")
    model = WarmStartModel(mlp, basis.contiguous(), torch.zeros(6, device="cuda"), ones6,
                           torch.zeros(r, device="cuda"), torch.full((r,), 1e3, device="cuda"), r)
    model.install(ctx)
    coil = figure8_coil(64)
    top = np.array([0.0, 0.0, 90.0])
    c = np.stack([top, top + [10.0, 0, -0.6]])
    h = c + [0.0, 50.0, 0.0]
    for prec in (_native.PREC_SPLIT, _native.PREC_MIXED):
        warm = ctx.solve_block(coil, c, h, [4.0, 4.0], 1e6, magnitude=True, warm_start=True, precision=prec)
        cold = ctx.solve_block(coil, c, h, [4.0, 4.0], 1e6, magnitude=True, warm_start=False, precision=prec)
        assert not warm["warm_used"].any()
        np.testing.assert_array_equal(warm["magnE"], cold["magnE"])
        np.testing.assert_array_equal(warm["iterations"], cold["iterations"])
    ctx.set_warm_start(0, 0, 0, None, None, None, None, None, None, None)
    with pytest.raises(ValueError, match="no warm-start network"):
        ctx.solve_block(coil, c, h, [4.0, 4.0], 1e6, warm_start=True)


@pytest.mark.parametrize("M,N", [(178636, 32), (20000, 16), (8192 + 77, 32)])
def test_streamed_tall_gemm_matches_tiled_bitwise_and_fp64(M, N, monkeypatch):
    """The tall, narrow product (the basis prolongation) runs on persistent CTAs that stream A and
    keep two TMEM accumulators; it issues the same MMAs in the same order as the tiled kernel, so
    the two agree bit for bit, and both match FP64 to accumulation rounding."""
    import ctypes as C

    from cunibs_b200 import _native
    from cunibs_b200.warmstart import gemm

    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(M)
    K = 512
    a = torch.randn(M, K, generator=g).to(torch.bfloat16).to(dev)
    b = torch.randn(N, K, generator=g).to(torch.bfloat16).to(dev)
    streamed = torch.full((M, N), float("nan"), dtype=torch.float32, device=dev)
    gemm(a, b, out32=streamed)
    monkeypatch.setenv("CUNIBS_GEMM_TILED", "1")
    tiled = torch.full((M, N), float("nan"), dtype=torch.float32, device=dev)
    gemm(a, b, out32=tiled)
    lib = _native.load()
    _native.check(lib.cunibs_gemm_status(C.c_void_p(torch.cuda.current_stream().cuda_stream), None))
    assert torch.equal(streamed, tiled)
    want = a.double() @ b.double().T
    rel = float((streamed.double() - want).norm() / want.norm())
    assert rel <= 2e-6, rel

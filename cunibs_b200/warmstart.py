"""Learned warm start for the block PCG solve.

A small MLP maps a coil pose to the coefficients of a reduced basis of the grounded potential; the
basis times the predicted coefficients is the initial guess of PCG, which then runs to the same
tolerance. The plain zero-guess solve stays the fallback: a column whose guess has a relative
residual of 1 or more starts from zero instead.

* Training data: solves the plain method generates (FP64 PCG, zero guess) at random poses over the
  scalp cap above ``z_min_mm``.
* Basis: the leading ``rank`` left singular vectors of the training potentials (POD), kept as
  ``[V_hi | V_lo]`` in BF16 (about 16 significant bits through the split product).
* Targets: the Galerkin coefficients ``(V^T A V)^-1 V^T b`` of every training solve, the
  best guess in the energy norm that the basis can carry, shifted by their mean and divided by one
  common scale.
* Network: 6 pose inputs (coil origin / 100 mm, handle axis) -> ``depth`` SiLU layers of width
  ``hidden`` -> ``rank`` outputs, BF16 weights and activations, FP32 accumulation. Forward and
  backward products all run on the project's tcgen05 GEMM (``cunibs_gemm_bf16``); the loss, bias
  gradients and Adam updates are the project's kernels too. PyTorch holds the device buffers.

The solver-side half (features, inference, prolongation, fallback) runs inside the block solve.
"""

from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native

IN_PAD = 64  # pose features (6) padded to one 128-byte BF16 row


def _torch():
    import torch

    return torch


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream() -> C.c_void_p:
    return C.c_void_p(_torch().cuda.current_stream().cuda_stream)


def gemm(a16, b16, *, bias=None, gate=None, act=0, out32=None, out16=None, out16t=None) -> None:
    """out = a16 [M, K] . b16 [N, K]^T on the tensor cores (all device tensors, row-major)."""
    lib = _native.load()
    M, K = a16.shape
    N = b16.shape[0]
    ld_out = (out32 if out32 is not None else out16).stride(0) if (out32 is not None or out16 is not None) else N
    _native.check(lib.cunibs_gemm_bf16(
        _p(a16), a16.stride(0), _p(b16), b16.stride(0), M, N, K, _p(bias), _p(gate),
        gate.stride(0) if gate is not None else 0, int(act), _p(out32), _p(out16), ld_out, _p(out16t),
        out16t.stride(0) if out16t is not None else 0, _stream()))


def pose_features(transforms: np.ndarray) -> np.ndarray:
    """The 6 raw pose numbers of (k, 4, 4) coil transforms: origin / 100 mm and the handle (y) axis."""
    T = np.asarray(transforms, np.float64).reshape(-1, 4, 4)
    return np.concatenate([T[:, :3, 3] * 0.01, T[:, :3, 1]], axis=1)


class PoseMLP:
    """The warm-start network, trained with the project's tensor-core kernels."""

    def __init__(self, n_out: int, hidden: int = 512, depth: int = 4, seed: int = 0, device: int = 0) -> None:
        torch = _torch()
        if hidden % 64 or hidden < 64:
            raise ValueError("hidden must be a positive multiple of 64")
        self.n_out = int(n_out)
        self.n_out_pad = (self.n_out + 63) // 64 * 64
        self.hidden = int(hidden)
        self.depth = int(depth)
        self.dev = torch.device("cuda", device)
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.W, self.b = [], []
        dims = [(IN_PAD, 6)] + [(self.hidden, self.hidden)] * (self.depth - 1)
        for l in range(self.depth + 1):
            fan_in_pad, fan_in = (IN_PAD, 6) if l == 0 else (self.hidden, self.hidden)
            out = self.hidden if l < self.depth else self.n_out_pad
            w = torch.zeros(out, fan_in_pad)
            bound = (6.0 / fan_in) ** 0.5 if l < self.depth else (1.0 / fan_in) ** 0.5
            w[:, :fan_in] = (torch.rand(out, fan_in, generator=g) * 2 - 1) * bound
            if l == self.depth:
                w[self.n_out:] = 0.0
            self.W.append(w.to(self.dev))
            self.b.append(torch.zeros(out, device=self.dev))
        del dims
        self.W16 = [w.to(torch.bfloat16) for w in self.W]
        self.W16t = [w.t().contiguous().to(torch.bfloat16) for w in self.W]
        self.mW = [torch.zeros_like(w) for w in self.W]
        self.vW = [torch.zeros_like(w) for w in self.W]
        self.mb = [torch.zeros_like(b) for b in self.b]
        self.vb = [torch.zeros_like(b) for b in self.b]
        self.gW = [torch.zeros_like(w) for w in self.W]
        self.gb = [torch.zeros_like(b) for b in self.b]
        self.step_count = 0
        self._scratch = torch.zeros(296, device=self.dev)
        self._loss = torch.zeros(1, device=self.dev)
        self._bufs: dict[int, dict] = {}

    def _buffers(self, B: int) -> dict:
        torch = _torch()
        if B not in self._bufs:
            bf, f32 = torch.bfloat16, torch.float32
            d = {"Z": [], "H": [], "Ht": [], "dZ": [], "dZ16": [], "dZt": []}
            for l in range(self.depth + 1):
                out = self.hidden if l < self.depth else self.n_out_pad
                d["Z"].append(torch.empty(B, out, device=self.dev, dtype=f32))
                d["H"].append(torch.empty(B, out, device=self.dev, dtype=bf))
                d["Ht"].append(torch.empty(out, B, device=self.dev, dtype=bf))
                d["dZ"].append(torch.empty(B, out, device=self.dev, dtype=f32))
                d["dZ16"].append(torch.empty(B, out, device=self.dev, dtype=bf))
                d["dZt"].append(torch.empty(out, B, device=self.dev, dtype=bf))
            self._bufs[B] = d
        return self._bufs[B]

    def forward(self, x16, x16t=None, keep: bool = False):
        """x16 [B, 64] BF16 standardised features -> FP32 [B, n_out_pad] (cached for backward if keep)."""
        B = x16.shape[0]
        buf = self._buffers(B)
        h = x16
        for l in range(self.depth + 1):
            last = l == self.depth
            gemm(h, self.W16[l], bias=self.b[l], act=0 if last else 1, out32=buf["Z"][l],
                 out16=None if last else buf["H"][l], out16t=buf["Ht"][l] if (keep and not last) else None)
            h = buf["H"][l]
        if keep:
            buf["x16t"] = x16t
        return buf["Z"][self.depth]

    def backward(self, d32, d16, d16t) -> None:
        """Gradients of the loss whose output gradient is d (FP32 / BF16 / BF16 transposed) into gW, gb."""
        B = d32.shape[0]
        buf = self._buffers(B)
        dZ, dZ16, dZt = d32, d16, d16t
        for l in range(self.depth, -1, -1):
            inp_t = buf["x16t"] if l == 0 else buf["Ht"][l - 1]
            gemm(dZt, inp_t, out32=self.gW[l])  # dW = dZ^T . H_prev  ([out, B] . [in, B]^T)
            _native.check(_native.load().cunibs_mlp_colsum(_p(dZ), B, dZ.shape[1], dZ.stride(0), _p(self.gb[l]),
                                                           _stream()))
            if l == 0:
                break
            # dZ_prev = (dZ . W) * silu'(Z_prev)
            gemm(dZ16, self.W16t[l], gate=buf["Z"][l - 1], out32=buf["dZ"][l - 1], out16=buf["dZ16"][l - 1],
                 out16t=buf["dZt"][l - 1])
            dZ, dZ16, dZt = buf["dZ"][l - 1], buf["dZ16"][l - 1], buf["dZt"][l - 1]

    def adam(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8, weight_decay: float = 0.0):
        lib = _native.load()
        self.step_count += 1
        t = self.step_count
        for l in range(self.depth + 1):
            W = self.W[l]
            _native.check(lib.cunibs_mlp_adam(_p(W), _p(self.mW[l]), _p(self.vW[l]), _p(self.gW[l]), W.numel(), lr,
                                              beta1, beta2, eps, t, weight_decay, W.shape[0], W.shape[1],
                                              _p(self.W16[l]), _p(self.W16t[l]), _stream()))
            b = self.b[l]
            _native.check(lib.cunibs_mlp_adam(_p(b), _p(self.mb[l]), _p(self.vb[l]), _p(self.gb[l]), b.numel(), lr,
                                              beta1, beta2, eps, t, 0.0, 1, b.numel(), None, None, _stream()))

    def loss_and_grad(self, pred, target):
        """MSE over the real outputs and its gradient (FP32, BF16, BF16 transposed)."""
        torch = _torch()
        B = pred.shape[0]
        d32 = torch.zeros_like(pred)
        d16 = torch.zeros(B, pred.shape[1], device=self.dev, dtype=torch.bfloat16)
        d16t = torch.zeros(pred.shape[1], B, device=self.dev, dtype=torch.bfloat16)
        _native.check(_native.load().cunibs_mlp_mse(_p(pred), _p(target), B, self.n_out, pred.stride(0),
                                                    _p(self._loss), _p(d32), _p(d16), _p(d16t), B, _p(self._scratch),
                                                    _stream()))
        return self._loss, d32, d16, d16t


@dataclass
class WarmStartModel:
    """A trained warm start for one subject: network, basis and standardisation, ready to install."""

    mlp: PoseMLP
    basis16: object           # torch BF16 [n_red, 2 r]: [V_hi | V_lo]
    feature_mean: object      # torch FP32 [6]
    feature_std: object
    coef_mean: object         # torch FP32 [r]
    coef_std: object
    rank: int
    stats: dict = field(default_factory=dict)

    def install(self, ctx: _native.Context) -> None:
        m = self.mlp
        ctx.set_warm_start(m.depth, m.hidden, self.rank, [w.data_ptr() for w in m.W16], [b.data_ptr() for b in m.b],
                           _p(self.feature_mean), _p(self.feature_std), _p(self.coef_mean), _p(self.coef_std),
                           _p(self.basis16))


def cap_poses(n: int, radius_mm: float = 90.0, z_min_mm: float = 40.0, seed: int = 0):
    """n (centre, handle) pairs: centres uniform over the sphere cap above z_min_mm, handle azimuth
    uniform in [0, 2 pi)."""
    rng = np.random.default_rng(seed)
    centers, handles = [], []
    while len(centers) < n:
        v = rng.standard_normal(3)
        v /= np.linalg.norm(v)
        if v[2] * radius_mm < z_min_mm:
            continue
        c = radius_mm * v
        t1 = np.cross(v, [0.0, 0.0, 1.0])
        t1 = t1 / np.linalg.norm(t1) if np.linalg.norm(t1) > 1e-6 else np.array([1.0, 0.0, 0.0])
        t2 = np.cross(v, t1)
        a = rng.uniform(0.0, 2.0 * np.pi)
        centers.append(c)
        handles.append(c + 50.0 * (np.cos(a) * t1 + np.sin(a) * t2))
    return np.stack(centers), np.stack(handles)


def generate_solves(ctx: _native.Context, coil, centers, handles, didt: float = 1e6, tolerance: float = 1e-8,
                    block: int = 8):
    """Plain FP64 zero-guess solves of the given poses: (transforms (n,4,4), grounded potentials as a
    torch FP64 [n, n_red] device tensor, iterations (n))."""
    torch = _torch()
    n = centers.shape[0]
    dev = torch.device("cuda", torch.cuda.current_device())
    pos = torch.tensor(coil.positions_m, dtype=torch.float64, device=dev)
    mom = torch.tensor(coil.moments, dtype=torch.float64, device=dev)
    X = torch.empty(n, ctx.n_nodes - 1, dtype=torch.float64, device=dev)
    T_all = np.empty((n, 4, 4))
    iters = np.empty(n, np.int32)
    keep = torch.ones(ctx.n_nodes, dtype=torch.bool, device=dev)
    keep[ctx.ground_node] = False
    for s in range(0, n, block):
        k = min(block, n - s)
        c = torch.tensor(centers[s:s + k], dtype=torch.float64, device=dev)
        h = torch.tensor(handles[s:s + k], dtype=torch.float64, device=dev)
        d = torch.full((k,), 4.0, dtype=torch.float64, device=dev)
        T = torch.empty(k, 16, dtype=torch.float64, device=dev)
        S = torch.empty(k, 16, dtype=torch.float64, device=dev)
        v = torch.empty(k, ctx.n_nodes, dtype=torch.float64, device=dev)
        it = torch.empty(k, dtype=torch.int32, device=dev)
        ctx.solve_block_device(pos.data_ptr(), mom.data_ptr(), pos.shape[0], c.data_ptr(), h.data_ptr(), d.data_ptr(),
                               k, didt, {"transforms": T.data_ptr(), "summary": S.data_ptr(), "v": v.data_ptr(),
                                         "iterations": it.data_ptr()},
                               precision=_native.PREC_PLAIN_FP64, tolerance=tolerance)
        X[s:s + k] = v[:, keep]
        T_all[s:s + k] = T.reshape(k, 4, 4).cpu().numpy()
        iters[s:s + k] = it.cpu().numpy()
    return T_all, X, iters


def _operator(ctx: _native.Context):
    """The grounded FP64 stiffness as a torch sparse CSR device tensor."""
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    n = ctx.n_nodes - 1
    ptr = torch.tensor(ctx.array("a_ptr", 0).astype(np.int64), device=dev)
    col = torch.tensor(ctx.array("a_col", 0).astype(np.int64), device=dev)
    val = torch.tensor(ctx.array("a_val", 0), device=dev)
    return torch.sparse_csr_tensor(ptr, col, val, size=(n, n))


def train_warm_start(ctx: _native.Context, coil, *, n_train: int = 4096, rank: int = 512, hidden: int = 512,
                     depth: int = 4, epochs: int = 400, batch: int = 256, lr: float = 1e-3, seed: int = 0,
                     tolerance: float = 1e-8, z_min_mm: float = 40.0, radius_mm: float = 90.0,
                     install: bool = True, energy: bool = True) -> WarmStartModel:
    """Generate training solves, build the basis, train the network on the GPU and (optionally)
    install it in the context. Returns the model with timing and loss statistics."""
    torch = _torch()
    t0 = time.perf_counter()
    rank = min(rank, n_train)  # the POD of n_train solves has at most n_train modes
    centers, handles = cap_poses(n_train, radius_mm, z_min_mm, seed)
    T, X, iters = generate_solves(ctx, coil, centers, handles, tolerance=tolerance)
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    # POD basis of the potentials, then the Galerkin coefficients of every training solve.
    t1 = time.perf_counter()
    G = X @ X.T
    evals, evecs = torch.linalg.eigh(G)
    order = torch.argsort(evals, descending=True)[:rank]
    lam = evals[order].clamp_min(evals[order][0] * 1e-14)
    V = (X.T @ evecs[:, order]) / lam.sqrt()                    # [n_red, r], orthonormal columns
    A = _operator(ctx)
    AV = A @ V
    Gal = V.T @ AV
    # Galerkin coefficients (V^T A V)^-1 V^T b with b = A x: V^T A x = (A V)^T x, A symmetric.
    coef = torch.linalg.solve(Gal, AV.T @ X.T).T.contiguous()  # [n_train, r]
    if energy:
        # A-orthonormal basis W = V L^-T (V^T A V = L L^T): the Galerkin coefficients are then
        # W^T b, and their Euclidean error is the guess's A-norm error, the norm PCG converges in.
        L = torch.linalg.cholesky(Gal)
        V = torch.linalg.solve_triangular(L, V.T, upper=False).T.contiguous()
        coef = (coef @ L).contiguous()  # V c = W L^T c, so the W-coefficients are L^T c
    del G, AV
    r = rank
    r_pad = (r + 63) // 64 * 64
    Vp = torch.zeros(V.shape[0], r_pad, dtype=torch.float64, device=V.device)
    Vp[:, :r] = V
    hi = Vp.to(torch.bfloat16)
    lo = (Vp - hi.to(torch.float64)).to(torch.bfloat16)
    basis16 = torch.cat([hi, lo], dim=1).contiguous()
    del V, Vp, hi, lo, X
    torch.cuda.synchronize()
    t_basis = time.perf_counter() - t1
    # Standardisation.
    feats = torch.tensor(pose_features(T), dtype=torch.float32, device=coef.device)
    f_mean, f_std = feats.mean(0), feats.std(0).clamp_min(1e-6)
    # One scale for every coefficient, so the loss weighs each mode by its share of the potential
    # (the basis is orthonormal: coefficient error is solution error); per-mode standardisation
    # would weigh the noisy tail modes like the dominant ones.
    c_mean = coef.mean(0).float()
    c_std = torch.full((coef.shape[1],), float((coef - coef.mean(0)).std()), device=coef.device,
                       dtype=torch.float32).clamp_min(1e-30)
    target = torch.zeros(n_train, r_pad, dtype=torch.float32, device=coef.device)
    target[:, :r] = (coef.float() - c_mean) / c_std
    x = torch.zeros(n_train, IN_PAD, dtype=torch.float32, device=coef.device)
    x[:, :6] = (feats - f_mean) / f_std
    x16 = x.to(torch.bfloat16)
    # Training.
    t2 = time.perf_counter()
    mlp = PoseMLP(r, hidden, depth, seed)
    if n_train < 2 * batch:
        batch = max(8, (n_train // 2) // 8 * 8)
    n_hold = max(batch, n_train // 8)
    n_fit = (n_train - n_hold) // batch * batch
    gen = torch.Generator(device="cpu").manual_seed(seed + 1)
    losses = []
    for ep in range(epochs):
        perm = torch.randperm(n_fit, generator=gen).to(coef.device)
        lr_ep = lr * 0.5 * (1.0 + np.cos(np.pi * ep / epochs))
        for s in range(0, n_fit, batch):
            idx = perm[s:s + batch]
            xb = x16[idx].contiguous()
            xbt = xb.t().contiguous()
            pred = mlp.forward(xb, xbt, keep=True)
            loss, d32, d16, d16t = mlp.loss_and_grad(pred, target[idx].contiguous())
            mlp.backward(d32, d16, d16t)
            mlp.adam(lr_ep)
        if ep % max(1, epochs // 20) == 0 or ep == epochs - 1:
            losses.append((ep, float(loss.item())))
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t2
    # Held-out error of the standardised coefficients.
    xh = x16[n_fit:n_fit + n_hold // batch * batch].contiguous()
    held = []
    mode_err = torch.zeros(r, dtype=torch.float64, device=coef.device)
    for s in range(0, xh.shape[0], batch):
        p = mlp.forward(xh[s:s + batch])
        tb = target[n_fit + s:n_fit + s + batch].contiguous()
        loss, *_ = mlp.loss_and_grad(p, tb)
        held.append(float(loss.item()))
        mode_err += ((p[:, :r].double() - tb[:, :r].double()) ** 2).sum(0)
    # Where the held-out error sits: its share in the leading modes (the guess's A-norm error is the
    # coefficient error, the basis being A-orthonormal).
    err_share = {}
    if held:
        cum = torch.cumsum(mode_err, 0) / mode_err.sum().clamp_min(1e-300)
        err_share = {str(m): round(float(cum[m - 1]), 4) for m in (8, 16, 32, 64, 128) if m <= r}
    # Every GEMM of the training and the held-out pass reports an expired barrier wait to the
    # device's status word: a network trained on invalid products is refused here.
    _native.check(_native.load().cunibs_gemm_status(_stream(), None))
    model = WarmStartModel(mlp, basis16, f_mean.contiguous(), f_std.contiguous(), c_mean.contiguous(),
                           c_std.contiguous(), r)
    model.stats = {"n_train": n_train, "rank": r, "train_iterations_mean": float(iters.mean()),
                   "data_s": round(t_data, 3), "basis_s": round(t_basis, 3), "train_s": round(t_train, 3),
                   "loss_curve": losses, "heldout_mse": float(np.mean(held)) if held else None,
                   "train_mse": losses[-1][1] if losses else None, "n_fit": n_fit, "epochs": epochs,
                   "batch": batch, "heldout_error_share_leading_modes": err_share}
    if install:
        model.install(ctx)
    return model

"""Benchmark: placements/s of the per-placement field solve on the 1M-tet 10-tissue sphere head.

Workload: 8-shell sphere of radius 90 mm with an eye and a muscle cap, Kuhn
lattice at 2.63 mm (1.0M tetrahedra, 0.18M nodes; a 1.5 mm lattice reaches 1M tetrahedra only at
a 51 mm radius, so the lattice is coarsened to keep a head-sized sphere), +-0.2 mm seeded node jitter;
figure-8 coil of 2 x 2048 dipoles; 8 placements on a 15-degree grid of the upper hemisphere solved as
one block (block_k = 8) to relative residual 1e-8. A step is one block of 8 placements: coil
placement, dA/dt, right-hand side, block PCG, field recovery (harmonic by default, as Subject.simulate)
and gray-matter summary.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--precision split|mixed|plain]

Prints one JSON line (rank 0). ``value`` is device-timed with CUDA events on the library's stream
around all timed steps, inputs resident in HBM, L2 flushed before every step's solve, blocks
submitted two deep as Subject.iter_simulate runs them (a block's placement, dA/dt and right-hand side
beside the previous block's solve); ``e2e`` goes through the host C ABI (cunibs_submit_block /
cunibs_finish_block) with host buffers, timed by the wall clock.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from cunibs_b200.synthetic import EIGHT_SHELLS, EYE_CAP, MUSCLE_CAP, figure8_coil, sphere_head  # noqa: E402

METRIC = "placements/s @1M tets, rel.res 1e-8: learned+mixed vs plain FP64 PCG, same B200"
TOL = 1e-8
PARITY_ORACLE_TOL = 1e-12  # the oracle's solve in the parity check: the exact discrete field
K_BLOCK = 8


def workload():
    mesh = sphere_head(2.63, 90.0, EIGHT_SHELLS, (EYE_CAP, MUSCLE_CAP), jitter_mm=0.2, seed=0)
    coil = figure8_coil(2048)
    sites = []
    for th, ph in [(0, 0), (15, 0), (15, 90), (15, 180), (15, 270), (30, 45), (30, 135), (30, 225)]:
        t, f = np.radians(th), np.radians(ph)
        c = 90.0 * np.array([np.sin(t) * np.cos(f), np.sin(t) * np.sin(f), np.cos(t)])
        sites.append((c, c + 50.0 * np.array([-np.sin(f), np.cos(f), 0.0])))
    return mesh, coil, sites


def config_dict(mesh, extra=None):
    d = {"workload": "1M-tet 10-tissue sphere head, 8 placements x 2x2048-dipole figure-8", "n_tets": int(mesh.n_tets),
         "n_nodes": int(mesh.n_nodes), "lattice_mm": 2.63, "radius_mm": 90.0, "dipoles": 4096, "block_k": K_BLOCK,
         "placements_per_step": K_BLOCK, "tolerance": TOL}
    if extra:
        d.update(extra)
    return d


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled from before the warm-up to the end of the
    comparison arms. Each sample carries nvidia-smi's own timestamp, so the summary holds the
    samples taken inside the timed region. nvidia-smi starts slowly and a short timed region may
    hold fewer than three samples; the summary then takes the three nearest to it and reports how
    far outside the region they lie (slack_ms). Throttle reasons seen anywhere in the sampled
    window are reported as well."""

    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device: int, command: str = "nvidia-smi") -> None:
        self.device = device
        self.command = command
        self.proc = None
        self.lines: list[str] = []
        self.t = None
        self.region: tuple[float, float] | None = None

    def start(self, wait_s: float = 5.0) -> "ClockSampler":
        """Starts sampling every 100 ms and waits (at most wait_s) for the first sample."""
        try:
            self.proc = subprocess.Popen(
                [self.command, "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
            return self
        import atexit

        atexit.register(self.stop)
        t_end = time.time() + wait_s
        while not self.lines and self.proc.poll() is None and time.time() < t_end:
            time.sleep(0.02)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def mark(self, t0: float, t1: float) -> None:
        """The timed region's start and end (time.time())."""
        self.region = (t0, t1)

    def stop(self) -> None:
        if self.proc is not None and self.proc.poll() is None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            if self.t is not None:
                self.t.join(timeout=5)

    @staticmethod
    def _when(stamp: str) -> float | None:
        import datetime

        for fmt in ("%Y/%m/%d %H:%M:%S.%f", "%Y/%m/%d %H:%M:%S"):
            try:
                return datetime.datetime.strptime(stamp.strip(), fmt).timestamp()
            except ValueError:
                continue
        return None

    def _samples(self) -> list[tuple[float | None, float, float, set]]:
        out = []
        for line in list(self.lines):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm, mx = float(parts[1]), float(parts[2])
            except ValueError:
                continue
            reasons = {n for n, v in zip(self.REASONS, parts[3:7]) if v.lower() == "active"}
            out.append((self._when(parts[0]), sm, mx, reasons))
        return out

    def summary(self) -> dict:
        samples = self._samples()
        window = sorted(set().union(*(r for *_, r in samples))) if samples else []
        chosen, inside, slack = samples, None, None
        timed = [x for x in samples if x[0] is not None]
        if self.region is not None and timed and len(timed) == len(samples):
            t0, t1 = self.region
            dist = [max(t0 - x[0], x[0] - t1, 0.0) for x in timed]
            inside = sum(d == 0.0 for d in dist)
            order = sorted(range(len(timed)), key=lambda i: dist[i])
            keep = [i for i in order if dist[i] == 0.0]
            if len(keep) < 3:
                keep = order[:3]
            chosen = [timed[i] for i in keep]
            slack = round(max(dist[i] for i in keep) * 1e3, 1)
        sm = [x[1] for x in chosen]
        mx = [x[2] for x in chosen]
        reasons = sorted(set().union(*(x[3] for x in chosen))) if chosen else []
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(chosen), "in_region": inside, "slack_ms": slack,
                "window_samples": len(samples), "window_reasons": window}


def job_throughput(local_ms: float, steps: int, world: int, dist=None, device="cpu") -> tuple[float, float]:
    """Whole-job placements/s of `world` replicas that each timed `steps` blocks of K_BLOCK
    placements: the slowest rank's time (max over ranks) bounds the job."""
    import torch

    total_ms = float(local_ms)
    if dist is not None and world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    return total_ms, world * steps * K_BLOCK / (total_ms / 1e3)


def solve_bytes_per_iteration(ctx, K: int, precision: str) -> tuple[float, float]:
    """Algorithmic bytes of one PCG iteration and of one FP64 refinement step at block width K.

    Unique bytes each kernel must move, no reuse credit. v_b/v_x: the V-cycle's value/vector bytes,
    4 except in plain FP64; k_b/k_x: the Krylov body's, 4 only in mixed precision. On level l with n rows, nnz entries, a prolongator of
    pnnz entries and nc coarse rows:
      SpMV      nnz*(v_b+4) + 4*(n+1) + 2*v_x*K*n      (values, columns, row pointers, x and y)
      Chebyshev SpMV + 4*n + 4*v_x*K*n                  (+ dinv; x_cur, x_prev, b, out)
      residual  SpMV + 3*v_x*K*n
      restrict  pnnz*(v_b+4) + 4*(nc+1) + v_x*K*(n+nc) (+ the fused first coarse step: dinv, x)
      prolong   pnnz*(v_b+4) + 4*(n+1) + v_x*K*(nc+2n) (x_f read and written)
      coarse    v_b*nc^2 + 2*v_x*K*nc
    and the PCG body's BLAS-1 passes count each (n, K) vector read or written once.
    """
    # The V-cycle streams FP32 copies except in plain FP64; the Krylov body is FP32 only in mixed.
    vb = vx = 8 if precision == "plain" else 4
    kb = kx = 4 if precision == "mixed" else 8
    sizes = ctx.levels()
    L = ctx.vcycle_levels  # levels the V-cycle smooths; the one below is solved densely
    sizes = list(sizes[:L]) + [ctx.bottom_rows]
    deg = 2
    total = 0.0
    for lev in range(L):
        n, nc = sizes[lev], sizes[lev + 1]
        nnz = ctx.array("a_col", lev).shape[0]
        pnnz = ctx.array("p_col", lev).shape[0]
        spmv = nnz * (vb + 4) + 4 * (n + 1) + 2 * vx * K * n
        cheb = spmv + 4 * n + 4 * vx * K * n
        if lev == 0:
            total += 4 * n + 2 * vx * K * n  # zero-guess first step x = a0*dinv*b
        total += (deg - 1) * cheb + spmv + 3 * vx * K * n
        total += pnnz * (vb + 4) + 4 * (nc + 1) + vx * K * (n + nc)
        if lev + 1 < L:
            total += 4 * nc + vx * K * nc
        total += pnnz * (vb + 4) + 4 * (n + 1) + vx * K * (nc + 2 * n)
        total += deg * cheb
    nc = ctx.bottom_rows
    total += vb * nc * nc + 2 * vx * K * nc
    n0 = sizes[0]
    nnz0 = ctx.array("a_col", 0).shape[0] if L > 0 else 0
    total += nnz0 * (kb + 4) + 4 * (n0 + 1) + 2 * kx * K * n0  # Ap = A p (+ p.Ap)
    total += 6 * kx * K * n0  # x += a p, r -= a Ap (+ ||r||)
    if precision == "split":
        total += vx * K * n0  # r rounded to FP32 for the V-cycle
    total += 2 * vx * K * n0  # r.z
    total += (2 * kx + vx) * K * n0  # p = z + b p
    outer = nnz0 * 12 + 4 * (n0 + 1) + (8 + 8 + 4) * K * n0 + 20 * K * n0  # B - A X in FP64; X += d
    return float(total), float(outer)


def run_ours(args) -> dict:
    import torch

    from cunibs_b200 import _native

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta

        dist_mod.init_process_group("nccl", timeout=timedelta(seconds=300))
        dist = dist_mod

    mesh, coil, sites = workload()
    p = _native.default_params()
    p.device = local
    p.tolerance = TOL
    p.precision = {"mixed": _native.PREC_MIXED, "split": _native.PREC_SPLIT, "plain": _native.PREC_PLAIN_FP64}[
        args.precision]
    if args.cheby_degree > 0:
        p.cheby_degree = args.cheby_degree
    if args.cheby_lower_ratio > 0:
        p.cheby_lower_ratio = args.cheby_lower_ratio
    t0 = time.perf_counter()
    ctx = _native.Context(mesh.nodes_mm, mesh.tet_nodes, mesh.tet_tags, mesh.skin_tris, p)
    setup_s = time.perf_counter() - t0
    ctx.set_timing(True)
    if args.overlap > 0:
        ctx.set_overlap(args.overlap)
    use_table = args.coil_field == "table"
    ctx.set_coil_table(use_table)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=local)

    centers = np.stack([c for c, _ in sites])
    handles = np.stack([h for _, h in sites])
    dists = np.full(K_BLOCK, 4.0)
    dev = torch.device("cuda", local)
    d_pos = torch.tensor(coil.positions_m, dtype=torch.float64, device=dev)
    d_mom = torch.tensor(coil.moments, dtype=torch.float64, device=dev)
    d_c = torch.tensor(centers, dtype=torch.float64, device=dev)
    d_h = torch.tensor(handles, dtype=torch.float64, device=dev)
    d_d = torch.tensor(dists, dtype=torch.float64, device=dev)
    d_T = torch.empty((K_BLOCK, 16), dtype=torch.float64, device=dev)
    d_S = torch.empty((K_BLOCK, 16), dtype=torch.float64, device=dev)
    outs = {"transforms": d_T.data_ptr(), "summary": d_S.data_ptr()}
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    warm_stats = None
    if args.warm_start == "on":
        from cunibs_b200.warmstart import train_warm_start

        with torch.cuda.device(local):
            model = train_warm_start(ctx, coil, n_train=args.train, rank=args.rank, hidden=args.hidden,
                                     epochs=args.epochs, seed=1)
        warm_stats = {k: v for k, v in model.stats.items() if k != "loss_curve"}
    d_used = torch.zeros(K_BLOCK, dtype=torch.int32, device=dev)
    d_rel0 = torch.zeros(K_BLOCK, dtype=torch.float64, device=dev)
    d_it = torch.zeros(K_BLOCK, dtype=torch.int32, device=dev)
    outs.update({"warm_used": d_used.data_ptr(), "init_relres": d_rel0.data_ptr(), "iterations": d_it.data_ptr()})

    def step(precision=_native.PREC_DEFAULT, warm=args.warm_start == "on"):
        return ctx.solve_block_device(d_pos.data_ptr(), d_mom.data_ptr(), coil.n_dipoles, d_c.data_ptr(),
                                      d_h.data_ptr(), d_d.data_ptr(), K_BLOCK, 1e6, outs, recovery=args.recovery,
                                      precision=precision, warm_start=warm)

    def submit(precision=_native.PREC_DEFAULT, warm=args.warm_start == "on"):
        return ctx.submit_block_device(d_pos.data_ptr(), d_mom.data_ptr(), coil.n_dipoles, d_c.data_ptr(),
                                       d_h.data_ptr(), d_d.data_ptr(), K_BLOCK, 1e6, recovery=args.recovery,
                                       precision=precision, warm_start=warm)

    def finish(ticket):
        # L2 flushed on the library stream before every block's solve.
        with torch.cuda.stream(stream):
            flush.zero_()
        return ctx.finish_block_device(ticket, outs)

    def pipelined(n, **kw):
        """Device time of n steps submitted two deep, as Subject.iter_simulate runs its blocks: each
        block's placement, dA/dt and right-hand side run beside the previous block's solve. CUDA
        events on the library stream bracket all n steps (pipeline fill and drain included)."""
        its, outer = [], []
        with torch.cuda.stream(stream):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        tickets = [submit(**kw)]
        for _ in range(n - 1):
            tickets.append(submit(**kw))
            it, o = finish(tickets.pop(0))
            its.append(it)
            outer.append(o)
        it, o = finish(tickets.pop(0))
        its.append(it)
        outer.append(o)
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), its, outer

    def timed(n, **kw):
        """Device time of n steps one at a time (CUDA events on the library stream around each,
        L2 flushed before each), with the stage breakdown."""
        ms, its, stages = [], [], np.zeros(5)
        for _ in range(n):
            with torch.cuda.stream(stream):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            step(**kw)
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            its.append(float(d_it.float().mean().item()))
            stages += ctx.stage_times()
        return float(sum(ms)), float(np.mean(its)), stages / n

    clocks = ClockSampler(local).start()
    pipelined(max(3, args.warmup))
    torch.cuda.synchronize()
    launches0 = _native.kernel_launches()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t_region = time.time()
    # An NVTX range around the timed steps lets a profiler capture exactly those launches.
    torch.cuda.nvtx.range_push("timed_steps")
    total_ms, iters, outers = pipelined(args.steps)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    clocks.mark(t_region, time.time())
    if dist is not None:
        dist.barrier()
    launches = _native.kernel_launches() - launches0
    warm_used = d_used.cpu().numpy().tolist()
    warm_rel0 = d_rel0.cpu().numpy().tolist()
    col_iters = float(d_it.float().mean().item())
    # The same blocks on the same GPU: one at a time (with the stage breakdown), without the
    # learned guess (this precision), with FP64 iterative refinement around FP32 PCG, and with
    # plain FP64 PCG; the comparison arms pipelined like the headline.
    n_cmp = max(3, min(args.steps, 8))
    for _ in range(2):
        step()
    seq_ms, _, stage_avg = timed(n_cmp)
    table_info = ctx.coil_table_info()
    # The same configuration with the dipole sum at every node (the reference's dA/dt), and the
    # plain method as the reference runs it: plain FP64 zero-guess PCG over the dipole sum.
    ctx.set_coil_table(False)
    for _ in range(2):
        step()
    _, _, stage_direct = timed(n_cmp)
    pipelined(2)
    direct_ms, _, _ = pipelined(n_cmp)
    pipelined(2, precision=_native.PREC_PLAIN_FP64, warm=False)
    plain_ms, _, _ = pipelined(n_cmp, precision=_native.PREC_PLAIN_FP64, warm=False)
    plain_it = float(d_it.float().mean().item())
    ctx.set_coil_table(use_table)
    pipelined(2, warm=False)
    cold_ms, cold_its, _ = pipelined(n_cmp, warm=False)
    cold_it = float(d_it.float().mean().item())
    proj = None
    if args.warm_start == "on":
        # The Galerkin projection of each block's right-hand sides onto the network's basis (no network).
        pipelined(2, warm="projection")
        torch.cuda.nvtx.range_push("projection_guess")  # lets a profiler capture exactly these blocks
        proj_ms, _, _ = pipelined(n_cmp, warm="projection")
        torch.cuda.nvtx.range_pop()
        proj = (proj_ms, float(d_it.float().mean().item()), [round(v, 5) for v in d_rel0.cpu().numpy().tolist()])
    pipelined(2, precision=_native.PREC_MIXED, warm=False)
    mixed_ms, _, _ = pipelined(n_cmp, precision=_native.PREC_MIXED, warm=False)
    mixed_it = float(d_it.float().mean().item())
    pipelined(2, precision=_native.PREC_PLAIN_FP64, warm=False)
    plain_table_ms, _, _ = pipelined(n_cmp, precision=_native.PREC_PLAIN_FP64, warm=False)
    clocks.stop()
    total_ms, value = job_throughput(total_ms, args.steps, world, dist, dev)
    seq_ms, seq_value = job_throughput(seq_ms, n_cmp, world, dist, dev)
    cold_ms, cold_value = job_throughput(cold_ms, n_cmp, world, dist, dev)
    mixed_ms, mixed_value = job_throughput(mixed_ms, n_cmp, world, dist, dev)
    plain_ms, plain_value = job_throughput(plain_ms, n_cmp, world, dist, dev)
    direct_ms, direct_value = job_throughput(direct_ms, n_cmp, world, dist, dev)
    plain_table_ms, plain_table_value = job_throughput(plain_table_ms, n_cmp, world, dist, dev)

    # End to end through the host C ABI (host buffers in and out), blocks submitted two deep
    # (cunibs_submit_block / cunibs_finish_block), timed by the wall clock around all of them. The
    # wall clock also sees the host, so the run is repeated three times and the median kept.
    n_e2e = max(3, args.steps)
    kw = dict(recovery=args.recovery, warm_start=args.warm_start == "on")
    e2e_runs = []
    for _ in range(3):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        tickets = [ctx.submit_block(coil, centers, handles, dists, 1e6, **kw)]
        for _ in range(n_e2e - 1):
            tickets.append(ctx.submit_block(coil, centers, handles, dists, 1e6, **kw))
            res = ctx.finish_block(tickets.pop(0))
        res = ctx.finish_block(tickets.pop(0))
        e2e_runs.append(time.perf_counter() - t1)
    e2e_s = float(np.median(e2e_runs))
    _, e2e_value = job_throughput(e2e_s * 1e3, n_e2e, world, dist, dev)
    h2d = coil.positions_m.nbytes + coil.moments.nbytes + centers.nbytes + handles.nbytes + dists.nbytes
    d2h = res["transform"].nbytes + res["summary"].nbytes + res["iterations"].nbytes + res["relative_residual"].nbytes

    draws = adm_line = multi = None
    if args.extras == "all":
        draws = conductivity_draws(ctx, coil, centers[:4], handles[:4], dists[:4], args.recovery, stream)
        adm_line = adm_measure(ctx, coil, sites, stream)
        multi = multi_subject_measure(coil, args.recovery) if world == 1 else None
    # The other benchmark configurations, each a line of its own (one GPU; rank 0 of a replica run).
    configs = None
    if args.configs == "all" and rank == 0:
        configs = {}
        if args.warm_start == "on":
            configs["learned_heldout"] = config_learned_heldout(ctx, coil, stream, n_train=args.train)
        configs["small_plain"] = config_small_plain(local, not args.no_cpu_baseline)
        configs["batched_uneven"] = config_batched_uneven()
        configs["conductivity_3_5m"] = config_conductivity_3_5m(local, not args.no_cpu_baseline)

    # Roofline of the SpMV-dominated iteration (solve stage).
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    per_it, per_outer = solve_bytes_per_iteration(ctx, K_BLOCK, args.precision)
    mean_iters = float(np.mean(iters))
    mean_outer = float(np.mean(outers))
    solve_ms = float(stage_avg[3])
    solve_bytes = per_it * mean_iters + per_outer * mean_outer
    achieved = solve_bytes / (solve_ms / 1e3) / 1e9
    # Measured DRAM bytes per PCG iteration (ncu over one timed block, warm L2), beside the
    # algorithmic bytes per iteration: the finest level's working set stays in L2.
    traffic = None
    tp = ROOT / "profiles" / "solve_traffic.json"
    if tp.exists():
        traffic = json.loads(tp.read_text()).get("dram_bytes_per_iteration")
    n_nodes = mesh.n_nodes
    dadt_ms = float(stage_avg[1])
    pair_evals = n_nodes * coil.n_dipoles * K_BLOCK
    line = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": "placements/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(total_ms / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"mixed": "f32 (FP32 PCG/V-cycle/dA-dt) with f64 refinement",
                  "split": "f64 PCG over an f32 V-cycle (f32 dA-dt)", "plain": "f64"}[args.precision]
                 + ("; bf16 tensor-core warm start" if args.warm_start == "on" else ""),
        "data": "synthetic: seeded sphere head and figure-8 coil",
        "arm": ("learned warm start + " if args.warm_start == "on" else "zero guess + ")
               + {"split": "split precision (FP64 PCG over the FP32 SpMV/V-cycle): the mixed-precision scheme "
                           "of the metric as timed here; FP64 refinement around FP32 PCG is the "
                           "mixed_refinement ablation",
                  "mixed": "FP64 refinement around FP32 PCG",
                  "plain": "plain FP64 PCG"}[args.precision],
        "config": config_dict(mesh, {"precision": args.precision, "recovery": args.recovery,
                                     "warm_start": (f"MLP 6-4x{args.hidden}-{args.rank}, {args.train} plain-method training solves, "
                                                    f"{args.epochs} epochs"
                                                    if args.warm_start == "on" else "off"),
                                     "l2": "flushed (256 MB write) before every step's solve",
                                     "pipeline": "blocks submitted two deep: placement/dA-dt/RHS of step i+1 "
                                                 "beside the solve of step i",
                                     "overlap_blocks_per_sm": args.overlap if args.overlap > 0 else 2,
                                     "cheby_degree": int(p.cheby_degree),
                                     "cheby_lower_ratio": float(p.cheby_lower_ratio),
                                     "coil_field": ("table (coil-frame samples, tricubic) beyond 15 mm of the "
                                                    "coil, dipole sum nearer" if use_table
                                                    else "dipole sum at every node"),
                                     "parallelism": f"replicas x{world}"}),
        "e2e": {"value": round(e2e_value, 3), "unit": "placements/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "runs_s": [round(x, 5) for x in e2e_runs],
                "what": f"median of 3 wall-clock runs of {n_e2e} blocks through the host C ABI"},
        "gpu_launches": int(launches),
        "vs_plain_fp64": {"value": round(plain_value, 3), "unit": "placements/s",
                          "iterations": plain_it, "ratio": round((plain_ms / n_cmp) / (total_ms / args.steps), 3),
                          "what": "plain FP64 zero-guess PCG with the dipole sum at every node (the "
                                  "reference's method), same blocks, same pipeline, same GPU"},
        "ablation": {"zero_guess": {"value": round(cold_value, 3), "iterations": cold_it,
                                    "what": f"{args.precision}, no learned guess"},
                     "mixed_refinement_zero_guess": {"value": round(mixed_value, 3), "iterations": mixed_it,
                                                     "what": "FP32 PCG + FP32 V-cycle inside FP64 refinement"},
                     "dipole_sum_every_node": {"value": round(direct_value, 3),
                                               "what": "this configuration with the coil table off"},
                     "plain_fp64_zero_guess_table": {"value": round(plain_table_value, 3),
                                                     "what": "plain FP64 zero-guess PCG with the coil table"},
                     "one_block_at_a_time": {"value": round(seq_value, 3),
                                             "what": "this configuration without the two-deep pipeline"},
                     "basis_projection_guess": None if proj is None else {
                         "value": round(job_throughput(proj[0], n_cmp, world, dist, dev)[1], 3),
                         "iterations": proj[1], "init_relres": proj[2],
                         "what": "Galerkin projection of the right-hand sides onto the learned basis, no network"},
                     "this_run": {"warm_start": args.warm_start, "iterations": col_iters,
                                  "warm_used": warm_used, "init_relres": [round(v, 5) for v in warm_rel0]}},
        "warm_start": warm_stats,
        "roofline": {"bound": "hbm", "kernel": "block PCG solve stage (SpMV-dominated iteration)",
                     "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                     "frac": round(achieved / hbm_peak, 4), "traffic": traffic,
                     "traffic_unit": "DRAM bytes per PCG iteration (ncu, warm L2)",
                     "bytes_per_iteration": per_it, "iterations": mean_iters, "outer_steps": mean_outer,
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
        "stages_ms": {k: round(float(v), 4) for k, v in zip(["place", "dadt", "rhs", "solve", "post"], stage_avg)},
        "dadt": {"ms": round(dadt_ms, 4), "ms_dipole_sum": round(float(stage_direct[1]), 4),
                 "pair_evals_per_step_dipole_sum": int(pair_evals),
                 "gpair_per_s_dipole_sum": round(pair_evals / (float(stage_direct[1]) / 1e3) / 1e9, 2),
                 "table": {"in_use": table_info["in_use"], "points": table_info["points"],
                           "layers": table_info["layers"], "check_rel_l2": table_info["check_rel_l2"],
                           "near_fraction": (round(table_info["last_near_nodes"] / table_info["last_node_placements"], 5)
                                             if table_info["last_near_nodes"] >= 0 else None)}},
        "setup_s": round(setup_s, 3),
        "conductivity_draws": draws,
        "adm": adm_line,
        "multi_subject": multi,
        "configs": configs,
        "clocks": clocks.summary(),
    }
    if rank == 0 and not args.no_cpu_baseline:
        # The headline path's fields of the same block (learned guess, this precision), outside the
        # timed region, for the parity check against the FP64 oracle.
        gpu = ctx.solve_block(coil, centers, handles, dists, 1e6, magnitude=True, recovery=args.recovery,
                              warm_start=args.warm_start == "on")
        line["cpu_baseline"], line["parity"] = cpu_baseline(mesh, coil, sites, args.recovery, gpu)
    if dist is not None:
        dist.destroy_process_group()
    return line if rank == 0 else None


def conductivity_draws(ctx, coil, centers, handles, dists, recovery, stream, n_draws=12, seed=0) -> dict:
    """Conductivity Monte Carlo on the same mesh: every tissue's conductivity lognormal with the
    table value as median and log-sd 0.25 (seeded), one block of the first 4 placements. The study
    (cunibs_sigma_begin once, then cunibs_sigma_draw per draw: operator components, coil field held,
    sensitivity-subspace guess) against a keep-coarse re-assembly and a zero-guess block solve per
    draw. Device time on the library stream around all draws (host API, outputs copied back each
    draw); L2 not flushed."""
    import torch

    from cunibs_b200.uq import nominal_sigma_table

    nominal = nominal_sigma_table()
    tags = tuple(range(1, 11))
    rng = np.random.default_rng(seed)
    sig = nominal[list(tags)] * np.exp(0.25 * rng.standard_normal((n_draws, len(tags))))
    k = centers.shape[0]

    def device_ms(fn):
        with torch.cuda.stream(stream):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        out = fn()
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), out

    def keep_coarse():
        its = []
        for s in sig:
            table = nominal.copy()
            table[list(tags)] = s
            ctx.set_conductivity(table, keep_coarse=True)
            its.append(ctx.solve_block(coil, centers, handles, dists, 1e6, recovery=recovery)["iterations"].mean())
        ctx.set_conductivity(nominal, keep_coarse=True)
        return its

    def study():
        its, rel0 = [], []
        # An NVTX range around the draws lets a profiler capture exactly their launches.
        torch.cuda.nvtx.range_push("conductivity_draws")
        for s in sig:
            r = ctx.sigma_draw(s)
            its.append(r["iterations"].mean())
            rel0.append(float(r["init_relres"].max()))
        torch.cuda.nvtx.range_pop()
        return its, rel0

    old_ms, old_its = device_ms(keep_coarse)
    # Opening the study twice, with the wall clock beside the device time of each: a first call that
    # alone is slow, or a host time far above the device time, locates one-off costs.
    begin_runs = []
    for rep in range(2):
        t0 = time.perf_counter()
        begin_ms, ranks = device_ms(lambda: ctx.sigma_begin(coil, centers, handles, dists, 1e6, nominal, tags,
                                                            recovery=recovery))
        begin_runs.append((round(begin_ms, 3), round(1e3 * (time.perf_counter() - t0), 3), ctx.phase_times()))
        if rep == 0:
            ctx.sigma_end()
    guesses = {}
    try:
        new_ms, (new_its, rel0) = device_ms(study)
        # The same draws from the nominal potential alone (what a predictor of the nominal solution
        # per pose can give at best) and from zero, on the same kept hierarchy.
        for mode in ("nominal", "zero"):
            ctx.sigma_set_guess(mode)
            g_ms, (g_its, g_rel0) = device_ms(study)
            guesses[mode] = {"ms_per_draw": round(g_ms / n_draws, 4), "iterations": round(float(np.mean(g_its)), 2),
                             "init_relres_max": round(max(g_rel0), 6)}
        ctx.sigma_set_guess("subspace")
    finally:
        ctx.sigma_end()
    return {"what": f"{n_draws} draws x {k} placements, 10 tissues lognormal (median = table, log-sd 0.25)",
            "study_ms_per_draw": round(new_ms / n_draws, 4), "study_iterations": round(float(np.mean(new_its)), 2),
            "study_begin_ms": round(begin_ms, 3), "study_begin_device_host_ms": begin_runs,
            "subspace_rank": ranks.tolist(),
            "guess_init_relres_max": round(max(rel0), 6),
            "keep_coarse_zero_guess_ms_per_draw": round(old_ms / n_draws, 4),
            "keep_coarse_iterations": round(float(np.mean(old_its)), 2),
            "placement_draws_per_s": round(k * n_draws / (new_ms / 1e3), 2),
            "ratio": round(old_ms / new_ms, 3),
            "guess_comparison": {"subspace": {"ms_per_draw": round(new_ms / n_draws, 4),
                                              "iterations": round(float(np.mean(new_its)), 2),
                                              "init_relres_max": round(max(rel0), 6)}, **guesses}}


def adm_measure(ctx, coil, sites, stream) -> dict:
    """Auxiliary dipole method on the same head: a magnitude target 18 mm below the vertex (three
    adjoint solves in one block at rel.res 1e-9), the reciprocity field on a 3 mm grid covering the
    coil at any rotation on the 8 sites, then the target field of 8 sites x 360 rotations by grid
    interpolation, and the optimiser over the 8 sites. Device time on the library stream (CUDA
    events around each host call)."""
    import torch

    from cunibs_b200 import adm

    def device_ms(fn):
        with torch.cuda.stream(stream):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        out = fn()
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), out

    centers = np.stack([c for c, _ in sites])
    target = adm.resolve_target(ctx, adm.Target([0.0, 0.0, 72.0]))
    adj_ms, adjoint = device_ms(lambda: adm.solve_adjoint(ctx, target))
    grid = adm._coverage_grid(ctx, coil, centers, 4.0, 3.0, 8.0)
    torch.cuda.nvtx.range_push("adm_qfield")
    q_runs = []
    for _ in range(2):  # the first and a repeat, device and wall clock (one-off costs show in the first)
        t0 = time.perf_counter()
        q_ms, recip = device_ms(lambda: adm.sample_qfield(adjoint, grid))
        q_runs.append((round(q_ms, 3), round(1e3 * (time.perf_counter() - t0), 3)))
    torch.cuda.nvtx.range_pop()
    pairs = grid.n_points * ctx.n_nodes * target.directions.shape[0]
    # 360 in-plane rotations per site: handle points around each site's own coil frame.
    angles = np.radians(np.arange(360.0))
    T0, _ = ctx.place(centers, np.stack([h for _, h in sites]), np.full(len(sites), 4.0))
    rot = np.cos(angles)[None, :, None] * T0[:, None, :3, 1] + np.sin(angles)[None, :, None] * T0[:, None, :3, 0]
    all_c = np.repeat(centers, 360, axis=0)
    T, _ = ctx.place(all_c, all_c + 50.0 * rot.reshape(-1, 3), np.full(all_c.shape[0], 4.0))
    adm.evaluate_frames(recip, coil, T[:8], 1e6)  # warm-up
    torch.cuda.nvtx.range_push("adm_evaluate")  # lets a profiler capture exactly this launch
    ev_ms, e = device_ms(lambda: adm.evaluate_frames(recip, coil, T, 1e6))
    torch.cuda.nvtx.range_pop()
    opt_ms, res = device_ms(lambda: adm.optimize_placement(recip, coil, centers, n_samples=9))
    out = {"what": "magnitude target (3 adjoint directions), 8 sites; grid 3 mm covering any rotation",
           "adjoint_ms": round(adj_ms, 3), "adjoint_iterations": adjoint.iterations.tolist(),
           "grid_points": int(grid.n_points), "qfield_ms": round(q_ms, 3), "qfield_device_host_ms": q_runs,
           "qfield_gpair_per_s": round(pairs / (q_ms / 1e3) / 1e9, 1),
           "evaluate_placements": int(T.shape[0]), "evaluate_ms": round(ev_ms, 3),
           "evaluate_placements_per_s": round(T.shape[0] / (ev_ms / 1e3), 1),
           "optimize_ms": round(opt_ms, 3), "best_objective_v_per_m": round(res.best_objective, 4),
           "sweep_max_v_per_m": round(float(np.linalg.norm(e, axis=1).max()), 4)}
    adjoint.handle.close()
    return out


def multi_subject_measure(coil, recovery, n_place=16, repeats=3) -> dict:
    """Three subjects of uneven size (0.3M, 0.6M and 1.0M tetrahedra, the same 10-tissue sphere at
    3.93, 3.12 and 2.63 mm) swept with 16 placements each: one after another, then side by side from
    one host thread per subject (cunibs_b200.batch). Wall clock around each whole run (results
    copied to the host), three repetitions of each alternating, the median kept; the per-subject results
    of the two runs are checked bitwise equal."""
    from cunibs_b200 import Placement, Subject
    from cunibs_b200.batch import SubjectJob, simulate_subjects

    rng = np.random.default_rng(7)
    sites = []
    for _ in range(n_place):
        th, ph = rng.uniform(0.0, np.radians(40.0)), rng.uniform(0.0, 2 * np.pi)
        c = 90.0 * np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
        sites.append(Placement(c, c + 50.0 * np.array([-np.sin(ph), np.cos(ph), 0.0])))
    subjects = [Subject(sphere_head(h, 90.0, EIGHT_SHELLS, (EYE_CAP, MUSCLE_CAP), jitter_mm=0.2, seed=0), tolerance=TOL)
                for h in (3.93, 3.12, 2.63)]
    jobs = [SubjectJob(s, coil, sites, options=dict(recovery=recovery, magnitude=True)) for s in subjects]
    for j in jobs:  # contexts, recovery operators and loop graphs built outside the timing
        list(j.subject.iter_simulate(coil, sites[:8], recovery=recovery))
    seq, con, same = [], [], True
    for _ in range(repeats):
        t0 = time.perf_counter()
        alone = [list(j.subject.iter_simulate(coil, sites, recovery=recovery, magnitude=True)) for j in jobs]
        seq.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        together = simulate_subjects(jobs)
        con.append(time.perf_counter() - t0)
        same = same and all(np.array_equal(a.magnE, b.magnE) for ra, rb in zip(alone, together) for a, b in zip(ra, rb))
    seq_s, con_s = float(np.median(seq)), float(np.median(con))
    out = {"what": "3 subjects (0.3M / 0.6M / 1.0M tets) x 16 placements, harmonic recovery, |E| retained",
           "n_tets": [int(s.context.n_tets) for s in subjects], "sequential_s": round(seq_s, 4),
           "concurrent_s": round(con_s, 4), "repeats_s": {"sequential": [round(t, 4) for t in seq],
                                                          "concurrent": [round(t, 4) for t in con]},
           "placements_per_s_sequential": round(3 * n_place / seq_s, 1),
           "placements_per_s_concurrent": round(3 * n_place / con_s, 1), "speedup": round(seq_s / con_s, 3),
           "bitwise_equal": bool(same)}
    for s in subjects:
        s.free()
    return out


def _device_ms(stream, fn):
    """CUDA-event time of fn() on the library stream (events on either side, synchronised)."""
    import torch

    with torch.cuda.stream(stream):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
    out = fn()
    with torch.cuda.stream(stream):
        e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1), out


def _gm_parity(gpu_magnE, gpu_peak, ref, tags) -> tuple[float, float]:
    gm = tags == 2
    a, b = np.asarray(gpu_magnE, np.float64)[gm], np.asarray(ref["magnE"][0], np.float64)[gm]
    return (float(np.linalg.norm(a - b) / np.linalg.norm(b)),
            float(abs(gpu_peak - ref["summary"][0][0]) / ref["summary"][0][0]))


def config_small_plain(local: int, with_oracle: bool, reps: int = 10) -> dict:
    """The plain-method small case: 64^3 lattice at 3 mm clipped to r <= 90 mm (five shells), a
    figure-8 of 2 x 512 z-dipoles 4 mm above the vertex, dI/dt 1e6, one placement per block
    (block_k 1), relative residual 1e-10. Context set-up time, then device time of `reps` one-placement
    blocks (host C ABI, harmonic recovery) for plain FP64 and the split default; parity of each
    against the FP64 oracle at 1e-12 (rank 0)."""
    import torch

    from cunibs_b200 import _native
    from cunibs_b200.synthetic import FIVE_SHELLS

    mesh = sphere_head(3.0, 90.0, FIVE_SHELLS, cells=64)
    coil = figure8_coil(512)
    c = np.array([[0.0, 0.0, 90.0]])
    h = c + [0.0, 50.0, 0.0]
    out = {"what": "64^3 x 3 mm sphere (5 shells), 2x512 z-dipole figure-8 4 mm above the vertex, "
                   "k = 1, rel.res 1e-10, harmonic recovery", "n_tets": int(mesh.n_tets)}
    ref = None
    if with_oracle:
        from oracle import Oracle

        orc = Oracle(mesh)
        ref = orc.solve(coil, c, h, [4.0], 1e6, tolerance=1e-12, recovery="harmonic")
    for name, prec in (("plain_fp64", _native.PREC_PLAIN_FP64), ("split", _native.PREC_SPLIT)):
        p = _native.default_params()
        p.device = local
        p.tolerance = 1e-10
        p.precision = prec
        t0 = time.perf_counter()
        ctx = _native.Context(mesh.nodes_mm, mesh.tet_nodes, mesh.tet_tags, mesh.skin_tris, p)
        torch.cuda.synchronize()
        setup_s = time.perf_counter() - t0
        stream = torch.cuda.ExternalStream(ctx.stream(), device=local)
        first = ctx.solve_block(coil, c, h, [4.0], 1e6, magnitude=True, recovery="harmonic")  # recovery operator
        ms, its = _device_ms(stream, lambda: [ctx.solve_block(coil, c, h, [4.0], 1e6, recovery="harmonic")[
            "iterations"][0] for _ in range(reps)])
        row = {"setup_s": round(setup_s, 3), "placements_per_s": round(reps / (ms / 1e3), 2),
               "ms_per_placement": round(ms / reps, 3), "iterations": int(its[0])}
        if ref is not None:
            # The oracle's element order is the context's (the same Morton layout, bit for bit).
            rel, peak = _gm_parity(first["magnE"][0], first["summary"][0][0], ref, ctx.array("tet_tags"))
            row["parity"] = {"gm_rel_l2": float(f"{rel:.3e}"), "peak_rel": float(f"{peak:.3e}"), "bar": 1e-5}
        out[name] = row
        ctx.close()
    return out


def config_batched_uneven(n_place: int = 64) -> dict:
    """Four sphere heads of uneven size (0.3M, 0.9M, 1.8M and 3.5M tets at outer radii 85, 88, 92 and
    95 mm), 64 placements each (uniform random centres on the scalp cap above z = 40 mm, handle
    azimuth uniform), harmonic recovery: each subject's block width and dA/dt overlap autotuned (widths
    4, 8, 16) on its own first 16 placements, then the four sweeps one after another and side by side
    (one host thread per subject). Wall clock around each whole run, results copied to the host; the
    side-by-side results are checked bitwise against the sequential ones."""
    from cunibs_b200 import Placement, Subject
    from cunibs_b200.batch import SubjectJob, simulate_subjects
    from cunibs_b200.synthetic import cap_placements

    coil = figure8_coil(2048)
    specs = [(3.71, 85.0, 11), (2.68, 88.0, 12), (2.23, 92.0, 13), (1.83, 95.0, 14)]
    subjects, jobs, tuned = [], [], []
    for spacing, radius, seed in specs:
        mesh = sphere_head(spacing, radius, EIGHT_SHELLS, (EYE_CAP, MUSCLE_CAP), jitter_mm=0.2, seed=0)
        subj = Subject(mesh, tolerance=TOL)
        sites = [Placement(cc, hh) for cc, hh in cap_placements(radius, n_place, 40.0, seed=seed)]
        res = subj.autotune(coil, sites[:16], widths=(4, 8, 16), overlaps=(1, 2), repeats=1)
        tuned.append({"block_k": res.block_k, "overlap": res.overlap_blocks_per_sm})
        subjects.append(subj)
        jobs.append(SubjectJob(subj, coil, sites, options=dict(recovery="harmonic", magnitude=True)))
    for j in jobs:  # loop graphs of the tuned width captured outside the timing
        list(j.subject.iter_simulate(coil, j.placements[:16], recovery="harmonic"))
    t0 = time.perf_counter()
    alone = [list(j.subject.iter_simulate(coil, j.placements, recovery="harmonic", magnitude=True)) for j in jobs]
    seq_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    together = simulate_subjects(jobs)
    con_s = time.perf_counter() - t0
    same = all(np.array_equal(a.magnE, b.magnE) for ra, rb in zip(alone, together) for a, b in zip(ra, rb))
    total = n_place * len(jobs)
    out = {"what": "4 subjects (0.3/0.9/1.8/3.5M tets, r 85-95 mm) x 64 cap placements, autotuned width "
                   "and overlap per subject, harmonic recovery, |E| retained",
           "n_tets": [int(s.context.n_tets) for s in subjects], "tuned": tuned,
           "sequential_s": round(seq_s, 4), "concurrent_s": round(con_s, 4),
           "placements_per_s_sequential": round(total / seq_s, 1),
           "placements_per_s_concurrent": round(total / con_s, 1), "bitwise_equal": bool(same)}
    for s in subjects:
        s.free()
    return out


def config_learned_heldout(ctx, coil, stream, n_held: int = 1024, n_train: int = 0) -> dict:
    """The learned warm start on held-out poses: 1024 random cap poses (a seed the training never
    used), solved in blocks of 8 to rel.res 1e-8 with the installed network's guess and with the zero
    guess, both two deep; mean PCG iterations, the guess's initial residual, and device-timed
    placements/s of each."""
    from cunibs_b200.synthetic import cap_placements

    poses = cap_placements(90.0, n_held, 40.0, seed=991)
    c = np.stack([p[0] for p in poses])
    h = np.stack([p[1] for p in poses])
    d = np.full(K_BLOCK, 4.0)

    def sweep(warm):
        its, rel0 = [], []
        tickets = [ctx.submit_block(coil, c[:K_BLOCK], h[:K_BLOCK], d, 1e6, warm_start=warm)]
        for b in range(1, n_held // K_BLOCK + 1):
            if b < n_held // K_BLOCK:
                s = slice(b * K_BLOCK, (b + 1) * K_BLOCK)
                tickets.append(ctx.submit_block(coil, c[s], h[s], d, 1e6, warm_start=warm))
            r = ctx.finish_block(tickets.pop(0))
            its += r["iterations"].tolist()
            rel0 += r["init_relres"].tolist()
        return its, rel0

    sweep(True)  # graphs
    ms_w, (its_w, rel_w) = _device_ms(stream, lambda: sweep(True))
    ms_z, (its_z, _) = _device_ms(stream, lambda: sweep(False))
    return {"what": f"{n_held} held-out cap poses, blocks of 8, rel.res 1e-8, harmonic recovery off (summary only)",
            "n_train": n_train, "iterations_learned": round(float(np.mean(its_w)), 3),
            "iterations_zero_guess": round(float(np.mean(its_z)), 3),
            "init_relres_median": round(float(np.median(rel_w)), 5), "init_relres_max": round(float(np.max(rel_w)), 5),
            "guess_kept_fraction": round(float(np.mean(np.array(rel_w) < 1.0)), 4),
            "placements_per_s_learned": round(n_held / (ms_w / 1e3), 1),
            "placements_per_s_zero_guess": round(n_held / (ms_z / 1e3), 1)}


def config_conductivity_3_5m(local: int, with_oracle: bool, n_draws: int = 512, seed: int = 0) -> dict:
    """The conductivity study at 3.5M tets: the ten-tissue sphere at 1.73 mm (90 mm), four cap
    placements, 512 draws with every tissue lognormal (median = table value, log-sd 0.25), mixed
    precision (FP64 PCG over the FP32 V-cycle) to rel.res 1e-8, harmonic recovery. Device time of
    the draws; the distribution of each placement's gray-matter peak |E| and p99 over the draws; the
    first two draws of the first placement against the FP64 oracle assembled with their tables (rank 0)."""
    import torch

    from cunibs_b200 import _native
    from cunibs_b200.synthetic import cap_placements
    from cunibs_b200.uq import nominal_sigma_table

    mesh = sphere_head(1.73, 90.0, EIGHT_SHELLS, (EYE_CAP, MUSCLE_CAP), jitter_mm=0.2, seed=0)
    coil = figure8_coil(2048)
    poses = cap_placements(90.0, 4, 40.0, seed=21)
    c = np.stack([p[0] for p in poses])
    h = np.stack([p[1] for p in poses])
    p = _native.default_params()
    p.device = local
    p.tolerance = TOL
    ctx = _native.Context(mesh.nodes_mm, mesh.tet_nodes, mesh.tet_tags, mesh.skin_tris, p)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=local)
    nominal = nominal_sigma_table()
    tags = tuple(range(1, 11))
    rng = np.random.default_rng(seed)
    sig = nominal[list(tags)] * np.exp(0.25 * rng.standard_normal((n_draws, len(tags))))
    ctx.solve_block(coil, c, h, [4.0] * 4, 1e6, recovery="harmonic")  # recovery operator and graphs
    begin_ms, _ = _device_ms(stream, lambda: ctx.sigma_begin(coil, c, h, [4.0] * 4, 1e6, nominal, tags,
                                                               magnitude=True, recovery="harmonic"))
    first = []
    try:
        def draws():
            peaks, p99, its, resetups = [], [], [], 0
            for i, s in enumerate(sig):
                r = ctx.sigma_draw(s)
                peaks.append(r["summary"][:, 0].copy())
                p99.append(r["summary"][:, 12].copy())
                its.append(float(r["iterations"].mean()))
                resetups += int(r["resetup"])
                if i < 2:
                    first.append((r["magnE"][0].copy(), float(r["summary"][0][0])))
            return np.array(peaks), np.array(p99), its, resetups
        ms, (peaks, p99, its, resetups) = _device_ms(stream, draws)
    finally:
        ctx.sigma_end()
    q = lambda a: {"mean": float(f"{a.mean():.6g}"), "std": float(f"{a.std():.6g}"),  # noqa: E731
                   "p5": float(f"{np.percentile(a, 5):.6g}"), "p50": float(f"{np.percentile(a, 50):.6g}"),
                   "p95": float(f"{np.percentile(a, 95):.6g}")}
    out = {"what": f"3.5M-tet ten-tissue head, 4 cap placements x {n_draws} draws (all 10 tissues lognormal, "
                   "log-sd 0.25), rel.res 1e-8, harmonic recovery", "n_tets": int(mesh.n_tets),
           "begin_ms": round(begin_ms, 2), "ms_per_draw": round(ms / n_draws, 3),
           "draws_per_s": round(n_draws / (ms / 1e3), 2), "placement_draws_per_s": round(4 * n_draws / (ms / 1e3), 1),
           "iterations_mean": round(float(np.mean(its)), 2), "full_resetups": resetups,
           "gm_peak_magnE": [q(peaks[:, j]) for j in range(4)], "gm_p99_magnE": [q(p99[:, j]) for j in range(4)]}
    if with_oracle:
        from oracle import Oracle, OracleParams

        worst_rel, worst_peak = 0.0, 0.0
        tet_tags = ctx.array("tet_tags")
        for i, (m, pk) in enumerate(first):
            table = nominal.copy()
            table[list(tags)] = sig[i]
            ref = Oracle(mesh, OracleParams(sigma_by_tag=tuple(table))).solve(
                coil, c[:1], h[:1], [4.0], 1e6, tolerance=1e-12, recovery="harmonic")
            rel, peak = _gm_parity(m, pk, ref, tet_tags)
            worst_rel, worst_peak = max(worst_rel, rel), max(worst_peak, peak)
        out["parity_first_draws"] = {"draws": len(first), "gm_rel_l2": float(f"{worst_rel:.3e}"),
                                     "peak_rel": float(f"{worst_peak:.3e}"), "bar": 1e-5}
    ctx.close()
    return out


def cpu_baseline(mesh, coil, sites, recovery, gpu, n_place=1) -> tuple[dict, dict]:
    """The FP64 CPU restatement (oracle/) on this host's cores: one placement of the same workload,
    timed; then the parity check of the GPU block ``gpu`` (the headline path's fields) against the
    oracle solved to 1e-12 on every placement of the block: gray-matter |E| relative L2 and peak |E|
    relative error, the product's stated bar being 1e-5 for both."""
    from oracle import Oracle

    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    orc = Oracle(mesh)
    if recovery != "raw":
        orc.recovery(recovery)  # per-subject setup, like the operator build
    setup = time.perf_counter() - t0
    c = np.stack([s[0] for s in sites[:n_place]])
    h = np.stack([s[1] for s in sites[:n_place]])
    t1 = time.perf_counter()
    orc.solve(coil, c, h, np.full(n_place, 4.0), 1e6, tolerance=TOL, recovery=recovery)
    dt = time.perf_counter() - t1
    base = {"value": round(n_place / dt, 4), "unit": "placements/s", "cores": threads, "kind": "port",
            "cpu_model": cpu_model(),
            "sample": f"{n_place} placement(s) of the same workload, FP64 AMG-PCG to 1e-8 (setup {setup:.1f} s excluded)"}

    k = len(sites)
    ref = orc.solve(coil, np.stack([s[0] for s in sites]), np.stack([s[1] for s in sites]), np.full(k, 4.0), 1e6,
                    tolerance=PARITY_ORACLE_TOL, recovery=recovery)
    gm = mesh.tet_tags == 2
    rel, peak = [], []
    for i in range(k):
        a, b = gpu["magnE"][i].astype(np.float64)[gm], ref["magnE"][i].astype(np.float64)[gm]
        rel.append(float(np.linalg.norm(a - b) / np.linalg.norm(b)))
        peak.append(float(abs(gpu["summary"][i][0] - ref["summary"][i][0]) / ref["summary"][i][0]))
    parity = {"what": f"GPU block (this run's precision and guess, rel.res {TOL:g}) vs FP64 oracle "
                      f"(rel.res {PARITY_ORACLE_TOL:g}), {recovery} recovery, all {k} placements",
              "gm_rel_l2": max(rel), "peak_rel": max(peak), "oracle_tol": PARITY_ORACLE_TOL, "bar": 1e-5,
              "gm_rel_l2_per_placement": [float(f"{v:.3e}") for v in rel],
              "peak_rel_per_placement": [float(f"{v:.3e}") for v in peak],
              "pass": bool(max(rel) <= 1e-5 and max(peak) <= 1e-5)}
    return base, parity


def cpu_model() -> str:
    """The host CPU's model name (first "model name" of /proc/cpuinfo), or the platform's answer."""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform

    return platform.processor() or "unknown"


def run_reference(args) -> dict | None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    mesh, coil, sites = workload()
    from oracle import Oracle

    threads = os.cpu_count() or 1
    orc = Oracle(mesh)
    if args.recovery != "raw":
        orc.recovery(args.recovery)
    c = np.stack([s[0] for s in sites])
    h = np.stack([s[1] for s in sites])
    for i in range(args.warmup):
        j = i % len(sites)
        orc.solve(coil, c[j:j + 1], h[j:j + 1], [4.0], 1e6, tolerance=TOL, recovery=args.recovery)
    times = []
    for i in range(args.steps):
        j = i % len(sites)
        t1 = time.perf_counter()
        orc.solve(coil, c[j:j + 1], h[j:j + 1], [4.0], 1e6, tolerance=TOL, recovery=args.recovery)
        times.append(time.perf_counter() - t1)
    value = len(times) / sum(times)
    return {
        "metric": METRIC, "value": round(value, 4), "unit": "placements/s", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * sum(times) / len(times), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "impl": "reference",
        "data": "synthetic: seeded sphere head and figure-8 coil",
        "config": config_dict(mesh, {"precision": "f64", "recovery": args.recovery}),
        "cpu_baseline": {"value": round(value, 4), "unit": "placements/s", "cores": threads, "kind": "port",
                         "cpu_model": cpu_model(),
                         "sample": "one placement per step (the workload's 8 sites in turn), FP64 AMG-PCG to 1e-8"},
        "e2e": {"value": round(value, 4), "unit": "placements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["split", "mixed", "plain"], default="split")
    ap.add_argument("--recovery", choices=["harmonic", "spr_tissue", "spr_global", "raw"], default="harmonic")
    ap.add_argument("--warm-start", choices=["on", "off"], default="on")
    ap.add_argument("--train", type=int, default=8192, help="training solves of the warm-start network")
    ap.add_argument("--rank", type=int, default=256, help="reduced-basis size the network predicts")
    ap.add_argument("--hidden", type=int, default=512, help="width of the warm-start network's hidden layers")
    ap.add_argument("--epochs", type=int, default=400, help="training epochs of the warm-start network")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cheby-lower-ratio", type=float, default=0.0,
                    help="Chebyshev smoother's interval [lambda_max / ratio, lambda_max] (0: the reference's 12)")
    ap.add_argument("--cheby-degree", type=int, default=0,
                    help="Chebyshev smoother degree of the V-cycle (0: the reference's default, 2)")
    ap.add_argument("--coil-field", choices=["table", "direct"], default="table",
                    help="dA/dt from the coil table beyond 15 mm of the coil (default) or the dipole sum everywhere")
    ap.add_argument("--overlap", type=int, default=0,
                    help="dA/dt blocks per SM beside a running solve (0: the context's default, 2)")
    ap.add_argument("--extras", choices=["all", "none"], default="all",
                    help="also measure the conductivity draws, the auxiliary dipole method and the side-by-side "
                         "subjects on the headline head")
    ap.add_argument("--configs", choices=["all", "none"], default="all",
                    help="also measure the other benchmark configurations (small plain case, uneven subjects, "
                         "held-out learned guess, conductivity study at 3.5M tets)")
    args = ap.parse_args()
    line = run_reference(args) if args.impl == "reference" else run_ours(args)
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()

"""Autotuning of the sweep settings that leave every result bit unchanged.

A sweep's results do not depend on the block width (how many placements share one block solve,
up to the native solver's 16)
nor on how many dA/dt blocks per SM run beside the previous block's solve (both tested bit for
bit), so those two are chosen by measurement on the caller's own subject, coil and placements:
each candidate pair runs the pipelined sweep of ``Subject.iter_simulate`` and the fastest is kept
as the subject's default. The smoother degree and the lanes per SpMV row are not tuned: they
change the arithmetic (the order of a row's sum, the smoothing polynomial), and a result that
depended on a timing run would no longer be reproducible run to run; the lanes per row are
chosen from each operator's shape instead.
"""

from __future__ import annotations

import time
from collections.abc import Sequence
from dataclasses import dataclass, field

from .fem import SWEEP_MAX_BLOCK

OVERLAP_MAX = 16


@dataclass
class TuneResult:
    block_k: int
    overlap_blocks_per_sm: int
    placements_per_s: dict[tuple[int, int], float] = field(default_factory=dict)  # (block_k, overlap) -> rate


def autotune(subject, coil, placements: Sequence, *, widths: Sequence[int] = (2, 4, 8, 16),
             overlaps: Sequence[int] = (1, 2, 3, 4), recovery: str = "harmonic", repeats: int = 2,
             didt: float = 1e6, apply: bool = True) -> TuneResult:
    """Time every (block width, overlap) pair on ``placements`` (wall clock over the pipelined
    sweep, summary only, best of ``repeats`` after one warm-up) and, with ``apply``, make the best
    the subject's default for ``block_k=None`` sweeps and its context's dA/dt overlap."""
    widths = [int(w) for w in widths]
    overlaps = [int(o) for o in overlaps]
    if not widths or any(w < 1 or w > SWEEP_MAX_BLOCK for w in widths):
        raise ValueError(f"block widths must be in [1, {SWEEP_MAX_BLOCK}]")
    if not overlaps or any(o < 1 or o > OVERLAP_MAX for o in overlaps):
        raise ValueError(f"overlaps must be in [1, {OVERLAP_MAX}]")
    if repeats < 1:
        raise ValueError("repeats must be at least 1")
    sites = list(placements)
    if not sites:
        raise ValueError("autotune needs at least one placement")
    ctx = subject.context
    rates: dict[tuple[int, int], float] = {}
    old_k = subject.block_k_default
    try:
        for o in overlaps:
            ctx.set_overlap(o)
            for w in widths:
                # A block_k=None sweep at this width (an explicit block_k stops at MAX_BLOCK).
                subject.set_sweep_defaults(block_k=w)
                best = float("inf")
                for rep in range(repeats + 1):  # the first run captures this width's loop graphs
                    t0 = time.perf_counter()
                    for _ in subject.iter_simulate(coil, sites, didt, recovery=recovery):
                        pass
                    dt = time.perf_counter() - t0
                    if rep:
                        best = min(best, dt)
                rates[(w, o)] = len(sites) / best
    finally:
        subject.set_sweep_defaults(block_k=old_k)
    (bw, bo) = max(rates, key=lambda key: (rates[key], key[0], -key[1]))
    if apply:
        subject.set_sweep_defaults(block_k=bw, overlap_blocks_per_sm=bo)
    else:
        ctx.set_overlap(subject.overlap_blocks_per_sm)
    return TuneResult(block_k=bw, overlap_blocks_per_sm=bo, placements_per_s=rates)

"""Solver constants, the convergence error and recovery-mode validation (reference fem/solve.py:52-57,
368-405,501-505; fem/recovery.py:70-125)."""

from __future__ import annotations

import re
from typing import NamedTuple

DEFAULT_TOLERANCE = 1e-6
DEFAULT_MAX_ITERS = 2000
BLOCK_SIZES = (1, 2, 4, 8, 16)
# Widest block the Subject API chunks a sweep into for an explicit block_k (the reference's
# MAX_BLOCK is 8).
MAX_BLOCK = 8
# Widest block the native solver takes (cunibs_solve_opts.block_width). A sweep called with
# block_k=None may run this wide once the autotuner has chosen it: a placement's result does not
# depend on the block width, bit for bit.
SWEEP_MAX_BLOCK = 16

TISSUE_CONDUCTIVITY: dict[int, float] = {
    1: 0.126, 2: 0.275, 3: 1.654, 4: 0.010, 5: 0.465, 6: 0.5, 7: 0.008, 8: 0.025, 9: 0.6, 10: 0.16,
}
GM_TAG = 2

RECOVERY_MODES = ("raw", "spr_global", "spr_tissue", "harmonic")


def validate_recovery(recovery: str) -> str:
    if recovery not in RECOVERY_MODES:
        raise ValueError(f"Unknown recovery {recovery!r}; use one of {', '.join(map(repr, RECOVERY_MODES))}.")
    return recovery


class SolverConvergenceError(RuntimeError):
    """The PCG missed tolerance even after an FP64 retry (reference fem/solve.py:368-392)."""

    def __init__(self, iterations: int, relative_residual: float, tolerance: float, *, column: int | None = None,
                 message: str | None = None) -> None:
        where = "" if column is None else f" (column {column} of the block)"
        super().__init__(message or (f"PCG did not converge{where}: {iterations} iterations, relative residual "
                                     f"{relative_residual:.3e} > tolerance {tolerance:.3e}"))
        self.iterations = iterations
        self.relative_residual = relative_residual
        self.tolerance = tolerance
        self.column = column

    @classmethod
    def from_native(cls, message: str, tolerance: float) -> SolverConvergenceError:
        col = re.search(r"column (\d+)", message)
        its = re.search(r"(\d+) iterations", message)
        rel = re.search(r"relative residual ([0-9.eE+-]+)", message)
        return cls(int(its.group(1)) if its else 0, float(rel.group(1)) if rel else float("nan"), tolerance,
                   column=int(col.group(1)) if col else None, message=message)


class ColumnTelemetry(NamedTuple):
    iterations: int
    relative_residual: float


def solve_placements_block(context, dip_pos_m, dip_moment, sites, didt: float, *, recovery: str = "raw",
                           nodal: bool = False, potential: bool = True) -> list[dict]:
    """Up to MAX_BLOCK placements with device-resident fields (reference fem/solve.py:865-979).

    ``context`` is a :class:`cunibs_b200._native.Context` (``Subject.context``); ``sites`` are
    (center_mm, handle_mm, distance_mm) triples. Returns one dict per placement whose field arrays
    are CUDA tensors on the context's GPU, in its element and node order: ``E`` (M, 3) and
    ``magnE`` (M) float32 of the ``recovery`` field, ``v`` (N) float64 when ``potential``,
    ``E_slots`` (n_slots, 3) when ``nodal``; plus ``transform`` (4, 4), ``iterations`` and
    ``relative_residual``. The tensors export through DLPack (``torch.utils.dlpack`` or
    ``__dlpack__``), which takes the place of the reference's CuPy arrays. The device buffers are
    written by the library's device entry point (cunibs_solve_block_device): nothing crosses to
    the host but the small per-placement scalars.
    """
    import numpy as np
    import torch

    from . import _native

    recovery = validate_recovery(recovery)
    if nodal and recovery == "raw":
        raise ValueError("nodal=True needs a recovery mode")
    k = len(sites)
    if not 1 <= k <= MAX_BLOCK:
        raise ValueError(f"solve_placements_block: k={k} must be in [1, {MAX_BLOCK}]")
    dev = torch.device("cuda", int(context.params.device))
    f64 = dict(dtype=torch.float64, device=dev)
    pos = torch.as_tensor(np.ascontiguousarray(dip_pos_m, np.float64).reshape(-1, 3), **f64)
    mom = torch.as_tensor(np.ascontiguousarray(dip_moment, np.float64).reshape(-1, 3), **f64)
    centers = torch.as_tensor(np.array([np.asarray(s[0], np.float64) for s in sites]).reshape(k, 3), **f64)
    handles = torch.as_tensor(np.array([np.asarray(s[1], np.float64) for s in sites]).reshape(k, 3), **f64)
    dists = torch.as_tensor(np.array([float(s[2]) for s in sites]), **f64)
    out = {
        "transforms": torch.empty((k, 16), **f64),
        "summary": torch.empty((k, 16), **f64),
        "iterations": torch.empty(k, dtype=torch.int32, device=dev),
        "relres": torch.empty(k, **f64),
        "magnE": torch.empty((k, context.n_tets), dtype=torch.float32, device=dev),
        "E": torch.empty((k, context.n_tets, 3), dtype=torch.float32, device=dev),
    }
    if potential:
        out["v"] = torch.empty((k, context.n_nodes), **f64)
    if nodal:
        out["E_slots"] = torch.empty((k, context.recovery(recovery)["n_slots"], 3), dtype=torch.float32, device=dev)
    torch.cuda.synchronize(dev)  # the inputs were written on torch's stream; the library uses its own
    context.solve_block_device(pos.data_ptr(), mom.data_ptr(), pos.shape[0], centers.data_ptr(), handles.data_ptr(),
                               dists.data_ptr(), k, float(didt), {name: t.data_ptr() for name, t in out.items()},
                               recovery=recovery)
    transforms = out["transforms"].reshape(k, 4, 4).cpu().numpy()
    iters = out["iterations"].cpu().numpy()
    rel = out["relres"].cpu().numpy()
    res = []
    for i in range(k):
        r = {"transform": transforms[i], "E": out["E"][i], "magnE": out["magnE"][i],
             "iterations": int(iters[i]), "relative_residual": float(rel[i])}
        if potential:
            r["v"] = out["v"][i]
        if nodal:
            r["E_slots"] = out["E_slots"][i]
        res.append(r)
    return res

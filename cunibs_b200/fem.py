"""Solver constants, the convergence error and recovery-mode validation (reference fem/solve.py:52-57,
368-405,501-505; fem/recovery.py:70-125)."""

from __future__ import annotations

import re
from typing import NamedTuple

DEFAULT_TOLERANCE = 1e-6
DEFAULT_MAX_ITERS = 2000
BLOCK_SIZES = (1, 2, 4, 8, 16)
# Widest block the Subject API chunks a sweep into (the reference's MAX_BLOCK is 8).
MAX_BLOCK = 8

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

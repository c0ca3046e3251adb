"""Subject / Placement / FieldResult: the reference's public simulate API (simulation.py:132-870)."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import numpy.typing as npt


def _as_point(value: npt.ArrayLike) -> npt.NDArray[np.float64]:
    p = np.ascontiguousarray(value, dtype=np.float64).reshape(-1)
    if p.shape != (3,):
        raise ValueError(f"Expected a 3-vector, got shape {np.shape(value)}.")
    return p


@dataclass(frozen=True, init=False)
class Placement:
    """A coil placement on the scalp in millimetres (reference simulation.py:132-166).

    ``center_mm`` is the scalp target, ``handle_mm`` the positive handle direction and
    ``distance_mm`` the offset along the outward normal. All must be finite and the handle must
    differ from the centre.
    """

    center_mm: npt.NDArray[np.float64]
    handle_mm: npt.NDArray[np.float64]
    distance_mm: float = 4.0

    def __init__(self, center_mm: npt.ArrayLike, handle_mm: npt.ArrayLike, distance_mm: float = 4.0) -> None:
        center = _as_point(center_mm)
        handle = _as_point(handle_mm)
        distance = float(distance_mm)
        if not (np.isfinite(center).all() and np.isfinite(handle).all()):
            raise ValueError("center_mm and handle_mm must be finite 3-vectors.")
        if not np.isfinite(distance):
            raise ValueError("distance_mm must be finite.")
        if np.array_equal(center, handle):
            raise ValueError("handle_mm must differ from center_mm; it defines the coil's handle direction.")
        object.__setattr__(self, "center_mm", center)
        object.__setattr__(self, "handle_mm", handle)
        object.__setattr__(self, "distance_mm", distance)

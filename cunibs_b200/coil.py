"""Magnetic-dipole coil models (reference coil.py:52-98).

A coil is a set of point dipoles in its own frame: positions in metres, moments in A*m^2. The
coil frame's z axis points into the head and the frame origin is placed ``distance_mm`` above
the scalp along the outward normal.
"""

from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path

import numpy as np
import numpy.typing as npt

# The .ccd header states dIdtmax in A/us; the field wants A/s.
_CCD_DIDTMAX_TO_A_PER_S = 1e6


@dataclass(frozen=True)
class Coil:
    """Dipoles of a coil: ``positions_m`` (n, 3) metres, ``moments`` (n, 3) A*m^2."""

    positions_m: npt.NDArray[np.float64]
    moments: npt.NDArray[np.float64]
    name: str = ""
    didt_max: float | None = None
    metadata: dict[str, str | int | float] | None = None

    def __post_init__(self) -> None:
        pos = np.ascontiguousarray(self.positions_m, dtype=np.float64).reshape(-1, 3)
        mom = np.ascontiguousarray(self.moments, dtype=np.float64).reshape(-1, 3)
        if pos.shape != mom.shape:
            raise ValueError("positions_m and moments must both be (n, 3)")
        if not (np.isfinite(pos).all() and np.isfinite(mom).all()):
            raise ValueError("coil dipoles must be finite")
        object.__setattr__(self, "positions_m", pos)
        object.__setattr__(self, "moments", mom)

    @property
    def n_dipoles(self) -> int:
        return int(self.positions_m.shape[0])

    @classmethod
    def from_ccd(cls, ccd_file: str | Path) -> Coil:
        """Read a SimNIBS ``.ccd`` text coil: a ``#key=value;...`` header, a count, then rows of
        ``x y z mx my mz`` (the format the reference's ``encode_ccd`` consumes, coil.py:85-98)."""
        with Path(ccd_file).open() as f:
            meta_line = f.readline().strip().lstrip("#").strip()
            n = int(f.readline().strip())
            data = np.loadtxt(f, dtype=np.float64, max_rows=n).reshape(-1, 6)
        meta: dict[str, str | int | float] = {}
        for part in meta_line.split(";"):
            if "=" in part:
                k, v = part.split("=", 1)
                meta[k.strip()] = v.strip()
        didt = meta.get("dIdtmax")
        return cls(
            positions_m=data[:, 0:3],
            moments=data[:, 3:6],
            name=str(meta.get("coilname", Path(ccd_file).stem)),
            didt_max=None if didt is None else float(didt) * _CCD_DIDTMAX_TO_A_PER_S,
            metadata=meta,
        )

    @classmethod
    def load(cls, source: str | Path) -> Coil:
        """Load a coil file (reference coil.py:67-82): the ``.h5`` files of the reference's coil
        library (a ``dipoles`` (n, 6) dataset with the ``.ccd`` header as attributes), ``.ccd``
        text, or ``.npz`` with ``positions_m``/``moments`` arrays. ``.h5`` files are read with h5py
        where it is installed, else with this package's own reader (``cunibs_b200.h5lite``)."""
        p = Path(source)
        if p.suffix == ".ccd":
            return cls.from_ccd(p)
        if p.suffix == ".npz":
            with np.load(p) as z:
                return cls(z["positions_m"], z["moments"], name=str(z.get("name", p.stem)))
        try:
            import h5py
        except ImportError:
            from .h5lite import read_dataset

            data, attrs = read_dataset(p, "dipoles")
        else:
            with h5py.File(p, "r") as h5f:
                data = np.asarray(h5f["dipoles"], dtype=np.float64)
                attrs = {k: _decode_attr(v) for k, v in h5f["dipoles"].attrs.items()}
        data = np.asarray(data, dtype=np.float64)
        didt = attrs.get("dIdtmax")
        return cls(
            data[:, 0:3], data[:, 3:6], name=str(attrs.get("coilname", p.stem)),
            didt_max=None if didt is None else float(didt) * _CCD_DIDTMAX_TO_A_PER_S,
            metadata=attrs,
        )


def _decode_attr(v):
    """An h5py attribute value as str, int or float."""
    if isinstance(v, bytes):
        return v.decode()
    if isinstance(v, np.generic):
        return v.item()
    return v

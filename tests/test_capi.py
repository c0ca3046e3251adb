"""The C ABI library loads without a GPU and exports every entry point its header declares."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared(header: Path) -> list[str]:
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.findall(r"^\s*(?:const\s+)?[a-z_ ]+\**\s*\**(cunibs_[a-z0-9_]+)\s*\(", text, flags=re.M)


def test_library_exports_every_declared_symbol():
    from cunibs_b200 import _native

    lib = ctypes.CDLL(str(_native.library_path()))
    names = _declared(ROOT / "include" / "cunibs_b200.h")
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_defaults_and_errors_without_a_gpu():
    from cunibs_b200 import _native

    p = _native.default_params()
    assert p.tolerance == 1e-6 and p.max_iters == 2000 and p.min_coarse_rows == 128
    assert p.cheby_degree == 2 and p.cheby_lower_ratio == 12.0 and p.agg_rounds == 2
    with pytest.raises(ValueError):
        _native.check(_native.load().cunibs_context_info(None, None))


def test_placement_validation():
    from cunibs_b200 import Placement

    with pytest.raises(ValueError):
        Placement([0, 0, 0], [0, 0, 0])
    with pytest.raises(ValueError):
        Placement([0, 0, np.nan], [0, 1, 0])
    with pytest.raises(ValueError):
        Placement([0, 0, 0, 1], [0, 1, 0])
    p = Placement([1, 2, 3], [1, 3, 3])
    assert p.distance_mm == 4.0


def test_iter_simulate_validates_eagerly(cube_mesh):
    from cunibs_b200 import Placement, Subject
    from cunibs_b200.synthetic import figure8_coil

    s = Subject(cube_mesh)
    coil = figure8_coil(4)
    with pytest.raises(TypeError):
        s.iter_simulate(coil, Placement([0, 0, 0], [0, 1, 0]))
    with pytest.raises(ValueError, match="recovery"):
        s.iter_simulate(coil, [Placement([0, 0, 0], [0, 1, 0])], recovery="bogus")

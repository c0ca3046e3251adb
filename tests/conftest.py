"""Shared fixtures. GPU tests carry the ``gpu`` marker; everything else runs on the CPU.

Meshes come from the committed fixtures under tests/golden (generated by make_golden.py from the
reference checkout) or from the seeded synthetic generators in cunibs_b200.synthetic.
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a) and the built extension")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def pins() -> dict:
    return json.loads((GOLDEN / "pins.json").read_text())


@pytest.fixture(scope="session")
def patch_mesh():
    from cunibs_b200.mesh import HeadMesh

    with np.load(GOLDEN / "head_patch_r25.npz") as z:
        return HeadMesh(z["nodes_mm"], z["tet_nodes"], z["tet_tags"], z["skin_tris"])


@pytest.fixture(scope="session")
def d70_coil():
    from cunibs_b200.coil import Coil

    with np.load(GOLDEN / "magstim_d70.npz") as z:
        return Coil(z["positions_m"], z["moments"], name="MagStim_D70")


@pytest.fixture(scope="session")
def patch_placement(patch_mesh):
    from cunibs_b200.simulation import Placement

    skin_nodes = np.unique(patch_mesh.skin_tris)
    coords = patch_mesh.nodes_mm[skin_nodes]
    top = np.ascontiguousarray(coords[np.argmax(coords[:, 2])])
    return Placement(top, top + np.array([0.0, 50.0, 0.0]), 4.0)


@pytest.fixture(scope="session")
def small_sphere():
    """A 5-shell sphere head at 6 mm spacing (~20k tets) for fast end-to-end checks."""
    from cunibs_b200.synthetic import sphere_head

    return sphere_head(6.0, 90.0, jitter_mm=0.3, seed=1)


@pytest.fixture(scope="session")
def small_coil():
    from cunibs_b200.synthetic import figure8_coil

    return figure8_coil(64)


@pytest.fixture(scope="session")
def cube_mesh():
    """A solvable 100 mm all-gray-matter cube (six tetrahedra)."""
    from cunibs_b200.mesh import HeadMesh, boundary_faces

    corners = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0], [0, 0, 1], [1, 0, 1], [0, 1, 1], [1, 1, 1]], float)
    tets = np.array([[0, 1, 3, 7], [0, 3, 2, 7], [0, 2, 6, 7], [0, 6, 4, 7], [0, 4, 5, 7], [0, 5, 1, 7]], np.int32)
    nodes = corners * 100.0
    return HeadMesh(nodes, tets, np.full(6, 2, np.int32), boundary_faces(tets, nodes))


@pytest.fixture(scope="session")
def single_tissue_ball():
    """A one-tag (gray matter) jittered Kuhn ball, ~6k tets."""
    from cunibs_b200.synthetic import sphere_head

    return sphere_head(5.0, 40.0, shells=((1.0, 2),), jitter_mm=0.4, seed=4)

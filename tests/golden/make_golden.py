"""Regenerate the committed fixtures from the reference checkout (run where it is mounted).

    python tests/golden/make_golden.py /path/to/reference

Writes, next to this script:

* ``head_patch_r25.npz`` -- the reference's cropped head patch (tests/data/head_patch_r25.msh.gz),
  parsed with this package's own Gmsh 2.2 reader: nodes_mm, tet_nodes, tet_tags, skin_tris.
* ``magstim_d70.npz`` -- the bundled MagStim D70 coil (src/cunibs/coils/MagStim_D70.h5) as
  positions_m / moments, read with this package's own HDF5 reader (``cunibs_b200.h5lite``; h5py is
  not installed here).

The reference pins these fixtures are checked against are recorded in ``pins.json`` with the
test file and line they come from.
"""

from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from cunibs_b200.h5lite import read_dataset  # noqa: E402
from cunibs_b200.mesh import load_mesh  # noqa: E402


def main(reference: Path) -> None:
    mesh = load_mesh(reference / "tests/data/head_patch_r25.msh.gz")
    np.savez_compressed(
        HERE / "head_patch_r25.npz",
        nodes_mm=mesh.nodes_mm,
        tet_nodes=mesh.tet_nodes,
        tet_tags=mesh.tet_tags,
        skin_tris=mesh.skin_tris,
    )
    coil_path = reference / "src/cunibs/coils/MagStim_D70.h5"
    d, _attrs = read_dataset(coil_path, "dipoles")
    rows = d.shape[0]
    np.savez_compressed(HERE / "magstim_d70.npz", positions_m=d[:, 0:3], moments=d[:, 3:6])
    pins = {
        "patch_counts": {"n_nodes": 8404, "n_tets": 41139, "n_skin_tris": 1125,
                         "source": "tests/data/head_patch_r25.json; tests/test_realmesh.py:36-48"},
        "patch_hierarchy_sizes": {"value": [8403, 465], "source": "tests/test_solver_kernels.py:615-637"},
        "patch_peak_magnE_raw": {"value": 0.556405, "rel": 2e-3, "source": "tests/test_realmesh.py:24,115-134"},
        "patch_peak_magnE_harmonic": {"value": 0.484461, "rel": 2e-3, "source": "tests/test_realmesh.py:25,137-141"},
        "patch_peak_location_mm": {"value": [11.794, -1.125, 77.349], "atol": 2.0,
                                   "source": "tests/test_realmesh.py:26,133"},
        "patch_iterations_tol_1e-6": {"value": 11, "source": "tests/test_block_solve.py:284-287"},
        "d70_dipoles": int(rows),
    }
    (HERE / "pins.json").write_text(json.dumps(pins, indent=2) + "\n")
    print(f"patch: {mesh}; D70: {rows} dipoles")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CUNIBS_REFERENCE_ROOT", "")
    if not root:
        raise SystemExit("usage: make_golden.py <reference checkout> (or set CUNIBS_REFERENCE_ROOT)")
    main(Path(root))

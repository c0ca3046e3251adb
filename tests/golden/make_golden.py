"""Regenerate the committed fixtures from the reference checkout (run where it is mounted).

    python tests/golden/make_golden.py /path/to/reference

Writes, next to this script:

* ``head_patch_r25.npz`` -- the reference's cropped head patch (tests/data/head_patch_r25.msh.gz),
  parsed with this package's own Gmsh 2.2 reader: nodes_mm, tet_nodes, tet_tags, skin_tris.
* ``magstim_d70.npz`` -- the bundled MagStim D70 coil (src/cunibs/coils/MagStim_D70.h5) as
  positions_m / moments. The file is HDF5 with a chunked, deflate-compressed (n, 6) dataset; h5py
  is not available here, so the chunk B-tree is walked directly (a v1 B-tree of raw-data chunks,
  each chunk zlib-compressed) -- enough for this one dataset layout, not a general HDF5 reader.

The reference pins these fixtures are checked against are recorded in ``pins.json`` with the
test file and line they come from.
"""

from __future__ import annotations

import json
import struct
import sys
import zlib
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from cunibs_b200.mesh import load_mesh  # noqa: E402


def read_chunked_f64_dataset(path: Path, n_cols: int) -> np.ndarray:
    """Assemble a 2-D float64 dataset from the first leaf raw-data-chunk B-tree in an HDF5 file.

    Each B-tree entry is (chunk bytes, filter mask, chunk offset (row, col, 0), address); the
    chunks are placed by their offsets. Edge chunks come back full-size, so the caller trims to the
    dataspace's row count.
    """
    data = path.read_bytes()
    pos = 0
    while True:
        pos = data.find(b"TREE", pos)
        if pos < 0:
            raise ValueError("no raw-data chunk B-tree found")
        if data[pos + 4] == 1 and data[pos + 5] == 0:  # node type 1 (chunks), leaf level
            break
        pos += 4
    used = struct.unpack_from("<H", data, pos + 6)[0]
    q = pos + 24
    blocks = {}
    for _ in range(used):
        size, mask = struct.unpack_from("<II", data, q)
        row, col, _elem = struct.unpack_from("<3Q", data, q + 8)
        addr = struct.unpack_from("<Q", data, q + 32)[0]
        q += 40
        if mask != 0:
            raise ValueError("a filter mask other than deflate alone is not handled")
        blocks[(row, col)] = np.frombuffer(zlib.decompress(data[addr : addr + size]), "<f8")
    chunk_cols = sorted({c for _, c in blocks})
    row_starts = sorted({r for r, _ in blocks})
    width = n_cols // len(chunk_cols)
    rows_per = blocks[(0, 0)].size // width
    return np.vstack(
        [np.hstack([blocks[(r, c)].reshape(rows_per, width) for c in chunk_cols]) for r in row_starts]
    )


def dataset_rows(path: Path, n_cols: int) -> int:
    """The dataset's row count, from its dataspace message (dims stored as (rows, n_cols) u64)."""
    data = path.read_bytes()
    for off in range(0, min(len(data), 4096) - 16):
        rows, cols = struct.unpack_from("<QQ", data, off)
        if cols == n_cols and 0 < rows < 10**7 and data[off - 8 : off - 4] != b"TREE":
            return int(rows)
    raise ValueError("dataspace not found")


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
    full = read_chunked_f64_dataset(coil_path, 6)
    rows = dataset_rows(coil_path, 6)
    d = full[:rows]
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
    main(Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference"))

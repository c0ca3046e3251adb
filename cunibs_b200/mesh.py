"""Tetrahedral head meshes: the in-memory form, and a reader for binary Gmsh 2.2 files.

Mirrors the reference's ``cunibs.mesh`` surface (``HeadMesh``, ``load_mesh``, the tissue and
surface tag tables) so code written against it reads the same here (reference mesh.py:1-386).
"""

from __future__ import annotations

import gzip
import struct
from functools import cached_property
from pathlib import Path
from typing import Literal

import numpy as np
import numpy.typing as npt

SKIN_SURFACE_TAG = 1005

type TissueLabel = Literal[
    "white_matter",
    "gray_matter",
    "csf",
    "average_bone",
    "scalp",
    "eye_balls",
    "cortical_bone",
    "cancellous_bone",
    "blood",
    "muscle",
]

# Volume tag -> tissue label (reference mesh.py:32-43).
VOLUME_KEY_TO_LABEL: dict[int, TissueLabel] = {
    1: "white_matter",
    2: "gray_matter",
    3: "csf",
    4: "average_bone",
    5: "scalp",
    6: "eye_balls",
    7: "cortical_bone",
    8: "cancellous_bone",
    9: "blood",
    10: "muscle",
}

SURFACE_KEYS = frozenset({1001, 1002, 1003, 1004, 1005, 1006, 1007, 1008, 1009, 1010, 1099})

_NODES_PER_TYPE = {1: 2, 2: 3, 3: 4, 4: 4, 5: 8, 15: 1}
_TRIANGLE = 2
_TET = 4


class HeadMesh:
    """A tetrahedral head mesh: node coordinates in millimetres, zero-based element indices."""

    def __init__(
        self,
        nodes_mm: npt.ArrayLike,
        tet_nodes: npt.ArrayLike,
        tet_tags: npt.ArrayLike,
        skin_tris: npt.ArrayLike,
    ) -> None:
        self.nodes_mm = np.ascontiguousarray(nodes_mm, dtype=np.float64).reshape(-1, 3)
        self.tet_nodes = np.ascontiguousarray(tet_nodes, dtype=np.int32).reshape(-1, 4)
        self.tet_tags = np.ascontiguousarray(tet_tags, dtype=np.int32).reshape(-1)
        self.skin_tris = np.ascontiguousarray(skin_tris, dtype=np.int32).reshape(-1, 3)
        if self.tet_tags.shape[0] != self.tet_nodes.shape[0]:
            raise ValueError("tet_tags must have one entry per tetrahedron")

    @property
    def n_nodes(self) -> int:
        return int(self.nodes_mm.shape[0])

    @property
    def n_tets(self) -> int:
        return int(self.tet_nodes.shape[0])

    @cached_property
    def tet_barycenters_mm(self) -> npt.NDArray[np.float64]:
        return self.nodes_mm[self.tet_nodes].mean(axis=1)

    def __repr__(self) -> str:
        return f"HeadMesh(n_nodes={self.n_nodes}, n_tets={self.n_tets})"


def _fail(path: Path, problem: str) -> ValueError:
    return ValueError(f"{path}: {problem}")


class _Reader:
    """Cursor over a Gmsh 2.2 binary file held in memory (text headers, binary blocks)."""

    def __init__(self, data: bytes, path: Path) -> None:
        self.data = data
        self.pos = 0
        self.path = path

    def line(self) -> str:
        end = self.data.find(b"\n", self.pos)
        if end < 0:
            raise _fail(self.path, "truncated: expected a newline-terminated line")
        text = self.data[self.pos : end].decode(errors="replace").strip()
        self.pos = end + 1
        return text

    def expect(self, marker: str) -> None:
        # A binary block may be followed by its own newline before the closing marker.
        found = self.line()
        while found == "" and self.pos < len(self.data):
            found = self.line()
        if found != marker:
            raise _fail(self.path, f"expected {marker}, found {found!r}")

    def take(self, n_bytes: int) -> bytes:
        if n_bytes < 0 or self.pos + n_bytes > len(self.data):
            raise _fail(self.path, "truncated: a block extends past the end of the file")
        out = self.data[self.pos : self.pos + n_bytes]
        self.pos += n_bytes
        return out


def parse_msh_binary(path: str | Path) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """Parse a binary Gmsh 2.2 mesh (``.msh`` or ``.msh.gz``).

    Returns ``(nodes_mm, tet_nodes, tet_tags, surf_tris, surf_tags)`` with unreferenced nodes
    dropped and indices rebased to zero, as the reference loader does (mesh.py:280-304). Surface
    triangles with tags outside the surface table are skipped; tetrahedra with unknown volume
    tags are an error.
    """
    path = Path(path)
    raw = path.read_bytes()
    if raw[:2] == b"\x1f\x8b":
        raw = gzip.decompress(raw)
    r = _Reader(raw, path)
    r.expect("$MeshFormat")
    fields = r.line().split()
    if fields[1:] != ["1", "8"]:
        raise _fail(path, f"expected a binary Gmsh 2.2 header, found {' '.join(fields)!r}")
    if struct.unpack("<i", r.take(4))[0] != 1:
        raise _fail(path, "byte-order marker is not 1")
    r.line()
    r.expect("$EndMeshFormat")
    r.expect("$Nodes")
    n_nodes = int(r.line())
    node_dt = np.dtype([("id", "<i4"), ("xyz", "<f8", (3,))])
    nodes_xyz = np.frombuffer(r.take(n_nodes * node_dt.itemsize), dtype=node_dt)["xyz"]
    r.expect("$EndNodes")
    r.expect("$Elements")
    total = int(r.line())
    tets, ttags, tris, stags = [], [], [], []
    consumed = 0
    while consumed < total:
        etype, count, ntags = struct.unpack("<3i", r.take(12))
        if ntags != 2:
            raise _fail(path, f"element block declares {ntags} tags, expected 2")
        if etype == _TRIANGLE:
            blk = np.frombuffer(r.take(count * 24), dtype="<i4").reshape(count, 6)
            keep = np.isin(blk[:, 1], list(SURFACE_KEYS))
            tris.append(blk[keep, 3:])
            stags.append(blk[keep, 1])
        elif etype == _TET:
            blk = np.frombuffer(r.take(count * 28), dtype="<i4").reshape(count, 7)
            tets.append(blk[:, 3:])
            ttags.append(blk[:, 1])
        elif etype in _NODES_PER_TYPE:
            r.take(count * (1 + ntags + _NODES_PER_TYPE[etype]) * 4)
        else:
            raise _fail(path, f"unsupported Gmsh element type {etype}")
        consumed += count
    r.expect("$EndElements")
    if not tets:
        raise _fail(path, "no tetrahedron block")
    tet_nodes = np.concatenate(tets).astype(np.int64) - 1
    tet_tags = np.concatenate(ttags).astype(np.int32)
    bad = ~np.isin(tet_tags, list(VOLUME_KEY_TO_LABEL))
    if bad.any():
        raise _fail(path, f"{int(bad.sum())} tetrahedra carry volume tags absent from the tissue table")
    surf = np.concatenate(tris).astype(np.int64) - 1 if tris else np.empty((0, 3), np.int64)
    surf_tags = np.concatenate(stags).astype(np.int32) if stags else np.empty(0, np.int32)
    if tet_nodes.min() < 0 or tet_nodes.max() >= n_nodes:
        raise _fail(path, "a tetrahedron references a node id outside the node table")
    used = np.zeros(n_nodes, dtype=bool)
    used[tet_nodes] = True
    index = np.full(n_nodes, -1, dtype=np.int64)
    index[used] = np.arange(int(used.sum()))
    if surf.size and (surf.min() < 0 or surf.max() >= n_nodes or (index[surf] < 0).any()):
        raise _fail(path, "a surface triangle references a node no tetrahedron uses")
    nodes_mm = np.ascontiguousarray(nodes_xyz[used], dtype=np.float64)
    if not np.isfinite(nodes_mm).all():
        raise _fail(path, "referenced nodes have non-finite coordinates")
    return (
        nodes_mm,
        index[tet_nodes].astype(np.int32),
        tet_tags,
        index[surf].astype(np.int32).reshape(-1, 3),
        surf_tags,
    )


def load_mesh(mesh_file: str | Path) -> HeadMesh:
    """Load a binary Gmsh 2.2 tetrahedral head mesh; the skin is surface tag 1005."""
    nodes, tets, tags, tris, stags = parse_msh_binary(mesh_file)
    return HeadMesh(nodes, tets, tags, tris[stags == SKIN_SURFACE_TAG])


def boundary_faces(tets: np.ndarray, nodes: np.ndarray) -> np.ndarray:
    """Faces owned by exactly one tetrahedron, wound so their normals point outward."""
    corners = tets[:, [[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]]].reshape(-1, 3)
    opposite = tets[:, [3, 2, 1, 0]].reshape(-1)
    key = np.sort(corners, axis=1).astype(np.int64)
    n = int(tets.max()) + 1 if tets.size else 1
    code = (key[:, 0] * n + key[:, 1]) * n + key[:, 2]
    order = np.argsort(code, kind="stable")
    sc = code[order]
    first = np.ones(sc.shape[0], dtype=bool)
    first[1:] = sc[1:] != sc[:-1]
    run_start = np.flatnonzero(first)
    counts = np.diff(np.append(run_start, sc.shape[0]))
    single = order[run_start[counts == 1]]
    faces = corners[np.sort(single)].copy()
    opp = opposite[np.sort(single)]
    tri = nodes[faces]
    normal = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    inward = np.einsum("ij,ij->i", normal, nodes[opp] - tri[:, 0]) > 0
    faces[inward] = faces[inward][:, [0, 2, 1]]
    return np.ascontiguousarray(faces, dtype=np.int32)

"""Mesh I/O and the seeded synthetic generators (CPU)."""

from __future__ import annotations

import gzip
import struct

import numpy as np
import pytest

from cunibs_b200.mesh import boundary_faces, load_mesh
from cunibs_b200.synthetic import EIGHT_SHELLS, EYE_CAP, MUSCLE_CAP, figure8_coil, sphere_head


def _write_msh(path, nodes, tets, tags, tris, tri_tags):
    """Binary Gmsh 2.2 writer for the reader test (1-based ids, 2 tags per element)."""
    out = bytearray(b"$MeshFormat\n2.2 1 8\n" + struct.pack("<i", 1) + b"\n$EndMeshFormat\n")
    out += f"$Nodes\n{len(nodes)}\n".encode()
    for i, p in enumerate(nodes):
        out += struct.pack("<i3d", i + 1, *p)
    out += b"\n$EndNodes\n"
    out += f"$Elements\n{len(tets) + len(tris)}\n".encode()
    out += struct.pack("<3i", 2, len(tris), 2)
    for i, (t, g) in enumerate(zip(tris, tri_tags)):
        out += struct.pack("<6i", i + 1, g, g, *(np.asarray(t) + 1))
    out += struct.pack("<3i", 4, len(tets), 2)
    for i, (t, g) in enumerate(zip(tets, tags)):
        out += struct.pack("<7i", len(tris) + i + 1, g, g, *(np.asarray(t) + 1))
    out += b"\n$EndElements\n"
    path.write_bytes(gzip.compress(bytes(out)))


def test_gmsh_reader_round_trip(tmp_path, cube_mesh):
    m = cube_mesh
    tris = m.skin_tris
    p = tmp_path / "cube.msh.gz"
    _write_msh(p, m.nodes_mm, m.tet_nodes, m.tet_tags, np.vstack([tris, tris[:2]]), [1005] * len(tris) + [1002, 1002])
    got = load_mesh(p)
    np.testing.assert_array_equal(got.nodes_mm, m.nodes_mm)
    np.testing.assert_array_equal(got.tet_nodes, m.tet_nodes)
    np.testing.assert_array_equal(got.skin_tris, tris)


def test_gmsh_reader_rejects_unknown_volume_tag(tmp_path, cube_mesh):
    m = cube_mesh
    p = tmp_path / "bad.msh.gz"
    _write_msh(p, m.nodes_mm, m.tet_nodes, [2, 2, 2, 2, 2, 77], m.skin_tris, [1005] * len(m.skin_tris))
    with pytest.raises(ValueError, match="volume tags"):
        load_mesh(p)


def test_boundary_faces_are_closed_and_outward(small_sphere):
    m = small_sphere
    tri = m.nodes_mm[m.skin_tris]
    normal = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    # Consistently outward: the divergence theorem gives back the mesh volume (a staircase surface
    # has faces that face away from the centre locally, so a per-face radial test would not do).
    enclosed = (normal * tri[:, 0]).sum() / 6.0
    p = m.nodes_mm[m.tet_nodes]
    vol = np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0]).sum() / 6.0
    assert enclosed == pytest.approx(vol, rel=1e-9)
    # Closed surface: every edge is shared by exactly two triangles.
    e = np.sort(np.concatenate([m.skin_tris[:, [0, 1]], m.skin_tris[:, [1, 2]], m.skin_tris[:, [2, 0]]]), axis=1)
    _, counts = np.unique(e, axis=0, return_counts=True)
    assert (counts == 2).all()


def test_sphere_head_tags_and_orientation():
    m = sphere_head(6.0, 90.0, EIGHT_SHELLS, (EYE_CAP, MUSCLE_CAP), jitter_mm=0.2, seed=0)
    assert set(np.unique(m.tet_tags).tolist()) == set(range(1, 11))
    p = m.nodes_mm[m.tet_nodes]
    det = np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0])
    assert (det > 0).all()
    again = sphere_head(6.0, 90.0, EIGHT_SHELLS, (EYE_CAP, MUSCLE_CAP), jitter_mm=0.2, seed=0)
    np.testing.assert_array_equal(m.nodes_mm, again.nodes_mm)


def test_small_workload_size_matches_config():
    """64^3 lattice at 3 mm clipped to 90 mm: ~0.68M tets / 0.12M nodes."""
    m = sphere_head(3.0, 90.0, cells=64)
    assert 600_000 < m.n_tets < 700_000 and 100_000 < m.n_nodes < 130_000


def test_figure8_coil_unit_moment_per_wing():
    c = figure8_coil(512)
    assert c.n_dipoles == 1024
    np.testing.assert_allclose(c.moments[:512, 2].sum(), 1.0)
    np.testing.assert_allclose(c.moments[512:, 2].sum(), -1.0)
    r = np.linalg.norm(c.positions_m[:512, :2] - [-0.037, 0.0], axis=1)
    assert r.max() <= 0.035 + 1e-12


def test_boundary_faces_of_single_tet():
    nodes = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float)
    f = boundary_faces(np.array([[0, 1, 2, 3]]), nodes)
    assert f.shape == (4, 3)

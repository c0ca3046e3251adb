"""Seeded synthetic inputs: multi-shell sphere heads, figure-8 dipole coils, placement grids.

The benchmark workloads are synthetic (no head scans or coil files travel with the project):

* ``sphere_head`` builds a Kuhn-subdivided cubic lattice (6 tetrahedra per cube, all sharing the
  cube's main diagonal) clipped to a ball, tags each tetrahedron by the radius of its centroid,
  optionally overrides spherical caps (eye, muscle), and returns the outer boundary as the skin.
* ``figure8_coil`` lays two discs of z-moment dipoles side by side with opposite signs.
* ``cap_placements`` / ``grid_placements`` put coil centres on the scalp.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .coil import Coil
from .mesh import HeadMesh, boundary_faces

# Corner offsets and the 6-tet Kuhn split of a unit cube.
_CUBE_CORNERS = np.array(
    [[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0], [0, 0, 1], [1, 0, 1], [0, 1, 1], [1, 1, 1]],
    dtype=np.int64,
)
_KUHN_TETS = np.array(
    [[0, 1, 3, 7], [0, 3, 2, 7], [0, 2, 6, 7], [0, 6, 4, 7], [0, 4, 5, 7], [0, 5, 1, 7]],
    dtype=np.int64,
)

# (outer radius as a fraction of the head radius, tag). Five shells of the small workload:
# WM < 60, GM < 66, CSF < 70, bone < 78, scalp <= 90 at R = 90 mm.
FIVE_SHELLS = ((60 / 90, 1), (66 / 90, 2), (70 / 90, 3), (78 / 90, 4), (1.0, 5))
# Eight shells of the 1M-tet ten-tissue model (fractions of R): WM, GM, CSF, blood, compact
# bone, spongy bone, average bone, scalp; the eye and the muscle are caps on top of them.
EIGHT_SHELLS = (
    (58 / 90, 1),
    (64 / 90, 2),
    (68 / 90, 3),
    (69.5 / 90, 9),
    (71.5 / 90, 7),
    (75 / 90, 8),
    (77 / 90, 4),
    (1.0, 5),
)


@dataclass(frozen=True)
class Cap:
    """A tagged ball: tetrahedra whose centroid lies within ``radius`` of ``center`` (fractions of R)."""

    center: tuple[float, float, float]
    radius: float
    tag: int
    min_r: float = 0.0


EYE_CAP = Cap((0.0, 0.74, -0.42), 0.14, 6, 0.0)
MUSCLE_CAP = Cap((0.80, 0.0, -0.25), 0.33, 10, 70 / 90)


def sphere_head(
    spacing_mm: float,
    radius_mm: float = 90.0,
    shells: tuple[tuple[float, int], ...] = FIVE_SHELLS,
    caps: tuple[Cap, ...] = (),
    jitter_mm: float = 0.0,
    seed: int = 0,
    cells: int | None = None,
) -> HeadMesh:
    """Kuhn lattice clipped to ``r <= radius_mm``, tagged by centroid radius.

    ``cells`` fixes the lattice size (cells per axis, centred on the origin); by default it is
    the smallest that covers the ball. Node jitter is uniform in ``[-jitter_mm, jitter_mm]`` per
    axis, drawn from ``numpy.random.default_rng(seed)``.
    """
    if cells is None:
        cells = int(np.ceil(2 * radius_mm / spacing_mm)) + 1
    half = cells * spacing_mm / 2.0
    n1 = cells + 1
    lin = np.arange(n1, dtype=np.float64) * spacing_mm - half
    # Cube centres within reach of the ball: a tet's centroid lies inside its cube.
    ci = np.arange(cells)
    cx, cy, cz = np.meshgrid(ci, ci, ci, indexing="ij")
    cc = (np.stack([cx, cy, cz], -1).reshape(-1, 3) + 0.5) * spacing_mm - half
    reach = np.linalg.norm(cc, axis=1) <= radius_mm + spacing_mm
    cubes = np.stack([cx, cy, cz], -1).reshape(-1, 3)[reach]
    gid = lambda ijk: (ijk[..., 0] * n1 + ijk[..., 1]) * n1 + ijk[..., 2]  # noqa: E731
    corner_ids = gid(cubes[:, None, :] + _CUBE_CORNERS[None, :, :])  # (C, 8)
    tets = corner_ids[:, _KUHN_TETS].reshape(-1, 4)
    gx, gy, gz = np.meshgrid(lin, lin, lin, indexing="ij")
    all_nodes = np.stack([gx, gy, gz], -1).reshape(-1, 3)
    cent = all_nodes[tets].mean(axis=1)
    rc = np.linalg.norm(cent, axis=1)
    keep = rc <= radius_mm
    tets, cent, rc = tets[keep], cent[keep], rc[keep]
    used, inverse = np.unique(tets.ravel(), return_inverse=True)
    nodes = all_nodes[used].copy()
    tets = inverse.reshape(-1, 4).astype(np.int32)
    if jitter_mm > 0:
        rng = np.random.default_rng(seed)
        nodes += rng.uniform(-jitter_mm, jitter_mm, nodes.shape)
        cent = nodes[tets].mean(axis=1)
        rc = np.linalg.norm(cent, axis=1)
    tags = np.full(tets.shape[0], shells[-1][1], dtype=np.int32)
    for frac, tag in reversed(shells):
        tags[rc < frac * radius_mm] = tag
    for cap in caps:
        c = np.asarray(cap.center) * radius_mm
        inside = (np.linalg.norm(cent - c, axis=1) <= cap.radius * radius_mm) & (rc >= cap.min_r * radius_mm)
        tags[inside] = cap.tag
    # Kuhn tets of a lattice are consistently oriented only up to sign; fix positive volume order.
    p = nodes[tets]
    det = np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0])
    flip = det < 0
    tets[flip] = tets[flip][:, [0, 2, 1, 3]]
    skin = boundary_faces(tets, nodes)
    return HeadMesh(nodes, tets, tags, skin)


def figure8_coil(
    n_per_wing: int = 512,
    disc_radius_mm: float = 35.0,
    wing_offset_mm: float = 37.0,
    name: str = "figure8",
) -> Coil:
    """Two discs of z-moment dipoles centred at x = +-wing_offset, opposite signs.

    Dipoles fill each disc on a Vogel (golden-angle) spiral, each wing's moments summing to a unit
    total. Positions are in metres in the coil frame, whose z axis points into the head.
    """
    i = np.arange(n_per_wing, dtype=np.float64)
    golden = np.pi * (3.0 - np.sqrt(5.0))
    rad = disc_radius_mm * np.sqrt((i + 0.5) / n_per_wing)
    th = i * golden
    disc = np.stack([rad * np.cos(th), rad * np.sin(th), np.zeros_like(rad)], -1)
    pos = np.concatenate([disc + [-wing_offset_mm, 0, 0], disc + [wing_offset_mm, 0, 0]]) * 1e-3
    mom = np.zeros_like(pos)
    mom[:n_per_wing, 2] = 1.0 / n_per_wing
    mom[n_per_wing:, 2] = -1.0 / n_per_wing
    return Coil(positions_m=np.ascontiguousarray(pos), moments=np.ascontiguousarray(mom), name=name)


def grid_placements(
    radius_mm: float, polar_deg: list[float], azimuth_deg: list[float], handle_mm: float = 50.0
) -> list[tuple[np.ndarray, np.ndarray]]:
    """(center, handle) pairs on a polar/azimuth grid of the sphere; the handle points along +azimuth."""
    out = []
    for th in polar_deg:
        for ph in azimuth_deg:
            t, p = np.radians(th), np.radians(ph)
            c = radius_mm * np.array([np.sin(t) * np.cos(p), np.sin(t) * np.sin(p), np.cos(t)])
            tangent = np.array([-np.sin(p), np.cos(p), 0.0])
            out.append((c, c + handle_mm * tangent))
    return out


def cap_placements(
    radius_mm: float, n: int, min_z_mm: float = 40.0, seed: int = 0, handle_mm: float = 50.0
) -> list[tuple[np.ndarray, np.ndarray]]:
    """Uniform random centres on the spherical cap above ``min_z_mm``, handle azimuth uniform."""
    rng = np.random.default_rng(seed)
    zmin = min_z_mm / radius_mm
    out = []
    for _ in range(n):
        z = rng.uniform(zmin, 1.0)
        ph = rng.uniform(0.0, 2 * np.pi)
        s = np.sqrt(max(0.0, 1.0 - z * z))
        c = radius_mm * np.array([s * np.cos(ph), s * np.sin(ph), z])
        nrm = c / np.linalg.norm(c)
        a = rng.uniform(0.0, 2 * np.pi)
        ref = np.array([1.0, 0.0, 0.0]) if abs(nrm[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
        u = np.cross(nrm, ref)
        u /= np.linalg.norm(u)
        v = np.cross(nrm, u)
        out.append((c, c + handle_mm * (np.cos(a) * u + np.sin(a) * v)))
    return out

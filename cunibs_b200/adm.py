"""Auxiliary dipole method: reciprocity-based coil-placement evaluation and optimisation (reference
cunibs.adm: target.py, grid.py, reciprocity.py, evaluate.py, optimize.py).

A target functional of the E-field (a volume-weighted average of one component over a few
gray-matter elements, or the three components of a magnitude target) costs one block of adjoint
solves on the subject's own solver; the reciprocity field they define is sampled on a regular grid
above the scalp once, after which the target field of any coil placement is a trilinear
interpolation and a dipole sum (``cunibs_adm_*`` in the native library), with no FEM solve.

Functions take a :class:`~cunibs_b200.simulation.Subject` (or its native context) where the
reference takes its ``SolverContext``; element indices are in the subject's (Morton) order, as
every result array is. Grids are in metres, as in the reference.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import numpy.typing as npt

from . import _native, metrics
from .coil import Coil

ADJOINT_TOLERANCE = 1e-9  # the adjoint right-hand side is a near point source (reciprocity.py:40-45)
ADJOINT_MAX_ITERS = 3000


def _context(subject) -> _native.Context:
    return subject.context if hasattr(subject, "context") else subject


def _as_point(value: npt.ArrayLike) -> npt.NDArray[np.float64]:
    p = np.array(value, dtype=np.float64).reshape(-1)
    if p.shape != (3,):
        raise ValueError(f"Expected a 3-vector, got shape {np.shape(value)}.")
    return p


# --- target (target.py) ------------------------------------------------------------------------


@dataclass(frozen=True, init=False)
class Target:
    """A cortical target (target.py:26-60). ``direction=None`` asks for the direction-free
    magnitude (three adjoint directions); ``radius_mm`` averages over the region's elements whose
    barycentre lies within the ball, ``0`` picks the nearest element."""

    position_mm: npt.NDArray[np.float64]
    direction: npt.NDArray[np.float64] | None
    region: metrics.Region
    radius_mm: float

    def __init__(self, position_mm: npt.ArrayLike, direction: npt.ArrayLike | None = None, *,
                 region: metrics.Region = "gray_matter", radius_mm: float = 0.0) -> None:
        object.__setattr__(self, "position_mm", _as_point(position_mm))
        if direction is None:
            object.__setattr__(self, "direction", None)
        else:
            d = _as_point(direction)
            n = float(np.linalg.norm(d))
            if n == 0.0:
                raise ValueError("direction must be non-zero.")
            object.__setattr__(self, "direction", d / n)
        object.__setattr__(self, "region", region)
        object.__setattr__(self, "radius_mm", float(radius_mm))


@dataclass
class ResolvedTarget:
    """A target as weighted mesh elements and adjoint directions (target.py:63-72)."""

    elem_idx: npt.NDArray[np.int32]
    weights: npt.NDArray[np.float64]  # volume fractions, summing to 1
    directions: npt.NDArray[np.float64]  # (D, 3) orthonormal
    magnitude: bool
    barycenter_mm: npt.NDArray[np.float64]


def resolve_target(subject, target: Target) -> ResolvedTarget:
    """Map a :class:`Target` to region elements, volume weights and directions (target.py:75-109)."""
    ctx = _context(subject)
    barys = ctx.array("bary").reshape(-1, 3)
    tags = ctx.array("tet_tags")
    vols = ctx.array("vols")
    region_ids = np.flatnonzero(metrics.region_mask(tags, target.region)).astype(np.int32)
    if region_ids.size == 0:
        raise ValueError(f"Region {target.region!r} contains no elements.")
    d2 = ((barys[region_ids] - target.position_mm) ** 2).sum(1)
    if target.radius_mm <= 0.0:
        sel = region_ids[[int(np.argmin(d2))]]
    else:
        within = d2 <= target.radius_mm ** 2
        if not within.any():
            within = d2 == d2.min()
        sel = region_ids[within]
    v = vols[sel].astype(np.float64)
    weights = v / v.sum()
    if target.direction is None:
        directions, magnitude = np.eye(3), True
    else:
        directions, magnitude = np.asarray(target.direction, np.float64)[None], False
    return ResolvedTarget(elem_idx=np.ascontiguousarray(sel), weights=weights, directions=directions,
                          magnitude=magnitude, barycenter_mm=weights @ barys[sel])


# --- grid (grid.py) ----------------------------------------------------------------------------


@dataclass
class Grid:
    """Axis-aligned regular grid in metres (grid.py:10-56): ``origin_m`` is index (0, 0, 0)."""

    origin_m: npt.NDArray[np.float64]
    spacing_m: npt.NDArray[np.float64]
    shape: tuple[int, int, int]

    @property
    def n_points(self) -> int:
        return int(self.shape[0] * self.shape[1] * self.shape[2])

    @property
    def max_index(self) -> npt.NDArray[np.float64]:
        return np.asarray(self.shape, dtype=np.float64) - 1.0

    @property
    def upper_m(self) -> npt.NDArray[np.float64]:
        return self.origin_m + self.spacing_m * self.max_index

    @property
    def center_m(self) -> npt.NDArray[np.float64]:
        return 0.5 * (self.origin_m + self.upper_m)

    def points_m(self) -> npt.NDArray[np.float64]:
        ax = [self.origin_m[i] + self.spacing_m[i] * np.arange(self.shape[i], dtype=np.float64) for i in range(3)]
        gx, gy, gz = np.meshgrid(ax[0], ax[1], ax[2], indexing="ij")
        return np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1)

    def world_to_index(self, points_m: npt.ArrayLike) -> npt.NDArray[np.float64]:
        """Fractional index coordinates (3, N)."""
        return np.ascontiguousarray(((np.asarray(points_m) - self.origin_m[None, :]) / self.spacing_m[None, :]).T)


def build_grid(dipole_positions_m: npt.ArrayLike, spacing_mm: float, margin_mm: float) -> Grid:
    """A grid covering the positions (metres) dilated by ``margin_mm`` (grid.py:59-68)."""
    pts = np.asarray(dipole_positions_m, dtype=np.float64).reshape(-1, 3)
    spacing_m, margin_m = spacing_mm * 1e-3, margin_mm * 1e-3
    lo = pts.min(0) - margin_m
    span = pts.max(0) + margin_m - lo
    shape = tuple(int(np.ceil(span[i] / spacing_m)) + 1 for i in range(3))
    return Grid(origin_m=lo, spacing_m=np.full(3, spacing_m), shape=shape)


# --- adjoint and reciprocity field (reciprocity.py) ------------------------------------------


class AdjointField:
    """Nodal reciprocity weights of each adjoint direction (reciprocity.py:111-141), held on the
    device by a native handle."""

    def __init__(self, subject, target: ResolvedTarget, handle: _native.Adm) -> None:
        self.subject = subject
        self.target = target
        self.handle = handle

    @property
    def node_weights(self) -> npt.NDArray[np.float64]:
        """(D, n_nodes, 3) float64."""
        return self.handle.node_weights()

    @property
    def iterations(self) -> npt.NDArray[np.int32]:
        return self.handle.iterations

    @property
    def relative_residual(self) -> npt.NDArray[np.float64]:
        return self.handle.relres


def solve_adjoint(subject, target: ResolvedTarget, *, tolerance: float = ADJOINT_TOLERANCE,
                  max_iters: int = ADJOINT_MAX_ITERS) -> AdjointField:
    """The adjoint solves of every direction (one block solve) and their nodal weights."""
    h = _native.Adm(_context(subject), target.elem_idx, target.weights, target.directions, tolerance, max_iters)
    return AdjointField(subject, target, h)


def exact_functional(node_weights: npt.ArrayLike, dadt_nodes: npt.ArrayLike) -> npt.NDArray[np.float64]:
    """J_d = sum_n W_{d,n} . dA/dt_n (reciprocity.py:144-151), the validation path."""
    return np.einsum("dnk,nk->d", np.asarray(node_weights, np.float64), np.asarray(dadt_nodes, np.float64))


@dataclass
class ReciprocityField:
    """The adjoint weights sampled as Q on a grid (reciprocity.py:154-170): the target field of a
    placement is E_d = didt sum_j m_j . Q_d(s_j)."""

    subject: object
    target: ResolvedTarget
    grid: Grid
    adjoint: AdjointField
    magnitude: bool
    sample_id: int = 0

    def _ready(self) -> _native.Adm:
        h = self.adjoint.handle
        if h.sample_id != self.sample_id:  # the handle has sampled another grid since
            self.sample_id = _sample(h, self.grid)
        return h

    @property
    def q(self) -> npt.NDArray[np.float32]:
        """(D, nx, ny, nz, 3) float32."""
        return self._ready().qfield()


def _sample(h: _native.Adm, grid: Grid) -> int:
    return h.sample(grid.origin_m * 1e3, grid.spacing_m * 1e3, grid.shape)


def sample_qfield(adjoint: AdjointField, grid: Grid) -> ReciprocityField:
    """Q_d on ``grid`` by the FP32 dipole N-body with the mesh nodes as sources (reciprocity.py:173-213)."""
    sid = _sample(adjoint.handle, grid)
    return ReciprocityField(adjoint.subject, adjoint.target, grid, adjoint, adjoint.target.magnitude, sid)


def _coverage_grid(subject, coil: Coil, centers_mm, distance_mm: float, spacing_mm: float,
                   margin_mm: float) -> Grid:
    """A grid holding every coil dipole at any rotation on each centre (reciprocity.py:216-229)."""
    centers = np.asarray(centers_mm, dtype=np.float64).reshape(-1, 3)
    T, _ = _context(subject).place(centers, None, np.full(centers.shape[0], distance_mm))
    reach_mm = float(np.linalg.norm(np.asarray(coil.positions_m), axis=1).max()) * 1e3
    return build_grid(T[:, :3, 3] * 1e-3, spacing_mm=spacing_mm, margin_mm=reach_mm + margin_mm)


def build_reciprocity(subject, coil: Coil, target: Target, coverage_centers_mm: npt.ArrayLike, *,
                      distance_mm: float = 4.0, spacing_mm: float = 3.0, margin_mm: float = 8.0,
                      tolerance: float = ADJOINT_TOLERANCE, max_iters: int = ADJOINT_MAX_ITERS) -> ReciprocityField:
    """Adjoint solves plus a Q grid covering the candidate scalp positions (reciprocity.py:232-245)."""
    resolved = resolve_target(subject, target)
    adjoint = solve_adjoint(subject, resolved, tolerance=tolerance, max_iters=max_iters)
    grid = _coverage_grid(subject, coil, coverage_centers_mm, distance_mm, spacing_mm, margin_mm)
    return sample_qfield(adjoint, grid)


# --- evaluation (evaluate.py) ------------------------------------------------------------------


def _placements(placements) -> tuple[list, bool]:
    from .simulation import Placement

    single = isinstance(placements, Placement)
    return ([placements] if single else list(placements)), single


def _transforms(subject, pls) -> npt.NDArray[np.float64]:
    centers = np.stack([p.center_mm for p in pls])
    handles = np.stack([p.handle_mm for p in pls])
    dists = np.array([p.distance_mm for p in pls], dtype=np.float64)
    T, _ = _context(subject).place(centers, handles, dists)
    return T


def grid_for_placements(subject, coil: Coil, placements, spacing_mm: float = 3.0, margin_mm: float = 8.0) -> Grid:
    """A Q grid covering every coil dipole of the placements (evaluate.py:32-41)."""
    pls, _ = _placements(placements)
    T = _transforms(subject, pls)
    pos_mm = np.asarray(coil.positions_m) * 1e3
    s = (np.einsum("nj,pij->pni", pos_mm, T[:, :3, :3]) + T[:, None, :3, 3]) * 1e-3
    return build_grid(s.reshape(-1, 3), spacing_mm=spacing_mm, margin_mm=margin_mm)


def evaluate(recip: ReciprocityField, coil: Coil, placements, didt: float = 1e6) -> npt.NDArray[np.float64]:
    """Target E-vector (P, D) of each placement by grid interpolation (evaluate.py:114-131); a
    single Placement gives (D,). No FEM solve."""
    pls, single = _placements(placements)
    e = evaluate_frames(recip, coil, _transforms(recip.subject, pls), didt)
    return e[0] if single else e


def evaluate_frames(recip: ReciprocityField, coil: Coil, transforms: npt.ArrayLike,
                    didt: float = 1e6) -> npt.NDArray[np.float64]:
    """Target E-vector (P, D) for coil-to-head affines used verbatim (evaluate.py:134-152)."""
    return recip._ready().evaluate(coil, transforms, didt)


def evaluate_exact(adjoint: AdjointField, coil: Coil, placements, didt: float = 1e6,
                   center_m: npt.ArrayLike | None = None) -> npt.NDArray[np.float64]:
    """The same functional with Q evaluated exactly at every dipole (evaluate.py:155-193)."""
    pls, single = _placements(placements)
    T = _transforms(adjoint.subject, pls)
    c = None if center_m is None else np.asarray(center_m, np.float64) * 1e3
    e = adjoint.handle.evaluate_exact(coil, T, didt, c)
    return e[0] if single else e


# --- optimisation (optimize.py) ----------------------------------------------------------------


@dataclass
class OptimizeResult:
    """The best placement and the per-candidate objective map (optimize.py:30-41)."""

    best_center_mm: npt.NDArray[np.float64]
    best_handle_mm: npt.NDArray[np.float64]
    best_angle_rad: float
    best_E: npt.NDArray[np.float64]
    best_objective: float
    centers_mm: npt.NDArray[np.float64]
    center_objective: npt.NDArray[np.float64]
    center_handle_mm: npt.NDArray[np.float64]


def _inplane_basis(normal: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Two orthonormal in-plane vectors per normal (optimize.py:44-50)."""
    ref = np.eye(3)[np.argmin(np.abs(normal), axis=1)]
    u = np.cross(normal, ref)
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    return u, np.cross(normal, u)


def _objective(e: np.ndarray, magnitude: bool) -> np.ndarray:
    return np.linalg.norm(e, axis=-1) if magnitude else e[..., 0]


def _frame_stack(proj, normal, y, distance_mm) -> np.ndarray:
    z = np.broadcast_to(-normal, y.shape)
    m = np.zeros((*y.shape[:-1], 4, 4))
    m[..., :3, 0] = np.cross(y, z)
    m[..., :3, 1] = y
    m[..., :3, 2] = z
    m[..., :3, 3] = np.broadcast_to(proj + distance_mm * normal, y.shape)
    m[..., 3, 3] = 1.0
    return m


def _project(subject, centers: np.ndarray, distance_mm: float):
    """Scalp contact point, outward normal and in-plane basis per centre (optimize.py:135-147)."""
    T, _ = _context(subject).place(centers, None, np.full(centers.shape[0], distance_mm))
    normal = -T[:, :3, 2]
    proj = T[:, :3, 3] - distance_mm * normal
    u, v = _inplane_basis(normal)
    return proj, normal, u, v


def _parabolic_refine(obj_grid: np.ndarray, a_best: np.ndarray, thetas: np.ndarray) -> np.ndarray:
    """Vertex of the parabola through the maximum and its neighbours (optimize.py:117-132)."""
    n = thetas.shape[0]
    rows = np.arange(obj_grid.shape[0])
    dtheta = float(thetas[1] - thetas[0])
    fa = obj_grid[rows, (a_best - 1) % n]
    fb = obj_grid[rows, a_best]
    fc = obj_grid[rows, (a_best + 1) % n]
    denom = fa - 2.0 * fb + fc
    delta = np.where(denom < 0, 0.5 * (fa - fc) / np.where(denom < 0, denom, 1.0), 0.0)
    return thetas[a_best] + np.clip(delta, -0.5, 0.5) * dtheta


def fourier_kernel(theta_f: np.ndarray, theta_s: np.ndarray, n_samples: int) -> np.ndarray:
    """The interpolating Dirichlet kernel (F, K) of ``n_samples`` equispaced samples: exact for a
    trigonometric polynomial of degree (n_samples - 1) / 2 (optimize.py:200-206)."""
    d = theta_f[:, None] - theta_s[None, :]
    kernel = np.ones_like(d)
    for h in range(1, (n_samples - 1) // 2 + 1):
        kernel += 2.0 * np.cos(h * d)
    return kernel / n_samples


def optimize(subject, coil: Coil, target: Target, centers_mm: npt.ArrayLike, *, n_samples: int = 9,
             distance_mm: float = 4.0, didt: float = 1e6, spacing_mm: float = 3.0) -> OptimizeResult:
    """Build the reciprocity field and search centres x rotations with no FEM solve per placement
    (optimize.py:150-170)."""
    if n_samples % 2 == 0:
        raise ValueError("n_samples must be odd for symmetric Fourier interpolation.")
    recip = build_reciprocity(subject, coil, target, centers_mm, distance_mm=distance_mm, spacing_mm=spacing_mm)
    return optimize_placement(recip, coil, centers_mm, n_samples=n_samples, distance_mm=distance_mm, didt=didt)


def optimize_placement(recip: ReciprocityField, coil: Coil, centers_mm: npt.ArrayLike, *, n_samples: int = 9,
                       resolution: int = 512, distance_mm: float = 4.0, didt: float = 1e6) -> OptimizeResult:
    """Best position and in-plane angle (optimize.py:173-231): E_d(theta) sampled at ``n_samples``
    (odd) angles, Fourier-interpolated to ``resolution`` points, the objective maximised there and
    refined by a parabola, then evaluated once more at each position's own angle."""
    if n_samples % 2 == 0:
        raise ValueError("n_samples must be odd for symmetric Fourier interpolation.")
    centers = np.asarray(centers_mm, dtype=np.float64).reshape(-1, 3)
    proj, normal, u, v = _project(recip.subject, centers, distance_mm)
    c = proj.shape[0]
    theta_s = np.linspace(0.0, 2.0 * np.pi, n_samples, endpoint=False)
    y = np.cos(theta_s)[None, :, None] * u[:, None, :] + np.sin(theta_s)[None, :, None] * v[:, None, :]
    frames = _frame_stack(proj[:, None, :], normal[:, None, :], y, distance_mm).reshape(-1, 4, 4)
    e_s = evaluate_frames(recip, coil, frames, didt).reshape(c, n_samples, -1)  # (C, K, D)
    theta_f = np.linspace(0.0, 2.0 * np.pi, resolution, endpoint=False)
    e_f = np.tensordot(e_s, fourier_kernel(theta_f, theta_s, n_samples), axes=([1], [1]))  # (C, D, F)
    obj_f = _objective(np.moveaxis(e_f, 1, 2), recip.magnitude)
    theta = _parabolic_refine(obj_f, np.argmax(obj_f, axis=1), theta_f)
    y1 = np.cos(theta)[:, None] * u + np.sin(theta)[:, None] * v
    e = evaluate_frames(recip, coil, _frame_stack(proj, normal, y1, distance_mm), didt)
    obj = _objective(e, recip.magnitude)
    handle = proj + y1
    gi = int(np.argmax(obj))
    return OptimizeResult(best_center_mm=proj[gi].copy(), best_handle_mm=handle[gi].copy(),
                          best_angle_rad=float(theta[gi]), best_E=e[gi].copy(), best_objective=float(obj[gi]),
                          centers_mm=proj, center_objective=obj, center_handle_mm=handle)


__all__ = ["ADJOINT_MAX_ITERS", "ADJOINT_TOLERANCE", "AdjointField", "Grid", "OptimizeResult", "ReciprocityField",
           "ResolvedTarget", "Target", "build_grid", "build_reciprocity", "evaluate", "evaluate_exact",
           "evaluate_frames", "exact_functional", "grid_for_placements", "optimize", "optimize_placement",
           "resolve_target", "sample_qfield", "solve_adjoint"]

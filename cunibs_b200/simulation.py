"""Subject / Placement / FieldResult: the reference's public simulate API (simulation.py:132-870)."""

from __future__ import annotations

from collections import deque

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


import threading  # noqa: E402
from collections.abc import Iterator, Sequence  # noqa: E402
from dataclasses import field  # noqa: E402
from pathlib import Path  # noqa: E402
from typing import Literal  # noqa: E402

from . import _native, metrics  # noqa: E402
from .coil import Coil  # noqa: E402
from .fem import (  # noqa: E402
    DEFAULT_MAX_ITERS,
    DEFAULT_TOLERANCE,
    MAX_BLOCK,
    SWEEP_MAX_BLOCK,
    SolverConvergenceError,
    validate_recovery,
)
from .mesh import HeadMesh, load_mesh  # noqa: E402

_FORMAT_VERSION = 1
Precision = Literal["mixed", "split", "plain"]
_PRECISION_CODES = {"mixed": _native.PREC_MIXED, "split": _native.PREC_SPLIT, "plain": _native.PREC_PLAIN_FP64}


@dataclass(frozen=True)
class _Retain:
    magnitude: bool
    vectors: bool
    potential: bool
    nodal: bool = False


def _sites(placements, method: str) -> list[Placement]:
    if isinstance(placements, Placement):
        raise TypeError(f"{method}() takes a sequence of placements; wrap a single one in a list, or use simulate().")
    sites = list(placements)
    for s in sites:
        if not isinstance(s, Placement):
            raise TypeError(f"{method}() takes Placement objects, got {type(s).__name__}")
    return sites


class Subject:
    """A head mesh and its reusable GPU solver state (reference simulation.py:169-546).

    ``tolerance`` is the PCG stopping criterion ||r||/||b|| (the reference's DEFAULT_TOLERANCE is
    1e-6). ``precision`` selects "split" (FP64 PCG over an FP32 V-cycle, the default), "mixed"
    (FP32 PCG and V-cycle inside FP64 iterative refinement) or "plain" (FP64 throughout).
    """

    def __init__(self, mesh: HeadMesh, *, tolerance: float = DEFAULT_TOLERANCE, max_iters: int = DEFAULT_MAX_ITERS,
                 precision: Precision = "split", device: int = 0,
                 coil_field: Literal["table", "direct"] = "table") -> None:
        if precision not in _PRECISION_CODES:
            raise ValueError("precision must be 'mixed', 'split' or 'plain'")
        if coil_field not in ("table", "direct"):
            raise ValueError("coil_field must be 'table' or 'direct'")
        self._mesh = mesh
        self._ctx: _native.Context | None = None
        self._ordered: HeadMesh | None = None
        self._host_metrics: tuple[np.ndarray, np.ndarray, np.ndarray] | None = None
        self._host_slots: dict[str, tuple[np.ndarray, np.ndarray | None]] = {}
        self._host_tets: np.ndarray | None = None
        self._tolerance = float(tolerance)
        self._max_iters = int(max_iters)
        self._precision = precision
        self._device = int(device)
        self._lock = threading.RLock()
        self._block_k_default = MAX_BLOCK  # block width of block_k=None sweeps (autotune may lower it)
        self._overlap = 2                  # dA/dt blocks per SM beside a running solve
        # "table": nodes away from the coil read its field from a table sampled once per coil (about
        # 1e-7 relative); "direct": every node sums every dipole, as the reference does.
        self._coil_field = coil_field

    @classmethod
    def from_mesh(cls, mesh_file: str | Path, **kwargs) -> Subject:
        return cls(load_mesh(mesh_file), **kwargs)

    def free(self) -> None:
        """Release the device state; it is rebuilt lazily on the next call."""
        with self._lock:
            if self._ctx is not None:
                self._ctx.close()
            self._ctx = None
            self._ordered = None
            self._host_metrics = None
            self._host_slots.clear()
            self._host_tets = None

    def __enter__(self) -> Subject:
        return self

    def __exit__(self, *exc: object) -> None:
        self.free()

    @property
    def context(self) -> _native.Context:
        with self._lock:
            if self._ctx is None:
                p = _native.default_params()
                p.tolerance = self._tolerance
                p.max_iters = self._max_iters
                p.precision = _PRECISION_CODES[self._precision]
                p.device = self._device
                m = self._mesh
                self._ctx = _native.Context(m.nodes_mm, m.tet_nodes, m.tet_tags, m.skin_tris, p)
                self._ctx.set_overlap(self._overlap)
                self._ctx.set_coil_table(self._coil_field == "table")
            return self._ctx

    @property
    def block_k_default(self) -> int:
        """Placements per block of a sweep called with ``block_k=None``."""
        return self._block_k_default

    @property
    def coil_field(self) -> str:
        """How the coil's dA/dt reaches the nodes: "table" or "direct" (see ``__init__``)."""
        return self._coil_field

    @property
    def overlap_blocks_per_sm(self) -> int:
        return self._overlap

    def set_sweep_defaults(self, *, block_k: int | None = None, overlap_blocks_per_sm: int | None = None) -> None:
        """Settings that change no result bit: the block width of ``block_k=None`` sweeps (1 to
        SWEEP_MAX_BLOCK, 16: wider than an explicit block_k may ask, since the result does not
        depend on it) and the dA/dt blocks per SM that run beside a solve (1 to 16)."""
        with self._lock:
            if block_k is not None:
                if not 1 <= int(block_k) <= SWEEP_MAX_BLOCK:
                    raise ValueError(f"block_k must be in [1, {SWEEP_MAX_BLOCK}]")
                self._block_k_default = int(block_k)
            if overlap_blocks_per_sm is not None:
                if not 1 <= int(overlap_blocks_per_sm) <= 16:
                    raise ValueError("overlap_blocks_per_sm must be in [1, 16]")
                self._overlap = int(overlap_blocks_per_sm)
                if self._ctx is not None:
                    self._ctx.set_overlap(self._overlap)

    def autotune(self, coil: Coil, placements: Sequence[Placement], **kwargs):
        """Choose the sweep defaults by timing them on these placements (cunibs_b200.tune.autotune)."""
        from .tune import autotune

        return autotune(self, coil, placements, **kwargs)

    @property
    def mesh(self) -> HeadMesh:
        """The mesh in the Morton order every result array is indexed by."""
        with self._lock:
            if self._ordered is None:
                nodes, tets, tags, skin, _, _ = self.context.mesh()
                self._ordered = HeadMesh(nodes, tets, tags, skin)
            return self._ordered

    def _host_metric_inputs(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        with self._lock:
            if self._host_metrics is None:
                ctx = self.context
                vols = ctx.array("vols").astype(np.float32)
                self._host_metrics = (vols, ctx.array("tet_tags"), ctx.array("bary").reshape(-1, 3))
            return self._host_metrics

    def _host_slot_maps(self, recovery: str) -> tuple[np.ndarray, np.ndarray | None]:
        """Host (slot_node, slot_tag) of a recovery mode, shared by every result it produces."""
        with self._lock:
            if recovery not in self._host_slots:
                ctx = self.context
                tags = ctx.recovery_array(recovery, "slot_tag")
                self._host_slots[recovery] = (ctx.recovery_array(recovery, "slot_node"),
                                              tags if recovery != "spr_global" else None)
            return self._host_slots[recovery]

    def _host_tet_nodes(self) -> np.ndarray:
        with self._lock:
            if self._host_tets is None:
                self._host_tets = self.context.array("tet_nodes").reshape(-1, 4)
            return self._host_tets

    def recovery_operator(self, recovery: str) -> dict:
        """Build (once) and describe the patch weights of ``recovery`` (slot and fallback counts)."""
        recovery = validate_recovery(recovery)
        if recovery == "raw":
            raise ValueError("The raw mode has no recovery operator to build.")
        with self._lock:
            return self.context.recovery(recovery)

    def _iter_reduced(self, coil: Coil, sites: Sequence[Placement], didt: float, block_k: int | None,
                      retain: _Retain, recovery: str) -> Iterator[FieldResult]:
        ctx = self.context
        chunk_k = self._block_k_default if block_k is None else max(1, min(MAX_BLOCK, int(block_k)))
        slot_node, slot_tag = self._host_slot_maps(recovery) if retain.nodal else (None, None)
        # Per-node slots need the connectivity to say which nodes a region touches.
        tet_nodes = self._host_tet_nodes() if retain.nodal and slot_tag is None else None
        chunks = [sites[i : i + chunk_k] for i in range(0, len(sites), chunk_k)]

        def submit(chunk: Sequence[Placement]) -> int:
            centers = np.stack([s.center_mm for s in chunk])
            handles = np.stack([s.handle_mm for s in chunk])
            dists = np.array([s.distance_mm for s in chunk])
            with self._lock:
                return ctx.submit_block(coil, centers, handles, dists, didt, magnitude=retain.magnitude,
                                        vectors=retain.vectors, potential=retain.potential, recovery=recovery,
                                        nodal=retain.nodal)

        # Blocks go through the context two deep: the next block's coil placement, dA/dt and
        # right-hand side are prepared on the GPU beside this block's solve.
        tickets: deque[int] = deque()
        try:
            if chunks:
                tickets.append(submit(chunks[0]))
            for b, chunk in enumerate(chunks):
                if b + 1 < len(chunks):
                    tickets.append(submit(chunks[b + 1]))
                ticket = tickets.popleft()
                try:
                    with self._lock:
                        out = ctx.finish_block(ticket)
                except _native.ConvergenceFailure as exc:
                    raise SolverConvergenceError.from_native(str(exc), self._tolerance) from exc
                host = self._host_metric_inputs() if (retain.magnitude or retain.nodal) else None
                for i, site in enumerate(chunk):
                    yield FieldResult(
                        summary=metrics.from_summary_row(out["summary"][i]),
                        magnE=out["magnE"][i] if retain.magnitude else None,
                        E=out["E"][i] if retain.vectors else None,
                        v=out["v"][i] if retain.potential else None,
                        transform=out["transform"][i],
                        placement=site,
                        coil_name=coil.name,
                        didt=float(didt),
                        vols=host[0] if host else None,
                        tet_tags=host[1] if host else None,
                        barycenters_mm=host[2] if host else None,
                        recovery=recovery,
                        iterations=int(out["iterations"][i]),
                        relative_residual=float(out["relative_residual"][i]),
                        n_nodes=ctx.n_nodes if retain.nodal else None,
                        E_slots=out["E_slots"][i] if retain.nodal else None,
                        slot_node=slot_node,
                        slot_tag=slot_tag,
                        tet_nodes=tet_nodes,
                    )
        finally:
            # A consumer that stops early (or an error) leaves submitted blocks: drop them.
            with self._lock:
                for ticket in tickets:
                    if self._ctx is ctx:
                        ctx.cancel_block(ticket)

    def iter_simulate(self, coil: Coil, placements: Sequence[Placement], didt: float = 1e6, *,
                      magnitude: bool = False, vectors: bool = False, potential: bool = False,
                      nodal: bool = False, recovery: str = "harmonic", block_k: int | None = None) -> Iterator[FieldResult]:
        """Stream one FieldResult per placement, in order, solving blocks of ``block_k`` together.

        A placement's result does not depend on ``block_k`` or on which placements share its
        block. ``recovery`` selects how the reported field is derived from the solve ("harmonic",
        the default; "spr_tissue", "spr_global" or "raw"); ``nodal`` keeps the recovered field on its
        slots (read it with :meth:`FieldResult.nodal_field`). Arguments are validated here, before
        the first result is requested.
        """
        sites = _sites(placements, "iter_simulate")
        recovery = validate_recovery(recovery)
        if nodal and recovery == "raw":
            raise ValueError(
                "nodal=True needs a recovery mode: the raw per-tetrahedron field has no nodal form. "
                "Drop recovery='raw' to take the default, or name another mode."
            )
        if not isinstance(coil, Coil):
            raise TypeError("coil must be a cunibs_b200.Coil")
        retain = _Retain(bool(magnitude), bool(vectors), bool(potential), bool(nodal))
        return self._iter_reduced(coil, sites, float(didt), block_k, retain, recovery)

    def simulate(self, coil: Coil, placement: Placement, didt: float = 1e6, *, magnitude: bool = False,
                 vectors: bool = False, potential: bool = False, nodal: bool = False, recovery: str = "harmonic",
                 block_k: int | None = None) -> FieldResult:
        if not isinstance(placement, Placement):
            raise TypeError("simulate() takes a single Placement; use iter_simulate() for a sequence.")
        (result,) = self.iter_simulate(coil, [placement], didt, magnitude=magnitude, vectors=vectors,
                                       potential=potential, nodal=nodal, recovery=recovery, block_k=block_k)
        return result

    def roi(self, point_mm, radius_mm: float = 0.0, region: metrics.Region = "gray_matter"):
        """Volume-weighted ROI of ``region`` elements around ``point_mm`` (the nearest one when the
        radius is 0), usable as a ``record_rois`` probe or an auxiliary-dipole-method target
        (reference simulation.py:233-248)."""
        from . import adm

        return adm.resolve_target(self, adm.Target(point_mm, region=region, radius_mm=radius_mm))

    def depth_probes(self, cortical_point_mm, inward_dir, depths_mm: Sequence[float], radius_mm: float = 0.0,
                     region: metrics.Region = "all") -> list:
        """ROIs at increasing depth along ``inward_dir`` from a cortical point (simulation.py:250-267)."""
        p = np.array(cortical_point_mm, dtype=np.float64).reshape(-1)
        d = np.array(inward_dir, dtype=np.float64).reshape(-1)
        if p.shape != (3,) or d.shape != (3,):
            raise ValueError("cortical_point_mm and inward_dir must be 3-vectors")
        norm = float(np.linalg.norm(d))
        if not np.isfinite(norm) or norm == 0.0:
            raise ValueError("inward_dir must be a non-zero, finite 3-vector.")
        d = d / norm
        return [self.roi(p + depth * d, radius_mm=radius_mm, region=region) for depth in depths_mm]

    def iter_simulate_conductivity_uq(self, coil: Coil, placements: Sequence[Placement], config, didt: float = 1e6,
                                      *, moments: bool = False, recovery: str = "harmonic",
                                      focality_frac: float = 0.5, record_rois=None) -> Iterator:
        """Stream a conductivity Monte Carlo per placement (reference simulation.py:594-630).

        Every draw of ``config`` (:class:`cunibs_b200.uq.ConductivityUQConfig`) re-weights the
        stiffness and right-hand side and solves the placement to the subject's tolerance; the
        AMG hierarchy stays the nominal one (only its finest level follows the draw), the coil
        field is evaluated once, and PCG starts from the nominal solution corrected within the
        span of its conductivity sensitivities (cunibs_sigma_begin / cunibs_sigma_draw). Each
        :class:`cunibs_b200.uq.ConductivityUQResult` carries the per-draw gray-matter peak,
        focality (stimulated volume at ``focality_frac`` x p99.9, 0.5 or 0.75) and peak location;
        ``moments=True`` adds per-tetrahedron mean/std/cov of |E| and the summary of the mean field.
        ``record_rois`` ({name: ROI from :meth:`roi`}) adds each draw's volume-weighted mean |E| per
        ROI (``roi_samples``). The subject is back at the nominal conductivities afterwards.
        """
        from . import uq

        sites = _sites(placements, "iter_simulate_conductivity_uq")
        recovery = validate_recovery(recovery)
        if not isinstance(coil, Coil):
            raise TypeError("coil must be a cunibs_b200.Coil")
        if focality_frac not in (0.5, 0.75):
            raise ValueError("focality_frac must be 0.5 or 0.75 (the native summary's focality levels)")
        if not isinstance(config, uq.ConductivityUQConfig) or config.n_samples < 1:
            raise ValueError("config must be a ConductivityUQConfig with n_samples >= 1")
        rois = dict(record_rois or {})
        for name, r in rois.items():
            if not hasattr(r, "elem_idx") or not hasattr(r, "weights"):
                raise TypeError(f"record_rois[{name!r}] must be an ROI from Subject.roi")
        return self._iter_uq(coil, sites, config, float(didt), bool(moments), recovery, focality_frac, rois)

    def _iter_uq(self, coil, sites, config, didt, moments, recovery, focality_frac, rois):
        from . import uq

        ctx = self.context
        present = set(int(t) for t in np.unique(self.mesh.tet_tags))
        tags = tuple(config.perturbed_tags) if config.perturbed_tags is not None else tuple(sorted(present))
        for t in tags:
            if t not in uq.DEFAULT_TISSUE_COV and t not in config.tissue_cov:
                raise ValueError(f"no coefficient of variation for tissue tag {t}")
        draws = uq.sample_conductivities(config, tags)
        nominal = uq.nominal_sigma_table()
        f_col = 14 if focality_frac == 0.5 else 15
        host = self._host_metric_inputs() if moments else None
        n = config.n_samples
        # Every placement sees the same draws, so a chunk of up to MAX_BLOCK placements shares each
        # draw's operator update and one block solve; a placement's result does not depend on its
        # block-mates, so it is the one a run of that placement alone gives.
        for start in range(0, len(sites), MAX_BLOCK):
            chunk = sites[start:start + MAX_BLOCK]
            k = len(chunk)
            centers = np.stack([s.center_mm for s in chunk])
            handles = np.stack([s.handle_mm for s in chunk])
            dists = np.array([s.distance_mm for s in chunk])
            peak = np.empty((k, n))
            foc = np.empty((k, n))
            loc = np.empty((k, n, 3))
            its = np.empty((k, n), np.int32)
            roi_s = {name: np.empty((k, n)) for name in rois}
            s1 = s2 = None
            resetups = 0
            # The study holds the chunk's coil field, nominal solution and sensitivities; each draw
            # swaps the finest operator's values and starts PCG from the sensitivity-subspace guess.
            with self._lock:
                try:
                    ctx.sigma_begin(coil, centers, handles, dists, didt, nominal, tags,
                                    magnitude=moments or bool(rois), recovery=recovery)
                    for i in range(n):
                        try:
                            out = ctx.sigma_draw(draws[i])
                        except _native.ConvergenceFailure as exc:
                            raise SolverConvergenceError.from_native(str(exc), self._tolerance) from exc
                        resetups += out["resetup"]
                        rows = out["summary"]
                        peak[:, i], foc[:, i], loc[:, i] = rows[:, 0], rows[:, f_col], rows[:, 1:4]
                        its[:, i] = out["iterations"]
                        for name, r in rois.items():  # volume-weighted ROI means (run.py:378-379)
                            roi_s[name][:, i] = out["magnE"][:, r.elem_idx].astype(np.float64) @ r.weights
                        if moments:
                            m = out["magnE"].astype(np.float64)
                            s1 = m.copy() if s1 is None else s1 + m
                            s2 = m * m if s2 is None else s2 + m * m
                finally:
                    if self._ctx is ctx:
                        ctx.sigma_end()
            for j, site in enumerate(chunk):
                mean = std = cov = None
                if moments:
                    mean = s1[j] / n
                    std = np.sqrt(np.maximum(s2[j] / n - mean * mean, 0.0))
                    cov = np.divide(std, mean, out=np.zeros_like(std), where=mean > 0)
                res = uq.ConductivityUQResult(
                    mean_magnE=mean, std_magnE=std, cov_magnE=cov, n_samples=n, perturbed_tags=tags,
                    sigma_samples=draws, vols=host[0] if host else None, tet_tags=host[1] if host else None,
                    barycenters_mm=host[2] if host else None, placement=site, coil_name=coil.name, didt=didt,
                    peak_samples=peak[j], focality_samples=foc[j], peak_location_samples=loc[j],
                    iteration_samples=its[j], recovery=recovery, full_resetups=resetups,
                    roi_samples={name: roi_s[name][j].copy() for name in rois})
                if moments:
                    res.summary = res.compute_summary()
                yield res

    def simulate_conductivity_uq(self, coil: Coil, placement: Placement, config, didt: float = 1e6, *,
                                 moments: bool = False, recovery: str = "harmonic", focality_frac: float = 0.5,
                                 record_rois=None):
        """Conductivity Monte Carlo for a single placement (reference simulation.py:632-664)."""
        if not isinstance(placement, Placement):
            raise TypeError("simulate_conductivity_uq() takes a single Placement; use "
                            "iter_simulate_conductivity_uq() for a sequence.")
        (result,) = self.iter_simulate_conductivity_uq(coil, [placement], config, didt, moments=moments,
                                                       recovery=recovery, focality_frac=focality_frac,
                                                       record_rois=record_rois)
        return result


@dataclass
class FieldResult:
    """Gray-matter metrics for one placement plus whichever full-volume arrays were retained
    (reference simulation.py:668-870). Arrays are NumPy, in the subject's Morton order."""

    summary: metrics.FieldMetrics
    magnE: npt.NDArray[np.float32] | None
    E: npt.NDArray[np.float32] | None
    v: npt.NDArray[np.float64] | None
    transform: npt.NDArray[np.float64]
    placement: Placement
    coil_name: str
    didt: float
    vols: npt.NDArray[np.float32] | None
    tet_tags: npt.NDArray[np.int32] | None
    barycenters_mm: npt.NDArray[np.float64] | None
    recovery: str = "raw"
    iterations: int = 0
    relative_residual: float = 0.0
    n_nodes: int | None = None
    E_slots: npt.NDArray[np.float32] | None = None
    slot_node: npt.NDArray[np.int32] | None = None
    slot_tag: npt.NDArray[np.int32] | None = None
    tet_nodes: npt.NDArray[np.int32] | None = None
    _summaries: dict = field(default_factory=dict, repr=False)

    def nodal_field(self, region: metrics.Region = "gray_matter") -> npt.NDArray[np.float32]:
        """The recovered field at the mesh nodes on ``region``'s side of any boundary
        (reference simulation.py:709-747): ``(n_nodes, 3)``, NaN where ``region`` does not reach.

        For the tissue-restricted modes the field lives on (node, tissue) slots and is two-valued
        at a conductivity jump, so ``region="all"`` is rejected for them.
        """
        if self.E_slots is None or self.slot_node is None or self.n_nodes is None:
            raise ValueError("nodal_field needs the recovered nodal field, which this result did not retain. "
                             "Re-run with nodal=True.")
        if self.slot_tag is not None and region == "all":
            raise ValueError(f"nodal_field(region='all') is ambiguous for recovery={self.recovery!r}: its field is "
                             "two-valued at a tissue boundary, so a node there has one value per tissue. "
                             "Name a tissue label instead.")
        if self.slot_tag is not None:
            keep = self.slot_tag == metrics.region_tag(region)
        elif region == "all":
            keep = slice(None)
        else:
            if self.tet_nodes is None or self.tet_tags is None:
                raise ValueError("nodal_field for a specific region needs the mesh connectivity, which this result "
                                 "did not retain. Re-run with nodal=True.")
            touched = np.zeros(self.n_nodes, dtype=bool)
            touched[self.tet_nodes[metrics.region_mask(self.tet_tags, region)]] = True
            keep = touched[self.slot_node]
        out = np.full((self.n_nodes, 3), np.nan, dtype=np.float32)
        out[self.slot_node[keep]] = self.E_slots[keep]
        return out

    def _require_magnitude(self, what: str) -> np.ndarray:
        if self.magnE is None:
            raise ValueError(f"{what} needs the per-element |E|, which this result did not retain. Re-run with magnitude=True.")
        return self.magnE

    def peak_magnE(self, region: metrics.Region = "gray_matter") -> float:
        return self.summary_for(region)["peak_magnE"]

    def peak_location_mm(self, region: metrics.Region = "gray_matter") -> np.ndarray:
        return self.summary_for(region)["peak_location_mm"]

    def center_of_gravity_mm(self, region: metrics.Region = "gray_matter") -> np.ndarray:
        return self.summary_for(region)["center_of_gravity_mm"]

    def focality(self, frac: float = 0.5, region: metrics.Region = "gray_matter") -> float:
        key = f"{frac:g}"
        s = self.summary_for(region)
        if key in s["focality_m3"]:
            return s["focality_m3"][key]
        m = self._require_magnitude(f"focality at frac={key}")
        return metrics.focality(m, self.vols, metrics.region_mask(self.tet_tags, region), frac)

    def summary_for(self, region: metrics.Region) -> metrics.FieldMetrics:
        if region == self.summary["region"]:
            return self.summary
        if region not in self._summaries:
            m = self._require_magnitude(f"metrics for region {region!r}")
            self._summaries[region] = metrics.compute_metrics(m, self.vols, self.barycenters_mm, self.tet_tags, region=region)
        return self._summaries[region]

    def save(self, path: str | Path) -> None:
        """Write the result to a self-contained file (arrays not retained are absent). A ``.h5`` or
        ``.hdf5`` path gets the reference's HDF5 layout (simulation.py:805-838), written through h5py
        where it is installed, else through the built-in writer; any other path a ``.npz``."""
        if Path(path).suffix.lower() in (".h5", ".hdf5"):
            _write_hdf5_tree(path, self._hdf5_tree())
            return
        arrays = {k: getattr(self, k) for k in ("magnE", "E", "v", "vols", "tet_tags", "barycenters_mm", "E_slots",
                                                  "slot_node", "slot_tag", "tet_nodes")
                  if getattr(self, k) is not None}
        if self.n_nodes is not None:
            arrays["n_nodes"] = np.int64(self.n_nodes)
        s = self.summary
        np.savez_compressed(
            Path(path), transform=self.transform, format_version=_FORMAT_VERSION, recovery=self.recovery,
            coil_name=self.coil_name, didt=self.didt, placement_center_mm=self.placement.center_mm,
            placement_handle_mm=self.placement.handle_mm, placement_distance_mm=self.placement.distance_mm,
            summary_region=s["region"], summary_peak_magnE=s["peak_magnE"],
            summary_peak_location_mm=s["peak_location_mm"], summary_center_of_gravity_mm=s["center_of_gravity_mm"],
            summary_region_volume_m3=s["region_volume_m3"],
            summary_focality_keys=np.array(list(s["focality_m3"])), summary_focality_vals=np.array(list(s["focality_m3"].values())),
            summary_dist_keys=np.array(list(s["distribution"])), summary_dist_vals=np.array(list(s["distribution"].values())),
            iterations=self.iterations, relative_residual=self.relative_residual, **arrays)

    @classmethod
    def load(cls, path: str | Path) -> FieldResult:
        """Read a result saved by :meth:`save` (``.npz``), or an HDF5 result file in the reference's
        layout (simulation.py:805-870: datasets and attributes of the root group, the metrics in a
        ``summary`` group), recognised by its signature."""
        from . import h5lite

        if h5lite.is_hdf5(path):
            return cls._load_hdf5(path, _hdf5_tree(path))
        with np.load(Path(path), allow_pickle=False) as z:
            if int(z["format_version"]) != _FORMAT_VERSION:
                raise ValueError(f"{path}: file format version {int(z['format_version'])} is not readable (expected {_FORMAT_VERSION}).")
            opt = lambda k: np.asarray(z[k]) if k in z.files else None  # noqa: E731
            summary: metrics.FieldMetrics = {
                "region": str(z["summary_region"]),
                "peak_magnE": float(z["summary_peak_magnE"]),
                "peak_location_mm": np.asarray(z["summary_peak_location_mm"]),
                "center_of_gravity_mm": np.asarray(z["summary_center_of_gravity_mm"]),
                "region_volume_m3": float(z["summary_region_volume_m3"]),
                "focality_m3": {str(k): float(v) for k, v in zip(z["summary_focality_keys"], z["summary_focality_vals"])},
                "distribution": {str(k): float(v) for k, v in zip(z["summary_dist_keys"], z["summary_dist_vals"])},
            }
            return cls(summary=summary, magnE=opt("magnE"), E=opt("E"), v=opt("v"), transform=np.asarray(z["transform"]),
                       placement=Placement(z["placement_center_mm"], z["placement_handle_mm"], float(z["placement_distance_mm"])),
                       coil_name=str(z["coil_name"]), didt=float(z["didt"]), vols=opt("vols"), tet_tags=opt("tet_tags"),
                       barycenters_mm=opt("barycenters_mm"), recovery=str(z["recovery"]),
                       iterations=int(z["iterations"]), relative_residual=float(z["relative_residual"]),
                       n_nodes=int(z["n_nodes"]) if "n_nodes" in z.files else None, E_slots=opt("E_slots"),
                       slot_node=opt("slot_node"), slot_tag=opt("slot_tag"), tet_nodes=opt("tet_nodes"))

    def _hdf5_tree(self) -> dict:
        """The reference's HDF5 layout of this result (simulation.py:805-838) as a tree."""
        data = {k: getattr(self, k) for k in ("magnE", "E", "v", "vols", "tet_tags", "barycenters_mm", "E_slots",
                                               "slot_node", "slot_tag", "tet_nodes") if getattr(self, k) is not None}
        data["transform"] = self.transform
        attrs: dict = {"format_version": _FORMAT_VERSION, "recovery": self.recovery}
        if self.n_nodes is not None:
            attrs["n_nodes"] = int(self.n_nodes)
        attrs.update({"coil_name": self.coil_name, "didt": float(self.didt),
                      "placement_center_mm": np.asarray(self.placement.center_mm, np.float64),
                      "placement_handle_mm": np.asarray(self.placement.handle_mm, np.float64),
                      "placement_distance_mm": float(self.placement.distance_mm)})
        return {"attrs": attrs, "datasets": {k: (np.asarray(v), {}) for k, v in data.items()},
                "groups": {"summary": _metrics_tree(self.summary)}}

    @classmethod
    def _load_hdf5(cls, path, tree: dict) -> FieldResult:
        """The reference's HDF5 layout (simulation.py:839-870, _read_metrics 68-77) as a tree of
        ``{"attrs", "datasets", "groups"}`` dictionaries."""
        attrs, data = tree["attrs"], tree["datasets"]
        stored = int(attrs.get("format_version", 0))
        if stored != _FORMAT_VERSION:
            raise ValueError(f"{path}: file format version {stored} is not readable (expected {_FORMAT_VERSION}).")
        opt = lambda k: np.asarray(data[k][0]) if k in data else None  # noqa: E731
        summary = _metrics_from_tree(tree["groups"]["summary"])
        return cls(summary=summary, magnE=opt("magnE"), E=opt("E"), v=opt("v"), transform=np.asarray(data["transform"][0]),
                   placement=Placement(np.asarray(attrs["placement_center_mm"], np.float64),
                                       np.asarray(attrs["placement_handle_mm"], np.float64),
                                       float(attrs["placement_distance_mm"])),
                   coil_name=str(attrs["coil_name"]), didt=float(attrs["didt"]), vols=opt("vols"),
                   tet_tags=opt("tet_tags"), barycenters_mm=opt("barycenters_mm"),
                   recovery=str(attrs.get("recovery", "raw")),
                   n_nodes=int(attrs["n_nodes"]) if "n_nodes" in attrs else None, E_slots=opt("E_slots"),
                   slot_node=opt("slot_node"), slot_tag=opt("slot_tag"), tet_nodes=opt("tet_nodes"))


def _metrics_tree(m: metrics.FieldMetrics) -> dict:
    """The reference's metrics group layout (simulation.py:56-65) as a tree."""
    return {"attrs": {"region": str(m["region"]), "peak_magnE": float(m["peak_magnE"]),
                      "region_volume_m3": float(m["region_volume_m3"])},
            "datasets": {"peak_location_mm": (np.asarray(m["peak_location_mm"], np.float64), {}),
                         "center_of_gravity_mm": (np.asarray(m["center_of_gravity_mm"], np.float64), {})},
            "groups": {name: {"attrs": {str(k): float(v) for k, v in m[name].items()}, "datasets": {}, "groups": {}}
                       for name in ("focality_m3", "distribution")}}


def _write_hdf5_tree(path, tree: dict) -> None:
    """Writes a ``{"attrs", "datasets": {name: (array, attrs)}, "groups"}`` tree as an HDF5 file:
    through h5py where it is installed (datasets gzip-compressed, as the reference writes them), else
    through the built-in writer (contiguous datasets, strings as variable-length UTF-8)."""
    try:
        import h5py
    except ImportError:
        from . import h5lite

        h5lite.write_tree(path, tree)
        return

    def put(g, t: dict) -> None:
        for k, v in t.get("attrs", {}).items():
            g.attrs[k] = v
        for name, (arr, attrs) in t.get("datasets", {}).items():
            d = g.create_dataset(name, data=arr, compression="gzip" if np.asarray(arr).size > 16 else None)
            for k, v in attrs.items():
                d.attrs[k] = v
        for name, sub in t.get("groups", {}).items():
            put(g.create_group(name), sub)

    with h5py.File(path, "w") as f:
        put(f, tree)


def _metrics_from_tree(grp: dict) -> metrics.FieldMetrics:
    """FieldMetrics from a group in the reference's metrics layout (simulation.py:56-77)."""
    return {
        "region": str(grp["attrs"]["region"]),
        "peak_magnE": float(grp["attrs"]["peak_magnE"]),
        "peak_location_mm": np.asarray(grp["datasets"]["peak_location_mm"][0]),
        "center_of_gravity_mm": np.asarray(grp["datasets"]["center_of_gravity_mm"][0]),
        "region_volume_m3": float(grp["attrs"]["region_volume_m3"]),
        "focality_m3": {str(k): float(v) for k, v in grp["groups"]["focality_m3"]["attrs"].items()},
        "distribution": {str(k): float(v) for k, v in grp["groups"]["distribution"]["attrs"].items()},
    }


def _hdf5_tree(path) -> dict:
    """An HDF5 file as nested ``{"attrs", "datasets": {name: (array, attrs)}, "groups"}``
    dictionaries: through h5py where it is installed, else through the built-in reader (files in
    h5py's default format)."""
    try:
        import h5py
    except ImportError:
        from . import h5lite

        return h5lite.read_tree(path)

    def walk(g) -> dict:
        out = {"attrs": {k: _h5_value(v) for k, v in g.attrs.items()}, "datasets": {}, "groups": {}}
        for name, obj in g.items():
            if isinstance(obj, h5py.Group):
                out["groups"][name] = walk(obj)
            else:
                out["datasets"][name] = (np.asarray(obj), {k: _h5_value(v) for k, v in obj.attrs.items()})
        return out

    with h5py.File(path, "r") as f:
        return walk(f)


def _h5_value(v):
    if isinstance(v, bytes):
        return v.decode()
    if isinstance(v, np.ndarray) and v.shape == ():
        return v.item()
    return v

"""Monte Carlo conductivity uncertainty for one or more coil placements (reference uq/conductivity).

Every draw re-weights the stiffness and right-hand side by sampled tissue conductivities and solves
the placement again (the native study, ``cunibs_sigma_begin`` / ``cunibs_sigma_draw``). The
stiffness is a fixed sum of per-tissue components, so a draw's operator is one combination of them;
the context's AMG hierarchy stays the one built at the nominal conductivities, only the finest
level's values and smoother weights following each draw, which is the reference's
frozen-preconditioner scheme (uq/conductivity/assembly.py:1-70, run.py:203-387). Each draw starts
from the nominal solution plus the Galerkin projection of its residual onto the span of the
solution's conductivity sensitivities (run.py:105-200). PCG still solves each draw's operator to
the subject's tolerance, so the preconditioner and the guess only change the iteration count; a
draw that misses the tolerance is solved again after a full re-setup for it, and the nominal
hierarchy is then rebuilt, so accuracy never depends on the preconditioner tracking the draw.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path
from typing import Literal

import numpy as np
import numpy.typing as npt

from . import metrics
from .fem import TISSUE_CONDUCTIVITY

# Lognormal coefficients of variation per tissue tag (uq/conductivity/config.py:12-25).
DEFAULT_TISSUE_COV: dict[int, float] = {
    1: 0.15, 2: 0.15, 3: 0.05, 4: 0.35, 5: 0.20, 6: 0.20, 7: 0.35, 8: 0.35, 9: 0.15, 10: 0.20,
}

_FORMAT_VERSION = 1


@dataclass(frozen=True)
class ConductivityUQConfig:
    """Monte Carlo settings (uq/conductivity/config.py:29-53). Each perturbed tissue's conductivity is
    an independent draw with the given coefficient of variation; the lognormal model keeps it
    positive with its mean at the nominal table value."""

    n_samples: int = 500
    seed: int = 0
    tissue_cov: dict[int, float] = field(default_factory=dict)
    perturbed_tags: tuple[int, ...] | None = None
    distribution: Literal["lognormal", "normal"] = "lognormal"

    def cov_for(self, tag: int) -> float:
        if tag in self.tissue_cov:
            return self.tissue_cov[tag]
        return DEFAULT_TISSUE_COV[tag]


def sample_conductivities(config: ConductivityUQConfig, perturbed_tags: tuple[int, ...]) -> np.ndarray:
    """(n_samples, len(perturbed_tags)) draws (uq/conductivity/config.py:56-72): lognormal with the
    median parameterisation sigma0 * exp(s z - s^2 / 2), s = sqrt(log(1 + cov^2)), so the mean is
    sigma0; normal draws are clamped to 1e-6 of nominal. Seeded NumPy draws: the same distribution
    as the reference's, not its exact numbers (those come from CuPy's generator)."""
    if config.distribution not in ("lognormal", "normal"):
        raise ValueError("distribution must be 'lognormal' or 'normal'")
    rng = np.random.default_rng(config.seed)
    nominal = np.array([TISSUE_CONDUCTIVITY[t] for t in perturbed_tags], dtype=np.float64)
    covs = np.array([config.cov_for(t) for t in perturbed_tags], dtype=np.float64)
    z = rng.standard_normal((config.n_samples, len(perturbed_tags)))
    if config.distribution == "lognormal":
        s = np.sqrt(np.log1p(covs ** 2))
        return nominal * np.exp(z * s - 0.5 * s ** 2)
    return np.maximum(nominal * (1.0 + covs * z), 1e-6 * nominal)


def tissue_sensitivity(sigma_samples, y_samples, perturbed_tags) -> dict[int, float]:
    """First-order share of each perturbed tissue in the variance of a per-draw output
    (uq/conductivity/result.py:31-62): regress log y on the centred log conductivities; tag j's share
    is beta_j^2 Var(log sigma_j) / Var(log y). Not a Sobol index: no interactions, no departures
    from log-linearity."""
    x = np.log(np.asarray(sigma_samples, dtype=np.float64))
    logy = np.log(np.asarray(y_samples, dtype=np.float64))
    xc = x - x.mean(0)
    yc = logy - logy.mean()
    var_y = float(yc.var())
    if var_y == 0.0:
        return {int(t): 0.0 for t in perturbed_tags}
    beta, *_ = np.linalg.lstsq(xc, yc, rcond=None)
    contrib = beta ** 2 * xc.var(0) / var_y
    return {int(t): float(c) for t, c in zip(perturbed_tags, contrib)}


@dataclass
class ConductivityUQSummary:
    """Metrics of the ensemble-mean field and the largest local CoV (uq/conductivity/result.py:65-77)."""

    mean_field: metrics.FieldMetrics
    max_local_cov: float


@dataclass
class ConductivityUQResult:
    """One placement's conductivity Monte Carlo (uq/conductivity/result.py:79-235). The per-draw
    arrays are always present; the per-tetrahedron moments of |E| (mean, std, cov = std / mean)
    only with ``moments=True``. Arrays are NumPy, in the subject's element order."""

    mean_magnE: npt.NDArray[np.float64] | None
    std_magnE: npt.NDArray[np.float64] | None
    cov_magnE: npt.NDArray[np.float64] | None
    n_samples: int
    perturbed_tags: tuple[int, ...]
    sigma_samples: npt.NDArray[np.float64]
    vols: npt.NDArray | None
    tet_tags: npt.NDArray | None
    barycenters_mm: npt.NDArray | None
    placement: object
    coil_name: str
    didt: float
    peak_samples: npt.NDArray[np.float64]
    focality_samples: npt.NDArray[np.float64]
    peak_location_samples: npt.NDArray[np.float64]
    iteration_samples: npt.NDArray[np.int32]
    summary: ConductivityUQSummary | None = None
    recovery: str = "raw"
    full_resetups: int = 0  # draws solved again after a full re-setup
    roi_samples: dict[str, npt.NDArray[np.float64]] = field(default_factory=dict)  # name -> per-draw ROI mean |E|

    def compute_summary(self, region: metrics.Region = "gray_matter") -> ConductivityUQSummary:
        if self.mean_magnE is None or self.cov_magnE is None:
            raise ValueError(f"Metrics for region {region!r} need the per-element moment arrays, which this "
                             "result did not retain. Re-run with moments=True.")
        mask = metrics.region_mask(np.asarray(self.tet_tags), region)
        return ConductivityUQSummary(
            mean_field=metrics.compute_metrics(self.mean_magnE, self.vols, self.barycenters_mm, self.tet_tags,
                                               region=region),
            max_local_cov=float(np.asarray(self.cov_magnE)[mask].max()),
        )

    def _summary_for(self, region: metrics.Region) -> ConductivityUQSummary:
        if self.summary is not None and region == self.summary.mean_field["region"]:
            return self.summary
        return self.compute_summary(region)

    def peak_mean_magnE(self, region: metrics.Region = "gray_matter") -> float:
        """Peak of the ensemble-mean field in a region."""
        return self._summary_for(region).mean_field["peak_magnE"]

    def max_local_cov(self, region: metrics.Region = "gray_matter") -> float:
        """Largest per-tetrahedron coefficient of variation of |E| in a region."""
        return self._summary_for(region).max_local_cov

    def tissue_sensitivity(self, output: str = "peak") -> dict[int, float]:
        """Variance shares of the perturbed tissues in a per-draw output (result.py:31-62): "peak",
        "focality" or the name of an ROI recorded with ``record_rois``."""
        if output == "peak":
            y = self.peak_samples
        elif output == "focality":
            y = self.focality_samples
        elif output in self.roi_samples:
            y = self.roi_samples[output]
        else:
            raise ValueError(f"Unknown output {output!r}; expected 'peak', 'focality', or a recorded ROI name "
                             f"(available: {['peak', 'focality', *self.roi_samples]}).")
        return tissue_sensitivity(self.sigma_samples, y, self.perturbed_tags)

    def save(self, path: str | Path) -> None:
        """Write the result to a self-contained file (moment arrays only when retained). A ``.h5``
        or ``.hdf5`` path gets the reference's HDF5 layout (result.py:182-222; its files hold no
        per-draw iteration counts or re-setup count), any other path a ``.npz``."""
        if Path(path).suffix.lower() in (".h5", ".hdf5"):
            from .simulation import _write_hdf5_tree

            _write_hdf5_tree(path, self._hdf5_tree())
            return
        arrays = {k: getattr(self, k) for k in ("mean_magnE", "std_magnE", "cov_magnE", "vols", "tet_tags",
                                                  "barycenters_mm") if getattr(self, k) is not None}
        np.savez_compressed(
            Path(path), format_version=_FORMAT_VERSION, n_samples=self.n_samples,
            perturbed_tags=np.array(self.perturbed_tags, dtype=np.int64), sigma_samples=self.sigma_samples,
            placement_center_mm=self.placement.center_mm, placement_handle_mm=self.placement.handle_mm,
            placement_distance_mm=self.placement.distance_mm, coil_name=self.coil_name, didt=self.didt,
            peak_samples=self.peak_samples, focality_samples=self.focality_samples,
            peak_location_samples=self.peak_location_samples, iteration_samples=self.iteration_samples,
            recovery=self.recovery, full_resetups=self.full_resetups,
            roi_names=np.array(list(self.roi_samples), dtype=np.str_),
            roi_samples=np.stack([self.roi_samples[k] for k in self.roi_samples]) if self.roi_samples
            else np.zeros((0, self.n_samples)), **arrays)

    @classmethod
    def load(cls, path: str | Path) -> ConductivityUQResult:
        """Read a result saved by :meth:`save` (``.npz``), or an HDF5 result file in the reference's
        layout (result.py:182-262), recognised by its signature."""
        from . import h5lite
        from .simulation import Placement, _hdf5_tree

        if h5lite.is_hdf5(path):
            return cls._load_hdf5(path, _hdf5_tree(path))
        with np.load(Path(path), allow_pickle=False) as z:
            if int(z["format_version"]) != _FORMAT_VERSION:
                raise ValueError(f"{path}: file format version {int(z['format_version'])} is not readable.")
            opt = lambda k: np.asarray(z[k]) if k in z.files else None  # noqa: E731
            res = cls(
                mean_magnE=opt("mean_magnE"), std_magnE=opt("std_magnE"), cov_magnE=opt("cov_magnE"),
                n_samples=int(z["n_samples"]), perturbed_tags=tuple(int(t) for t in z["perturbed_tags"]),
                sigma_samples=np.asarray(z["sigma_samples"]), vols=opt("vols"), tet_tags=opt("tet_tags"),
                barycenters_mm=opt("barycenters_mm"),
                placement=Placement(np.asarray(z["placement_center_mm"]), np.asarray(z["placement_handle_mm"]),
                                    float(z["placement_distance_mm"])),
                coil_name=str(z["coil_name"]), didt=float(z["didt"]), peak_samples=np.asarray(z["peak_samples"]),
                focality_samples=np.asarray(z["focality_samples"]),
                peak_location_samples=np.asarray(z["peak_location_samples"]),
                iteration_samples=np.asarray(z["iteration_samples"]), recovery=str(z["recovery"]),
                full_resetups=int(z["full_resetups"]),
                roi_samples={str(n): np.asarray(v) for n, v in zip(z["roi_names"], z["roi_samples"])}
                if "roi_names" in z.files else {})
        if res.mean_magnE is not None:
            res.summary = res.compute_summary()
        return res

    def _hdf5_tree(self) -> dict:
        """The reference's HDF5 layout of this result (result.py:182-222) as a tree."""
        from .simulation import _metrics_tree

        if self.summary is None:
            raise ValueError("This result has no summary to save; call compute_summary() first.")
        data = {k: getattr(self, k) for k in ("mean_magnE", "std_magnE", "cov_magnE", "vols", "tet_tags",
                                               "barycenters_mm") if getattr(self, k) is not None}
        data["sigma_samples"] = self.sigma_samples
        for k in ("peak_samples", "focality_samples", "peak_location_samples"):
            data[k] = getattr(self, k)
        summary = {"attrs": {"max_local_cov": float(self.summary.max_local_cov)}, "datasets": {},
                   "groups": {"mean_field": _metrics_tree(self.summary.mean_field)}}
        roi = {"attrs": {}, "datasets": {k: (np.asarray(v), {}) for k, v in self.roi_samples.items()}, "groups": {}}
        attrs = {"format_version": _FORMAT_VERSION, "recovery": self.recovery, "n_samples": int(self.n_samples),
                 "perturbed_tags": np.asarray(self.perturbed_tags, dtype=np.int32), "coil_name": self.coil_name,
                 "didt": float(self.didt), "placement_center_mm": np.asarray(self.placement.center_mm, np.float64),
                 "placement_handle_mm": np.asarray(self.placement.handle_mm, np.float64),
                 "placement_distance_mm": float(self.placement.distance_mm)}
        return {"attrs": attrs, "datasets": {k: (np.asarray(v), {}) for k, v in data.items()},
                "groups": {"summary": summary, "roi_samples": roi}}

    @classmethod
    def _load_hdf5(cls, path, tree: dict) -> ConductivityUQResult:
        """The reference's HDF5 layout (result.py:193-262) as a tree of ``{"attrs", "datasets",
        "groups"}`` dictionaries. Its files hold no per-draw iteration counts: those load as -1."""
        from .simulation import Placement, _metrics_from_tree

        attrs, data, groups = tree["attrs"], tree["datasets"], tree["groups"]
        stored = int(attrs.get("format_version", 0))
        if stored != _FORMAT_VERSION:
            raise ValueError(f"{path}: file format version {stored} is not readable (expected {_FORMAT_VERSION}).")
        opt = lambda k: np.asarray(data[k][0]) if k in data else None  # noqa: E731
        n = int(attrs["n_samples"])
        summary = groups["summary"]
        roi = groups.get("roi_samples", {"datasets": {}})["datasets"]
        return cls(
            mean_magnE=opt("mean_magnE"), std_magnE=opt("std_magnE"), cov_magnE=opt("cov_magnE"), n_samples=n,
            perturbed_tags=tuple(int(t) for t in np.atleast_1d(attrs["perturbed_tags"])),
            sigma_samples=np.asarray(data["sigma_samples"][0]), vols=opt("vols"), tet_tags=opt("tet_tags"),
            barycenters_mm=opt("barycenters_mm"),
            placement=Placement(np.asarray(attrs["placement_center_mm"], np.float64),
                                np.asarray(attrs["placement_handle_mm"], np.float64),
                                float(attrs["placement_distance_mm"])),
            coil_name=str(attrs["coil_name"]), didt=float(attrs["didt"]),
            peak_samples=np.asarray(data["peak_samples"][0]), focality_samples=np.asarray(data["focality_samples"][0]),
            peak_location_samples=np.asarray(data["peak_location_samples"][0]),
            iteration_samples=np.full(n, -1, np.int32), recovery=str(attrs.get("recovery", "raw")),
            summary=ConductivityUQSummary(mean_field=_metrics_from_tree(summary["groups"]["mean_field"]),
                                          max_local_cov=float(summary["attrs"]["max_local_cov"])),
            roi_samples={str(k): np.asarray(v[0]) for k, v in roi.items()})


def nominal_sigma_table() -> np.ndarray:
    """The nominal conductivity per tag (index = tag, 11 entries)."""
    sigma = np.zeros(11)
    for tag, s in TISSUE_CONDUCTIVITY.items():
        sigma[tag] = s
    return sigma

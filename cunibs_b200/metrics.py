"""Volume-weighted E-field metrics (reference metrics.py:1-279), host-side.

The per-placement gray-matter summary of a sweep is computed on the GPU inside the block solve
(cunibs_solve_block); the functions here serve the on-demand metrics of a retained ``magnE``
(another region, another focality fraction) and convert the native summary row to the reference's
``FieldMetrics`` dictionary.
"""

from __future__ import annotations

from typing import Literal, TypedDict

import numpy as np
import numpy.typing as npt

from .mesh import VOLUME_KEY_TO_LABEL, TissueLabel

type Region = TissueLabel | Literal["all"]

_LABEL_TO_TAG: dict[str, int] = {label: tag for tag, label in VOLUME_KEY_TO_LABEL.items()}
SUMMARY_PERCENTILES = (50.0, 95.0, 99.0, 99.9)
SUMMARY_FOCALITY_FRACS = (0.5, 0.75)
FOCALITY_ANCHOR_PERCENTILE = 99.9


class FieldMetrics(TypedDict):
    region: Region
    peak_magnE: float
    peak_location_mm: npt.NDArray[np.float64]
    center_of_gravity_mm: npt.NDArray[np.float64]
    region_volume_m3: float
    focality_m3: dict[str, float]
    distribution: dict[str, float]


def region_tag(region: Region) -> int:
    tag = _LABEL_TO_TAG.get(region)
    if tag is None:
        raise ValueError(f"Unknown region {region!r}; use a tissue label: {sorted(_LABEL_TO_TAG)}.")
    return tag


def region_mask(tet_tags: np.ndarray, region: Region) -> np.ndarray:
    if region == "all":
        return np.ones(tet_tags.shape[0], dtype=bool)
    return tet_tags == region_tag(region)


def weighted_quantiles(values: np.ndarray, weights: np.ndarray, qs: np.ndarray) -> np.ndarray:
    """Volume-weighted quantiles at midpoint positions (metrics.py:82-95)."""
    order = np.argsort(values, kind="stable")
    v = np.asarray(values)[order]
    w = np.asarray(weights, dtype=np.float64)[order]
    cw = np.cumsum(w)
    pos = (cw - 0.5 * w) / cw[-1]
    return np.interp(np.asarray(qs, dtype=np.float64), pos, v)


def focality(magnE, vols, mask, frac: float = 0.5, anchor_percentile: float = FOCALITY_ANCHOR_PERCENTILE) -> float:
    m = np.asarray(magnE)[mask]
    w = np.asarray(vols, dtype=np.float64)[mask]
    q = np.float64(np.float32(anchor_percentile / 100.0))
    anchor = float(weighted_quantiles(m, w, np.array([q]))[0])
    return float(w[m >= frac * anchor].sum())


def compute_metrics(magnE, vols, barycenters_mm, tet_tags, *, region: Region = "gray_matter") -> FieldMetrics:
    mask = region_mask(np.asarray(tet_tags), region)
    m = np.asarray(magnE)[mask]
    w = np.asarray(vols, dtype=np.float64)[mask]
    bary = np.asarray(barycenters_mm)[mask]
    wsum = w.sum()
    mean = float((w * m).sum() / wsum)
    var = float((w * (m - mean) ** 2).sum() / wsum)
    qs = np.array([np.float32(p / 100.0) for p in SUMMARY_PERCENTILES], dtype=np.float64)
    pv = weighted_quantiles(m, w, qs)
    ww = w * m
    anchor = float(pv[-1])
    return {
        "region": region,
        "peak_magnE": float(m.max()),
        "peak_location_mm": np.asarray(bary[int(np.argmax(m))], dtype=np.float64),
        "center_of_gravity_mm": (ww[:, None] * bary).sum(0) / ww.sum(),
        "region_volume_m3": float(wsum),
        "focality_m3": {f"{f:g}": float(w[m >= f * anchor].sum()) for f in SUMMARY_FOCALITY_FRACS},
        "distribution": {"mean": mean, "std": float(np.sqrt(var)),
                         **{f"p{p:g}": float(v) for p, v in zip(SUMMARY_PERCENTILES, pv)}},
    }


def from_summary_row(row: np.ndarray, region: Region = "gray_matter") -> FieldMetrics:
    """The native CUNIBS_SUMMARY_* row as a FieldMetrics dictionary."""
    return {
        "region": region,
        "peak_magnE": float(row[0]),
        "peak_location_mm": np.array(row[1:4], dtype=np.float64),
        "center_of_gravity_mm": np.array(row[4:7], dtype=np.float64),
        "region_volume_m3": float(row[7]),
        "focality_m3": {"0.5": float(row[14]), "0.75": float(row[15])},
        "distribution": {"mean": float(row[8]), "std": float(row[9]), "p50": float(row[10]),
                         "p95": float(row[11]), "p99": float(row[12]), "p99.9": float(row[13])},
    }

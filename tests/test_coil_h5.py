"""The reference's bundled .h5 coils read without h5py (cunibs_b200.h5lite through Coil.load).

The committed fixture tests/golden/magstim_d70.npz holds the MagStim D70 dipoles, extracted from
the reference's coil library by tests/golden/make_golden.py. Where the reference checkout is
present, every bundled coil is read and the D70 is checked against the fixture bit for bit.
"""

from __future__ import annotations

import os
from pathlib import Path

import numpy as np
import pytest

from cunibs_b200 import Coil

GOLDEN = Path(__file__).resolve().parent / "golden" / "magstim_d70.npz"
# The reference checkout, when mounted, is named by CUNIBS_REFERENCE_ROOT; the tests that read its
# coil library are skipped otherwise.
_REF = os.environ.get("CUNIBS_REFERENCE_ROOT", "")
COILS = Path(_REF) / "src" / "cunibs" / "coils" if _REF else Path("/nonexistent")


@pytest.mark.skipif(not COILS.is_dir(), reason="the reference's coil library is not mounted")
def test_every_bundled_coil_loads_and_d70_matches_the_fixture():
    files = sorted(COILS.glob("*.h5"))
    assert len(files) >= 20
    for f in files:
        c = Coil.load(f)
        assert c.n_dipoles == int(c.metadata["num_elements"]) > 0
        assert c.name == str(c.metadata["coilname"]) and c.didt_max > 0
        assert np.abs(c.moments).sum() > 0
    d70 = Coil.load(COILS / "MagStim_D70.h5")
    g = np.load(GOLDEN)
    np.testing.assert_array_equal(d70.positions_m, g["positions_m"])
    np.testing.assert_array_equal(d70.moments, g["moments"])
    assert d70.name == "D70" and d70.didt_max == pytest.approx(114.73e6)


def test_h5lite_rejects_other_files(tmp_path):
    from cunibs_b200.h5lite import read_dataset

    bad = tmp_path / "x.h5"
    bad.write_bytes(b"not an hdf5 file at all")
    with pytest.raises(ValueError, match="HDF5"):
        read_dataset(bad, "dipoles")


@pytest.mark.skipif(not COILS.is_dir(), reason="the reference's coil library is not mounted")
def test_tree_reader_agrees_with_the_dataset_reader_on_every_coil():
    from cunibs_b200 import h5lite

    for f in sorted(COILS.glob("*.h5")):
        assert h5lite.is_hdf5(f)
        tree = h5lite.read_tree(f)
        a, attrs = h5lite.read_dataset(f, "dipoles")
        b, battrs = tree["datasets"]["dipoles"]
        np.testing.assert_array_equal(a, b)
        assert attrs == battrs and tree["groups"] == {}


def _result():
    from cunibs_b200 import Placement
    from cunibs_b200.simulation import FieldResult

    rng = np.random.default_rng(5)
    summary = {"region": "gray_matter", "peak_magnE": 101.5, "peak_location_mm": np.array([1.0, 2.0, 80.0]),
               "center_of_gravity_mm": np.array([0.5, 1.5, 78.0]), "region_volume_m3": 3.2e-4,
               "focality_m3": {"50": 1.1e-6, "75": 4.0e-7}, "distribution": {"p50": 20.0, "p99": 90.0}}
    return FieldResult(summary=summary, magnE=rng.random(40, dtype=np.float32), E=None, v=rng.random(12),
                       transform=np.eye(4), placement=Placement([0.0, 0.0, 90.0], [0.0, 50.0, 90.0], 4.0),
                       coil_name="D70", didt=1e6, vols=rng.random(40, dtype=np.float32),
                       tet_tags=np.full(40, 2, np.int32), barycenters_mm=rng.random((40, 3)), recovery="harmonic",
                       n_nodes=12, E_slots=rng.random((12, 3), dtype=np.float32), slot_node=np.arange(12, dtype=np.int32))


def _reference_layout(r) -> dict:
    """The tree the reference's FieldResult.save writes (simulation.py:805-837, _write_metrics 56-65)."""
    data = {k: (getattr(r, k), {}) for k in ("magnE", "E", "v", "vols", "tet_tags", "barycenters_mm", "E_slots",
                                              "slot_node", "slot_tag", "tet_nodes") if getattr(r, k) is not None}
    data["transform"] = (r.transform, {})
    s = r.summary
    summary = {"attrs": {"region": s["region"], "peak_magnE": s["peak_magnE"], "region_volume_m3": s["region_volume_m3"]},
               "datasets": {"peak_location_mm": (s["peak_location_mm"], {}),
                            "center_of_gravity_mm": (s["center_of_gravity_mm"], {})},
               "groups": {"focality_m3": {"attrs": dict(s["focality_m3"]), "datasets": {}, "groups": {}},
                          "distribution": {"attrs": dict(s["distribution"]), "datasets": {}, "groups": {}}}}
    attrs = {"format_version": 1, "recovery": r.recovery, "n_nodes": r.n_nodes, "coil_name": r.coil_name,
             "didt": r.didt, "placement_center_mm": r.placement.center_mm, "placement_handle_mm": r.placement.handle_mm,
             "placement_distance_mm": r.placement.distance_mm}
    return {"attrs": attrs, "datasets": data, "groups": {"summary": summary}}


def test_field_result_loads_the_reference_hdf5_layout(tmp_path, monkeypatch):
    from cunibs_b200 import simulation

    r = _result()
    tree = _reference_layout(r)
    f = tmp_path / "result.h5"
    f.write_bytes(b"\x89HDF\r\n\x1a\n" + bytes(64))  # the signature routes load() to the HDF5 reader
    monkeypatch.setattr(simulation, "_hdf5_tree", lambda path: tree)
    got = simulation.FieldResult.load(f)
    for k in ("magnE", "v", "vols", "tet_tags", "barycenters_mm", "E_slots", "slot_node", "transform"):
        np.testing.assert_array_equal(getattr(got, k), getattr(r, k))
    assert got.E is None and got.slot_tag is None and got.tet_nodes is None
    assert (got.coil_name, got.didt, got.recovery, got.n_nodes) == ("D70", 1e6, "harmonic", 12)
    np.testing.assert_array_equal(got.placement.center_mm, r.placement.center_mm)
    assert got.placement.distance_mm == 4.0
    assert got.summary["region"] == "gray_matter" and got.summary["focality_m3"] == r.summary["focality_m3"]
    assert got.summary["distribution"] == r.summary["distribution"]
    np.testing.assert_array_equal(got.summary["peak_location_mm"], r.summary["peak_location_mm"])
    # The same result through the .npz path matches too.
    r.save(tmp_path / "result.npz")
    back = simulation.FieldResult.load(tmp_path / "result.npz")
    np.testing.assert_array_equal(back.magnE, got.magnE)
    assert back.summary["peak_magnE"] == got.summary["peak_magnE"]


def test_field_result_hdf5_version_is_checked(tmp_path, monkeypatch):
    from cunibs_b200 import simulation

    tree = _reference_layout(_result())
    tree["attrs"]["format_version"] = 2
    f = tmp_path / "result.h5"
    f.write_bytes(b"\x89HDF\r\n\x1a\n" + bytes(64))
    monkeypatch.setattr(simulation, "_hdf5_tree", lambda path: tree)
    with pytest.raises(ValueError, match="format version 2"):
        simulation.FieldResult.load(f)


def test_conductivity_result_loads_the_reference_hdf5_layout(tmp_path, monkeypatch):
    from cunibs_b200 import simulation
    from cunibs_b200.uq import ConductivityUQResult

    rng = np.random.default_rng(9)
    n, m = 16, 40
    metrics_grp = _reference_layout(_result())["groups"]["summary"]
    tree = {
        "attrs": {"format_version": 1, "recovery": "harmonic", "n_samples": n,
                  "perturbed_tags": np.array([1, 2, 3], np.int32), "coil_name": "D70", "didt": 1e6,
                  "placement_center_mm": np.array([0.0, 0.0, 90.0]), "placement_handle_mm": np.array([0.0, 50.0, 90.0]),
                  "placement_distance_mm": 4.0},
        "datasets": {"mean_magnE": (rng.random(m), {}), "std_magnE": (rng.random(m), {}), "cov_magnE": (rng.random(m), {}),
                     "vols": (rng.random(m), {}), "tet_tags": (np.full(m, 2, np.int32), {}),
                     "barycenters_mm": (rng.random((m, 3)), {}), "sigma_samples": (rng.random((n, 3)), {}),
                     "peak_samples": (rng.random(n), {}), "focality_samples": (rng.random(n), {}),
                     "peak_location_samples": (rng.random((n, 3)), {})},
        "groups": {"summary": {"attrs": {"max_local_cov": 0.31}, "datasets": {}, "groups": {"mean_field": metrics_grp}},
                   "roi_samples": {"attrs": {}, "datasets": {"m1": (rng.random(n), {})}, "groups": {}}},
    }
    f = tmp_path / "uq.h5"
    f.write_bytes(b"\x89HDF\r\n\x1a\n" + bytes(64))
    monkeypatch.setattr(simulation, "_hdf5_tree", lambda path: tree)
    got = ConductivityUQResult.load(f)
    assert got.n_samples == n and got.perturbed_tags == (1, 2, 3) and got.recovery == "harmonic"
    for k in ("mean_magnE", "std_magnE", "cov_magnE", "vols", "tet_tags", "barycenters_mm", "sigma_samples",
              "peak_samples", "focality_samples", "peak_location_samples"):
        np.testing.assert_array_equal(getattr(got, k), tree["datasets"][k][0])
    np.testing.assert_array_equal(got.roi_samples["m1"], tree["groups"]["roi_samples"]["datasets"]["m1"][0])
    assert got.summary.max_local_cov == 0.31 and got.summary.mean_field["region"] == "gray_matter"
    assert (got.iteration_samples == -1).all() and got.iteration_samples.shape == (n,)
    assert set(got.tissue_sensitivity("m1")) == {1, 2, 3}


@pytest.mark.skipif(not COILS.is_dir(), reason="the reference's coil library is not mounted")
def test_truncated_files_raise_value_errors(tmp_path):
    from cunibs_b200 import h5lite

    data = (COILS / "MagStim_D70.h5").read_bytes()
    for n in (100, 900, 2000, 5000, len(data) - 64):
        p = tmp_path / f"cut{n}.h5"
        p.write_bytes(data[:n])
        for read in (lambda: h5lite.read_tree(p), lambda: h5lite.read_dataset(p, "dipoles")):
            with pytest.raises(ValueError, match="HDF5"):
                read()

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


def test_field_result_hdf5_save_round_trip(tmp_path):
    """FieldResult.save to .h5 writes the reference's layout (simulation.py:805-838); the built-in
    reader reads it back as that layout and load() restores every retained array and the summary."""
    from cunibs_b200 import h5lite, simulation

    r = _result()
    path = tmp_path / "result.h5"
    r.save(path)
    assert h5lite.is_hdf5(path)
    tree = h5lite.read_tree(path)
    want = _reference_layout(r)
    assert set(tree["datasets"]) == set(want["datasets"])
    assert set(tree["attrs"]) == set(want["attrs"])
    assert set(tree["groups"]["summary"]["groups"]) == {"focality_m3", "distribution"}
    got = simulation.FieldResult.load(path)
    for k in ("magnE", "v", "vols", "tet_tags", "barycenters_mm", "E_slots", "slot_node", "transform"):
        a, b = getattr(got, k), getattr(r, k)
        np.testing.assert_array_equal(a, b)
        assert a.dtype == np.asarray(b).dtype
    assert got.E is None and got.slot_tag is None and got.tet_nodes is None
    assert (got.coil_name, got.didt, got.recovery, got.n_nodes) == (r.coil_name, r.didt, r.recovery, r.n_nodes)
    np.testing.assert_array_equal(got.placement.handle_mm, r.placement.handle_mm)
    assert got.summary["focality_m3"] == r.summary["focality_m3"]
    assert got.summary["distribution"] == r.summary["distribution"]
    assert got.summary["peak_magnE"] == r.summary["peak_magnE"]


def test_conductivity_result_hdf5_save_round_trip(tmp_path):
    from cunibs_b200 import h5lite
    from cunibs_b200.simulation import Placement
    from cunibs_b200.uq import ConductivityUQResult, ConductivityUQSummary

    rng = np.random.default_rng(4)
    n, m = 6, 40
    mean = rng.random(m).astype(np.float32)
    summary = ConductivityUQSummary(mean_field=_result().summary, max_local_cov=0.31)
    res = ConductivityUQResult(
        mean_magnE=mean, std_magnE=mean * 0.1, cov_magnE=None, n_samples=n, perturbed_tags=(1, 2, 3),
        sigma_samples=rng.random((n, 3)), vols=rng.random(m), tet_tags=np.full(m, 2, np.int32),
        barycenters_mm=rng.random((m, 3)), placement=Placement([0.0, 0.0, 90.0], [0.0, 50.0, 90.0]),
        coil_name="fig8", didt=1e6, peak_samples=rng.random(n), focality_samples=rng.random((n, 2)),
        peak_location_samples=rng.random((n, 3)), iteration_samples=np.full(n, 12, np.int32), recovery="raw",
        summary=summary, roi_samples={"m1": rng.random(n), "s1": rng.random(n)})
    path = tmp_path / "uq.h5"
    res.save(path)
    tree = h5lite.read_tree(path)
    assert set(tree["groups"]) == {"summary", "roi_samples"}
    assert tree["attrs"]["perturbed_tags"].dtype == np.int32
    got = ConductivityUQResult.load(path)
    for k in ("mean_magnE", "std_magnE", "sigma_samples", "peak_samples", "focality_samples",
              "peak_location_samples", "vols", "tet_tags", "barycenters_mm"):
        np.testing.assert_array_equal(getattr(got, k), getattr(res, k))
    assert got.cov_magnE is None and got.perturbed_tags == (1, 2, 3) and got.n_samples == n
    assert set(got.roi_samples) == {"m1", "s1"}
    np.testing.assert_array_equal(got.roi_samples["s1"], res.roi_samples["s1"])
    assert got.summary.max_local_cov == 0.31


def test_writer_covers_types_shapes_and_many_members(tmp_path):
    """Every attribute kind the layouts use, empty and 0-d datasets, nested groups, and a group with
    more members than one symbol-table node holds (several nodes under one B-tree node)."""
    from cunibs_b200 import h5lite

    rng = np.random.default_rng(1)
    tree = {"attrs": {"s": "text with ü", "i": 7, "f": 2.5, "v": np.array([1.0, 2.0, 3.0]),
                      "ti": np.array([1, 2], np.int32), "strs": ["a", "bc"]},
            "datasets": {f"d{i:02d}": (rng.random((3, i + 1)).astype(np.float32 if i % 2 else np.float64),
                                       {"k": i}) for i in range(20)},
            "groups": {"g": {"attrs": {"x": 1.0}, "datasets": {"empty": (np.zeros((0, 3)), {}),
                                                                "ints": (np.arange(10, dtype=np.int64), {})},
                             "groups": {"h": {"attrs": {}, "datasets": {}, "groups": {}}}}}}
    path = tmp_path / "t.h5"
    h5lite.write_tree(path, tree)
    got = h5lite.read_tree(path)
    assert got["attrs"]["s"] == "text with ü" and got["attrs"]["i"] == 7 and got["attrs"]["f"] == 2.5
    np.testing.assert_array_equal(got["attrs"]["v"], [1.0, 2.0, 3.0])
    assert got["attrs"]["ti"].dtype == np.int32 and got["attrs"]["strs"] == ["a", "bc"]
    assert sorted(got["datasets"]) == sorted(tree["datasets"])
    for name, (arr, attrs) in tree["datasets"].items():
        back, battrs = got["datasets"][name]
        np.testing.assert_array_equal(back, arr)
        assert back.dtype == arr.dtype and battrs == attrs
        np.testing.assert_array_equal(h5lite.read_dataset(path, name)[0], arr)
    g = got["groups"]["g"]
    assert g["attrs"] == {"x": 1.0} and g["datasets"]["empty"][0].shape == (0, 3)
    np.testing.assert_array_equal(g["datasets"]["ints"][0], np.arange(10))
    assert g["groups"]["h"] == {"attrs": {}, "datasets": {}, "groups": {}}


@pytest.mark.skipif(not COILS.is_dir(), reason="the reference's coil library is not mounted")
def test_writer_matches_a_bundled_coil_structure(tmp_path):
    """A coil file rewritten by the built-in writer reads back (through both readers) equal to the
    bundled one: the same dataset, attributes and string encoding."""
    from cunibs_b200 import h5lite

    src = COILS / "MagStim_D70.h5"
    tree = h5lite.read_tree(src)
    out = tmp_path / "d70.h5"
    h5lite.write_tree(out, tree)
    again = h5lite.read_tree(out)
    a, aa = tree["datasets"]["dipoles"]
    b, ba = again["datasets"]["dipoles"]
    np.testing.assert_array_equal(a, b)
    assert aa == ba and again["attrs"] == tree["attrs"]
    np.testing.assert_array_equal(h5lite.read_dataset(out, "dipoles")[0], a)
    c = Coil.load(out)
    assert c.name == "D70" and c.n_dipoles == a.shape[0]


def test_group_cycle_raises_value_error_naming_the_file(tmp_path):
    """A malformed file whose group links form a cycle: a subgroup's symbol-table entry pointing back
    at the root group's object header."""
    import struct

    from cunibs_b200 import h5lite

    path = tmp_path / "cycle.h5"
    h5lite.write_tree(path, {"attrs": {}, "datasets": {}, "groups": {"sub": {"attrs": {}, "datasets": {}, "groups": {}}}})
    data = bytearray(path.read_bytes())
    root_header = struct.unpack_from("<Q", data, 64)[0]
    snod = data.index(b"SNOD")
    struct.pack_into("<Q", data, snod + 8 + 8, root_header)  # entry 0's object header -> the root
    path.write_bytes(bytes(data))
    with pytest.raises(ValueError, match=f"{path}.*reached twice"):
        h5lite.read_tree(path)

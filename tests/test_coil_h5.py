"""The reference's bundled .h5 coils read without h5py (cunibs_b200.h5lite through Coil.load).

The committed fixture tests/golden/magstim_d70.npz holds the MagStim D70 dipoles, extracted from
the reference's coil library by tests/golden/make_golden.py. Where the reference checkout is
present, every bundled coil is read and the D70 is checked against the fixture bit for bit.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from cunibs_b200 import Coil

GOLDEN = Path(__file__).resolve().parent / "golden" / "magstim_d70.npz"
COILS = Path("/root/reference/src/cunibs/coils")


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

"""Field files in the reference's format (src/mod_io.f90:7-149): pinned against
tests/golden/field_5x3x4.dat, written by the reference's own Python writer
(tests/golden/make_golden_io.py)."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_reads_reference_file():
    import prj
    want = np.load(os.path.join(GOLD, "field_5x3x4.npz"))["A"]
    assert prj.field_header(os.path.join(GOLD, "field_5x3x4.dat")) == (5, 3, 4)
    got = prj.read_field(os.path.join(GOLD, "field_5x3x4.dat"))
    np.testing.assert_array_equal(got, want)
    assert got[0, 0, 0] == np.pi


def test_writes_reference_bytes(tmp_path):
    import prj
    want = np.load(os.path.join(GOLD, "field_5x3x4.npz"))["A"]
    path = tmp_path / "out.dat"
    prj.write_field(str(path), np.asfortranarray(want))
    assert path.read_bytes() == open(os.path.join(GOLD, "field_5x3x4.dat"), "rb").read()


def test_halo_layout_round_trip(tmp_path):
    """halo=True reads and writes the interior of a halo'd array; the halos stay untouched."""
    import prj
    rng = np.random.default_rng(3)
    nx, nz, ny = 7, 5, 6
    H = np.asfortranarray(rng.normal(size=(nx + 2, nz + 2, ny + 2)))
    path = str(tmp_path / "h.dat")
    prj.write_field(path, H, halo=True)
    np.testing.assert_array_equal(prj.read_field(path), H[1:-1, 1:-1, 1:-1])
    G = np.full((nx + 2, nz + 2, ny + 2), -7.0, order="F")
    prj.read_field(path, G, halo=True)
    np.testing.assert_array_equal(G[1:-1, 1:-1, 1:-1], H[1:-1, 1:-1, 1:-1])
    G[1:-1, 1:-1, 1:-1] = -7.0
    assert np.all(G == -7.0)
    assert os.path.getsize(path) == 12 + 8 * nx * nz * ny


def test_grid_mismatch_and_short_file(tmp_path):
    import prj
    path = str(tmp_path / "a.dat")
    prj.write_field(path, np.zeros((4, 3, 2), order="F"))
    with pytest.raises(prj.PrjError) as e:
        prj.read_field(path, np.zeros((4, 3, 3), order="F"))
    assert e.value.code == prj.PRJ_ERR_ARG and "mismatch" in str(e.value)
    with open(path, "r+b") as f:
        f.truncate(12 + 8 * 10)
    with pytest.raises(prj.PrjError):
        prj.read_field(path)
    with pytest.raises(prj.PrjError):
        prj.read_field(str(tmp_path / "missing.dat"))

"""Readers of a reference case's geometry folder (prj_geom_read_*).

The fixture tests/golden/geom_12 was written by the reference's own
calc_bands.py writer (tests/golden/make_golden_io.py); the values it was written
from are in tests/golden/geom_12.npz.  The readers must give them back bit for
bit (read_column_r8, src/mod_utils.f90:14-35), refuse what the reference's
reader stops on, and feed a plan that solves like one built from yu.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

GEOM = os.path.join(GOLDEN, "geom_12")


@pytest.fixture(scope="module")
def ref():
    return dict(np.load(os.path.join(GOLDEN, "geom_12.npz")))


def test_bands_and_metrics_bitwise(ref):
    import prj
    geo = prj.read_geom(GEOM)
    abc, abc00 = ref["P_band_abc"], ref["P_band_abc_00"]
    for i in range(3):
        np.testing.assert_array_equal(geo["bands"][i], abc[:, i])
        np.testing.assert_array_equal(geo["bands"][3 + i], abc00[:, i])
    ny = int(ref["grid"][2])
    np.testing.assert_array_equal(geo["metrics"][0], ref["inv_dy_p"])
    np.testing.assert_array_equal(geo["metrics"][1], ref["dPdy_ddy_lh"][:ny, 0])
    np.testing.assert_array_equal(geo["metrics"][2], ref["dPdy_ddy_lh"][:ny, 1])
    # the engine's own band and metric builders agree with the files bit for bit
    for got, want in zip(prj.bands(ref["yu"], "reference"), geo["bands"]):
        np.testing.assert_array_equal(got, want)
    for got, want in zip(prj.metrics(ref["yu"]), geo["metrics"]):
        np.testing.assert_array_equal(got, want)


def test_base_params(ref):
    import prj
    c = prj.read_geom(GEOM)["params"]
    assert (c["nx"], c["nz"], c["ny"]) == tuple(int(v) for v in ref["grid"])
    assert (c["dx"], c["dz"]) == tuple(float(v) for v in ref["dxdz"])
    assert c["dtmax"] == float(ref["dtmax"]) and c["nstep"] == 100
    walls = [c[f"wall_{k}_{s}"] for s in ("bot", "top") for k in "UVW"]
    np.testing.assert_array_equal(walls, ref["walls"])
    assert c["use_incompressible"] == 1 and c["use_rough_surf"] == 0


def _col(path, icol, n, n_prev):
    import prj
    L = prj.load_library()
    out = np.zeros(max(n, 1))
    rc = L.prj_geom_read_column(os.fsencode(path), icol, n, n_prev, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return rc, out[:n], L.prj_last_error_string().decode()


def test_read_column_offsets_and_errors(ref, tmp_path):
    import prj
    f = os.path.join(GEOM, "P_band_abc.dat")
    rc, out, _ = _col(f, 1, 5, 4)  # a rank's slice: rows 4..8 of the b column
    assert rc == prj.PRJ_OK
    np.testing.assert_array_equal(out, ref["P_band_abc"][4:9, 1])
    rc, _, msg = _col(f, 0, 10, 3)  # rows 3..12 of 12: past the row count
    assert rc == prj.PRJ_ERR_ARG and "mismatch" in msg
    rc, _, msg = _col(f, 4, 3, 0)
    assert rc == prj.PRJ_ERR_ARG and "icol" in msg
    rc, _, msg = _col(str(tmp_path / "missing.dat"), 0, 1, 0)
    assert rc == prj.PRJ_ERR_ARG and "cannot open" in msg
    short = tmp_path / "short.dat"
    short.write_text("3\n1.0 2.0\n3.0\n4.0 5.0\n")
    rc, _, msg = _col(str(short), 1, 3, 0)
    assert rc == prj.PRJ_ERR_ARG and "fewer" in msg
    trunc = tmp_path / "trunc.dat"
    trunc.write_text("4\n1.0\n2.0\n")
    rc, _, msg = _col(str(trunc), 0, 3, 0)
    assert rc == prj.PRJ_ERR_ARG and "present" in msg


@pytest.mark.gpu
def test_plan_from_geom_solves_like_oracle(cuda_device, oracle, ref):
    import prj
    import torch
    from gpu_util import from_dev, to_dev
    nx, nz, ny = (int(v) for v in ref["grid"])
    dx, dz = (float(v) for v in ref["dxdz"])
    rhs = np.asfortranarray(np.random.default_rng(7).uniform(-1, 1, (nx, nz, ny)))
    with prj.Plan.from_geom(GEOM) as plan:
        assert plan.case["ny"] == ny
        t = to_dev(rhs)
        plan.poisson_fp64(t)
        torch.cuda.synchronize()
        P = from_dev(t)
    b6 = (*ref["P_band_abc"].T, *ref["P_band_abc_00"].T)
    Po, _ = oracle.poisson(rhs, dx, dz, b6)
    assert rel_l2(P, Po) <= 1e-12

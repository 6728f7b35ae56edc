"""CPU tests of the C ABI: the library builds, loads, exports every declared
symbol, and its host-only functions and argument checks work without a GPU."""
import ctypes
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HEADERS = sorted(glob.glob(os.path.join(ROOT, "include", "*.h")))


def declared_functions():
    names = []
    for h in HEADERS:
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+\s*\**\s*(prj_\w+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def test_headers_declare_functions():
    names = declared_functions()
    assert "prj_plan_create" in names and "prj_poisson_fp64" in names and "prj_projection_step" in names


def test_library_exports_every_declared_symbol():
    import prj
    lib = prj.load_library()
    out = subprocess.run(["nm", "-D", "--defined-only", prj.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT\s+(prj_\w+)", out))
    for name in declared_functions():
        assert name in exported, f"{name} declared in include/ but not exported"
        assert getattr(lib, name) is not None
    assert set(prj.EXPORTS) <= exported


def test_version_and_error_string():
    import prj
    lib = prj.load_library()
    assert b"sm_100a" in lib.prj_version()
    assert isinstance(lib.prj_last_error_string(), bytes)


def test_host_band_builders_match_oracle(oracle):
    import prj
    import pyoracle
    import workloads
    for yu in (workloads.tanh_faces(96), workloads.tanh_faces(7, 1.5), workloads.wall_refined_faces(64)):
        for mode in ("reference", "consistent"):
            got = prj.bands(yu, mode)
            for g, r in zip(got, pyoracle.bands(yu, mode)):
                np.testing.assert_array_equal(g, r)
            for g, r in zip(got, oracle.bands_from_yu(yu, mode)):
                np.testing.assert_array_equal(g, r)
        for g, r in zip(prj.metrics(yu), pyoracle.metrics(yu)):
            np.testing.assert_array_equal(g, r)


def test_host_band_builder_rejects_bad_grid():
    import prj
    with pytest.raises(prj.PrjError) as e:
        prj.bands(np.array([0.0, 1.0, 0.5]), "reference")
    assert e.value.code == prj.PRJ_ERR_ARG
    with pytest.raises(prj.PrjError):
        prj.metrics(np.array([0.0]))


@pytest.mark.parametrize("nx,nz,ny,dx", [(0, 8, 8, 0.1), (8, 0, 8, 0.1), (8, 8, 1, 0.1), (8, 8, 8, -1.0),
                                          (9000, 8, 8, 0.1), (8, 5000, 8, 0.1)])
def test_plan_create_rejects_bad_arguments(nx, nz, ny, dx):
    import prj
    b = [np.ones(max(ny, 1)) for _ in range(6)]
    lib = prj.load_library()
    h = ctypes.c_void_p()
    pp = [v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for v in b]
    rc = lib.prj_plan_create(nx, nz, ny, dx, 0.1, *pp, None, None, None, 0, 0, ctypes.byref(h))
    assert rc == prj.PRJ_ERR_ARG
    assert not h.value
    assert lib.prj_last_error_string()


def test_plan_create_rejects_nonfinite_bands():
    import prj
    b = [np.ones(8) for _ in range(6)]
    b[1][3] = np.nan
    with pytest.raises(prj.PrjError) as e:
        prj.Plan(8, 8, 8, 0.1, 0.1, b)
    assert e.value.code == prj.PRJ_ERR_ARG


def test_null_plan_is_rejected():
    import prj
    lib = prj.load_library()
    assert lib.prj_poisson_fp64(None, None, None) == prj.PRJ_ERR_ARG
    assert lib.prj_plan_destroy(None) == prj.PRJ_OK


def test_fortran_mirror_rejects_multirank():
    import prj
    b = [np.ones(8) for _ in range(6)]
    with pytest.raises(prj.PrjError) as e:
        prj.init_spec_poisson_multigpu(*b, 8, 8, 8, 10.0, 10.0, mpi_divs_z=2, mpi_divs_y=1)
    assert e.value.code == prj.PRJ_ERR_UNSUPPORTED

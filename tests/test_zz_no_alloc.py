"""GPU test of prj_poisson_fp64_noalloc, the Poisson solve for callers that
cannot allocate device memory (for example a Fortran/OpenACC host program that
owns every device array, or a time loop that must not call cudaMalloc).

It calls the entry point through the C ABI and compares each result with the
planned entry point (prj_plan_create + prj_poisson_fp64) and with the CPU
oracle on the same input, within the FP64 tolerance of the other parity tests,
on several calls in a row of different sizes (the calls share one static
scratch array, so each call must start from a clean state, its device error
word included).  It also checks that a grid too large for the scratch array is
refused with a clear message and leaves P untouched.

This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2
from gpu_util import from_dev, to_dev

pytestmark = pytest.mark.gpu

TOL_REL = 1e-12


def _noalloc(lib, bands6, dx, dz, t):
    import torch
    ny, nz, nx = t.shape
    b = [np.ascontiguousarray(v, dtype=np.float64) for v in bands6]
    ptr = [v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for v in b]
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return lib.prj_poisson_fp64_noalloc(nx, nz, ny, float(dx), float(dz), *ptr, ctypes.c_void_p(t.data_ptr()), stream)


def _planned(bands6, dx, dz, rhs):
    import prj
    import torch
    nx, nz, ny = rhs.shape
    t = to_dev(rhs)
    with prj.Plan(nx, nz, ny, dx, dz, bands6) as plan:
        plan.poisson_fp64(t)
        torch.cuda.synchronize()
    return from_dev(t)


def _case(shape, seed, mode):
    import prj
    nx, nz, ny = shape
    rng = np.random.default_rng(seed)
    rhs = np.asfortranarray(rng.uniform(-1.0, 1.0, shape))
    yu = np.concatenate([[0.0], np.cumsum(rng.uniform(0.05, 0.2, ny))])
    dx, dz = rng.uniform(0.02, 0.2, 2)
    return rhs, prj.bands(yu, mode), dx, dz


def test_noalloc_matches_planned_solve(cuda_device, oracle):
    import prj
    import torch
    lib = prj.load_library()
    cases = [((128, 64, 96), 1, "reference"), ((30, 17, 21), 2, "consistent"),
             ((256, 128, 128), 3, "reference"), ((128, 64, 96), 1, "reference")]
    for shape, seed, mode in cases:
        rhs, b6, dx, dz = _case(shape, seed, mode)
        want = _planned(b6, dx, dz, rhs)
        t = to_dev(rhs)
        rc = _noalloc(lib, b6, dx, dz, t)
        assert rc == prj.PRJ_OK, lib.prj_last_error_string()
        torch.cuda.synchronize()
        got = from_dev(t)
        assert np.isfinite(got).all()
        assert rel_l2(got, want) <= TOL_REL, (shape, rel_l2(got, want))
        Po, _ = oracle.poisson(rhs, dx, dz, b6)
        assert rel_l2(got, Po) <= TOL_REL, (shape, rel_l2(got, Po))


def test_noalloc_rejects_grid_beyond_scratch(cuda_device):
    import prj
    import torch
    lib = prj.load_library()
    shape = (512, 256, 64)  # about 8.4e6 points: more scratch than the static array holds
    rhs, b6, dx, dz = _case(shape, 4, "reference")
    t = to_dev(rhs)
    rc = _noalloc(lib, b6, dx, dz, t)
    assert rc == prj.PRJ_ERR_ARG
    msg = lib.prj_last_error_string().decode()
    assert "scratch" in msg and "512 x 256 x 64" in msg
    torch.cuda.synchronize()
    np.testing.assert_array_equal(from_dev(t), rhs)

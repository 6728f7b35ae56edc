"""The one-solve-over-several-GPUs stages (prj_dist_*), run as 2 to 4 ranks emulated on one
GPU (one plan per rank, the all-to-all as in-process copies): the assembled P equals the
single-GPU solve bit for bit, with uneven plane and wavenumber splits.  Bad ranges are
refused with PRJ_ERR_ARG.  No test here runs on several GPUs (this harness has one)."""
import numpy as np
import pytest

from gpu_util import from_dev, to_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3, 4])
@pytest.mark.parametrize("shape", [(64, 37, 48), (96, 20, 64), (100, 9, 32)])
def test_emulated_ranks_equal_single_gpu(cuda_device, monkeypatch, world, shape):
    import prj
    import prj_dist
    import workloads
    nx, ny, nz = shape
    rhs, yu, dx, dz = workloads.poisson_rhs(nx, ny, nz, seed=31)
    bands = prj.bands(yu, "consistent")
    with prj.Plan(nx, nz, ny, dx, dz, bands) as plan:
        plan.set_tuning(z_mode=0)  # the split z kernels, which the ranks run
        ref = to_dev(rhs)
        plan.poisson_fp64(ref)
        ref = from_dev(ref)
    plans = [prj.Plan(nx, nz, ny, dx, dz, bands) for _ in range(world)]
    try:
        P = to_dev(rhs)
        prj_dist.solve_emulated(plans, P, world)
        out = from_dev(P)
    finally:
        for p in plans:
            p.close()
    np.testing.assert_array_equal(out, ref)


def test_bad_ranges_are_refused(cuda_device):
    import ctypes
    import torch
    import prj
    import workloads
    nx, ny, nz = 64, 8, 48
    rhs, yu, dx, dz = workloads.poisson_rhs(nx, ny, nz, seed=1)
    L = prj.load_library()
    with prj.Plan(nx, nz, ny, dx, dz, prj.bands(yu, "consistent")) as plan:
        buf = torch.zeros(ny * nz * nx, dtype=torch.float64, device="cuda")
        ptr = ctypes.c_void_p(buf.data_ptr())
        assert L.prj_dist_forward(plan.handle, ptr, 3, 2, None) == prj.PRJ_ERR_ARG
        assert L.prj_dist_forward(plan.handle, ptr, 0, ny + 1, None) == prj.PRJ_ERR_ARG
        bad = (ctypes.c_int * 3)(0, 10, 20)  # does not end at nx/2+1 = 33
        assert L.prj_dist_pack(plan.handle, 0, ny, bad, 2, ptr, None) == prj.PRJ_ERR_ARG
        assert L.prj_dist_thomas(plan.handle, ptr, 5, 40, None) == prj.PRJ_ERR_ARG
        torch.cuda.synchronize()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("shape", [(96, 40, 48), (64, 21, 32)])
def test_emulated_projection_step_equals_single_gpu(cuda_device, monkeypatch, world, shape):
    """The whole projection step over ranks (divergence of each rank's planes, the
    exchanges, the solve, the neighbour P plane, each rank's correction) equals the
    single-GPU step bit for bit in U, V, W (halos and wall planes included) and P."""
    import torch
    import prj
    import prj_dist
    import workloads
    from test_gpu_projection import run_engine
    nx, ny, nz = shape
    Uh, Vh, Wh, yu, dx, dz = workloads.projection_inputs(nx, ny, nz, seed=9)
    for F in (Uh, Vh, Wh):
        workloads.fill_halos(F)
    wall = (0.01, 0.0, -0.02, 0.03, 0.0, 0.04)
    with prj.Plan.from_yu(nx, nz, dx, dz, yu, "consistent") as plan:
        plan.set_tuning(z_mode=0)  # the split z kernels, which the ranks run
        ref = run_engine(plan, Uh, Vh, Wh, 0.6, wall)
    plans = [prj.Plan.from_yu(nx, nz, dx, dz, yu, "consistent") for _ in range(world)]
    try:
        t = lambda A: torch.from_numpy(np.ascontiguousarray(A.transpose(2, 1, 0))).cuda()
        dUh, dVh, dWh = t(Uh), t(Vh), t(Wh)
        dU, dV, dW = (torch.full_like(dUh, np.nan) for _ in range(3))
        dP = torch.zeros((ny, nz, nx), dtype=torch.float64, device="cuda")
        params = prj.StepParams(0.6, *wall, 0)
        prj_dist.project_emulated(plans, dUh, dVh, dWh, dU, dV, dW, dP, params, world)
        torch.cuda.synchronize()
        got = [A.cpu().numpy().transpose(2, 1, 0) for A in (dU, dV, dW, dP)]
    finally:
        for p in plans:
            p.close()
    for a, b in zip(got, ref[:4]):
        np.testing.assert_array_equal(a, b)

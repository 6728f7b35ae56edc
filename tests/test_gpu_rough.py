"""GPU tests of the rough-wall channel workload: wall-refined faces (uniform below
y = 0.1, 1.5% growth per cell) and a predictor zeroed inside a random roughness.

Tolerances: FP64 pressure within 1e-12 relative L2 of the oracle; FP32 storage with
FP64 refinement within 1e-11 of the FP64 pressure; max|div u| over the fluid cells
<= 1e-10 (divergence-consistent bands)."""
import numpy as np
import pytest

from conftest import rel_l2
from gpu_util import empty_like_dev, from_dev, to_dev

pytestmark = pytest.mark.gpu


def run(plan, Uh, Vh, Wh, mode):
    import torch
    g = plan.grid
    hs = (g.nx + 2, g.nz + 2, g.ny + 2)
    dU, dV, dW = (empty_like_dev(hs) for _ in range(3))
    dP = empty_like_dev((g.nx, g.nz, g.ny))
    st = plan.projection_step(to_dev(Uh), to_dev(Vh), to_dev(Wh), dU, dV, dW, dP, 1.0, mode=mode)
    torch.cuda.synchronize()
    return from_dev(dU), from_dev(dV), from_dev(dW), from_dev(dP), st


def fluid_div(U, V, W, dx, dz, idy, solid):
    """max |div u| over fluid cells of corrected halo'd [x+2, z+2, y+2] fields."""
    d = (U[2:, 1:-1, 1:-1] - U[1:-1, 1:-1, 1:-1]) / dx
    d += (W[1:-1, 2:, 1:-1] - W[1:-1, 1:-1, 1:-1]) / dz
    d += (V[1:-1, 1:-1, 2:] - V[1:-1, 1:-1, 1:-1]) * idy[None, None, :]
    return np.abs(d[~solid]).max()


def test_rough_fp64_matches_oracle(cuda_device, oracle):
    import prj
    import workloads
    nx, ny, nz = 96, 64, 48
    Uh, Vh, Wh, yu, dx, dz, solid = workloads.rough_projection_inputs(nx, ny, nz)
    assert 0.0 < solid.mean() < 0.5
    with prj.Plan.from_yu(nx, nz, dx, dz, yu, "consistent") as plan:
        U, V, W, P, st = run(plan, Uh, Vh, Wh, prj.MODE_FP64)
    Uo, Vo, Wo, Po = oracle.projection(Uh, Vh, Wh, dx, dz, 1.0, yu, "consistent")
    assert rel_l2(P, Po) <= 1e-12
    for a, b in ((U, Uo), (V, Vo), (W, Wo)):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
    idy = prj.metrics(yu)[0]
    assert fluid_div(U, V, W, dx, dz, idy, solid) <= 1e-10
    assert st["div_maxabs"] <= 1e-10


def test_rough_mixed_matches_fp64(cuda_device):
    import prj
    import workloads
    nx, ny, nz = 192, 128, 96
    Uh, Vh, Wh, yu, dx, dz, solid = workloads.rough_projection_inputs(nx, ny, nz)
    with prj.Plan.from_yu(nx, nz, dx, dz, yu, "consistent") as plan:
        _, _, _, P64, s64 = run(plan, Uh, Vh, Wh, prj.MODE_FP64)
        U, V, W, P32, s32 = run(plan, Uh, Vh, Wh, prj.MODE_FP32_REFINE)
    assert rel_l2(P32, P64) <= 1e-11, rel_l2(P32, P64)
    assert s32["last_update_rel"] < 1e-6
    idy = prj.metrics(yu)[0]
    assert fluid_div(U, V, W, dx, dz, idy, solid) <= 1e-10
    assert s32["div_maxabs"] <= 1e-10

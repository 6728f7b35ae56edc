"""GPU tests of the variable-density projection (prj_projection_step_vd) against the oracle's
restatement of mod_cfd_subroutines.f90:538-573 and :1153-1221.

Tolerances: P and u, v, w within 1e-12 (relative L2 / max-norm) of the oracle; the halos of
P_next are exact copies of the engine's own P; the FP32-storage + refinement mode within 1e-11
of FP64.  The reference's own tests hold no golden data for this branch, so parity rests on the
restatement and on the exact constant-density reduction to the incompressible step."""
import numpy as np
import pytest

from conftest import rel_l2
from gpu_util import empty_like_dev, from_dev, to_dev

pytestmark = pytest.mark.gpu


def run_vd(plan, fields, dt, wall=(0.0,) * 6, mode=0):
    import torch
    Uh, Vh, Wh, rho, Pn, Po, div = (to_dev(a) for a in fields)
    g = plan.grid
    hs = (g.nx + 2, g.nz + 2, g.ny + 2)
    U, V, W, Pnext = (empty_like_dev(hs) for _ in range(4))
    P = empty_like_dev((g.nx, g.nz, g.ny))
    st = plan.projection_step_vd(Uh, Vh, Wh, rho, Pn, Po, div, U, V, W, P, Pnext, dt, mode=mode, wall=wall)
    torch.cuda.synchronize()
    return from_dev(U), from_dev(V), from_dev(W), from_dev(P), from_dev(Pnext), st


@pytest.mark.parametrize("band_mode", ["reference", "consistent"])
@pytest.mark.parametrize("shape", [(64, 48, 32), (30, 17, 21), (128, 96, 64)])
def test_vd_matches_oracle(cuda_device, oracle, band_mode, shape):
    import prj
    import workloads
    nx, ny, nz = shape
    Uh, Vh, Wh, rho, Pn, Po, div, yu, dx, dz = workloads.vd_inputs(nx, ny, nz)
    wall = (0.01, 0.0, -0.02, 0.03, 0.0, 0.04)
    with prj.Plan.from_yu(nx, nz, dx, dz, yu, band_mode) as plan:
        U, V, W, P, Pnext, st = run_vd(plan, (Uh, Vh, Wh, rho, Pn, Po, div), 0.45, wall)
    Uo, Vo, Wo, Po_, Pno, rmin = oracle.projection_vd(Uh, Vh, Wh, rho, Pn, Po, div, dx, dz, 0.45, yu, band_mode, wall)
    assert st["rho_min"] == rmin == rho[1:-1, 1:-1, 1:-1].min()
    assert rel_l2(P, Po_) <= 1e-12
    assert rel_l2(Pnext, Pno) <= 1e-12
    for a, b in ((U, Uo), (V, Vo), (W, Wo)):
        assert np.isfinite(a).all()
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
    # P_next: the engine's own P with periodic halos and wall ghost planes, exactly
    np.testing.assert_array_equal(Pnext, workloads.fill_halos(np.pad(P, 1)))


@pytest.mark.parametrize("where", ["x", "z", "y"])
def test_vd_rho_min_ignores_halos(cuda_device, oracle, where):
    """rho_min is the minimum over the interior (mod_cfd_subroutines.f90:476-486): a smaller
    density planted in the x halo columns, the z halo rows or the wall ghost planes changes
    neither rho_min nor the agreement with the oracle (both read the same halo'd arrays)."""
    import prj
    import workloads
    nx, ny, nz = 30, 17, 21
    Uh, Vh, Wh, rho, Pn, Po, div, yu, dx, dz = workloads.vd_inputs(nx, ny, nz)
    rho = np.array(rho, order="F")
    inner_min = rho[1:-1, 1:-1, 1:-1].min()
    tiny = 0.5 * inner_min
    cells = {"x": [(0, 5, 7), (nx + 1, 3, 2)], "z": [(4, 0, 6), (9, nz + 1, 3)],
             "y": [(6, 7, 0), (2, 3, ny + 1)]}[where]
    for c in cells:
        rho[c] = tiny
    with prj.Plan.from_yu(nx, nz, dx, dz, yu, "consistent") as plan:
        U, V, W, P, Pnext, st = run_vd(plan, (Uh, Vh, Wh, rho, Pn, Po, div), 0.45)
    Uo, Vo, Wo, Po_, Pno, rmin = oracle.projection_vd(Uh, Vh, Wh, rho, Pn, Po, div, dx, dz, 0.45, yu,
                                                      "consistent", (0.0,) * 6)
    assert st["rho_min"] == rmin == inner_min
    assert rel_l2(P, Po_) <= 1e-12
    for a, b in ((U, Uo), (V, Vo), (W, Wo)):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_vd_constant_density_equals_incompressible(cuda_device):
    """rho = 2, div_now = 0: the variable-density step is the incompressible step bit for bit
    (P scaled by rho_min = 2 exactly)."""
    import prj
    import workloads
    nx, ny, nz = 96, 64, 48
    Uh, Vh, Wh, rho, Pn, Po, div, yu, dx, dz = workloads.vd_inputs(nx, ny, nz, rho_const=2.0)
    div[...] = 0.0
    with prj.Plan.from_yu(nx, nz, dx, dz, yu, "consistent") as plan:
        U, V, W, P, Pnext, st = run_vd(plan, (Uh, Vh, Wh, rho, Pn, Po, div), 0.8)
        dU, dV, dW = (empty_like_dev(Uh.shape) for _ in range(3))
        dP = empty_like_dev((nx, nz, ny))
        plan.projection_step(to_dev(Uh), to_dev(Vh), to_dev(Wh), dU, dV, dW, dP, 0.8)
    np.testing.assert_array_equal(P, 2.0 * from_dev(dP))
    for a, b in ((U, dU), (V, dV), (W, dW)):
        np.testing.assert_array_equal(a, from_dev(b))
    assert st["div_maxabs"] <= 1e-10


def test_vd_mixed_matches_fp64(cuda_device):
    import prj
    import workloads
    nx, ny, nz = 128, 96, 64
    fields = workloads.vd_inputs(nx, ny, nz, seed=8)
    yu, dx, dz = fields[7:]
    with prj.Plan.from_yu(nx, nz, dx, dz, yu, "consistent") as plan:
        U64, _, _, P64, _, s64 = run_vd(plan, fields[:7], 0.6)
        U32, _, _, P32, _, s32 = run_vd(plan, fields[:7], 0.6, mode=prj.MODE_FP32_REFINE)
    assert rel_l2(P32, P64) <= 1e-11
    assert np.abs(U32 - U64).max() <= 1e-10 * np.abs(U64).max()
    assert s32["refine_iters"] >= 1 and s64["refine_iters"] == 0


def test_vd_rejects_bad_arguments(cuda_device):
    import prj
    import workloads
    nx, ny, nz = 16, 8, 12
    Uh, Vh, Wh, rho, Pn, Po, div, yu, dx, dz = workloads.vd_inputs(nx, ny, nz)
    d = [to_dev(a) for a in (Uh, Vh, Wh, rho, Pn, Po, div)]
    hs = Uh.shape
    U, V, W, Pnext = (empty_like_dev(hs) for _ in range(4))
    P = empty_like_dev((nx, nz, ny))
    # P_next aliasing P_now (the rotation must be done by the caller, not in place)
    with prj.Plan.from_yu(nx, nz, dx, dz, yu) as plan:
        with pytest.raises(prj.PrjError) as e:
            plan.projection_step_vd(*d, U, V, W, P, d[4], 1.0)
        assert e.value.code == prj.PRJ_ERR_ARG
    # a plan without inv_dy_p_pad
    with prj.Plan(nx, nz, ny, dx, dz, prj.bands(yu), prj.metrics(yu)) as plan:
        with pytest.raises(prj.PrjError) as e:
            plan.projection_step_vd(*d, U, V, W, P, Pnext, 1.0)
        assert e.value.code == prj.PRJ_ERR_STATE

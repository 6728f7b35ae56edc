"""Parity of the projection step at the headline size and at a mid-size rough wall.

768 x 384 x 384 (Lx = 2 pi, Lz = pi, tanh faces with beta = 2, Poiseuille predictor
plus N(0, 0.1) noise, the workload of bench.py): the engine's P, U, V, W against the
CPU oracle's restatement of the reference's FFTW path (PSM:328-554 with the
divergence MCS:527-537 and correction MCS:1086-1152, :1223-1244) on the same input,
in both band modes.  The reference's own bands (mk_P_abc) are the parity mode; the
divergence-consistent bands are the mode the bench measures.

384 x 256 x 384 rough wall (the wall-refined grid and roughness mask of the
1536 x 512 x 768 case): FP64 against the oracle, and FP32 storage with FP64
refinement against the oracle.

Tolerances: P within 1e-12 relative L2 (FP64) or 1e-11 (FP32 + refinement);
velocities within 1e-12 (1e-11) of their largest magnitude, element-wise.
"""
import numpy as np
import pytest

from conftest import rel_l2
from gpu_util import empty_like_dev, from_dev, to_dev

pytestmark = pytest.mark.gpu


def run(plan, Uh, Vh, Wh, dt, mode):
    import torch
    g = plan.grid
    hs = (g.nx + 2, g.nz + 2, g.ny + 2)
    dU, dV, dW = (empty_like_dev(hs) for _ in range(3))
    dP = empty_like_dev((g.nx, g.nz, g.ny))
    st = plan.projection_step(to_dev(Uh), to_dev(Vh), to_dev(Wh), dU, dV, dW, dP, dt, mode=mode)
    torch.cuda.synchronize()
    out = tuple(from_dev(t) for t in (dU, dV, dW, dP))
    del dU, dV, dW, dP
    torch.cuda.empty_cache()
    return out + (st,)


def compare(got, want, tol_p, tol_u):
    U, V, W, P = got[:4]
    Uo, Vo, Wo, Po = want
    rp = rel_l2(P, Po)
    assert rp <= tol_p, rp
    for a, b in ((U, Uo), (V, Vo), (W, Wo)):
        err = float(np.abs(a - b).max())
        assert err <= tol_u * float(np.abs(b).max()), err
    return rp


@pytest.mark.parametrize("band_mode", ["reference", "consistent"])
def test_headline_step_matches_oracle(cuda_device, oracle, band_mode):
    import prj
    import workloads
    nx, ny, nz = 768, 384, 384
    Uh, Vh, Wh, yu, dx, dz = workloads.projection_inputs(nx, ny, nz, seed=1)
    with prj.Plan.from_yu(nx, nz, dx, dz, yu, band_mode) as plan:
        got = run(plan, Uh, Vh, Wh, 1.0, prj.MODE_FP64)
    want = oracle.projection(Uh, Vh, Wh, dx, dz, 1.0, yu, band_mode)
    compare(got, want, 1e-12, 1e-12)
    if band_mode == "consistent":
        assert got[4]["div_maxabs"] <= 1e-10


def test_rough_mid_size_matches_oracle(cuda_device, oracle):
    import prj
    import workloads
    nx, ny, nz = 384, 256, 384
    Uh, Vh, Wh, yu, dx, dz, solid = workloads.rough_projection_inputs(nx, ny, nz)
    assert 0.0 < solid.mean() < 0.5
    want = oracle.projection(Uh, Vh, Wh, dx, dz, 1.0, yu, "consistent")
    with prj.Plan.from_yu(nx, nz, dx, dz, yu, "consistent") as plan:
        got64 = run(plan, Uh, Vh, Wh, 1.0, prj.MODE_FP64)
        compare(got64, want, 1e-12, 1e-12)
        del got64
        got32 = run(plan, Uh, Vh, Wh, 1.0, prj.MODE_FP32_REFINE)
    compare(got32, want, 1e-11, 1e-11)

"""GPU parity of the full projection step (divergence -> Poisson -> correction)
against the C oracle's restatement of build_vars / run_spec / update_vars."""
import numpy as np
import pytest

from conftest import rel_l2
from gpu_util import empty_like_dev, from_dev, to_dev

pytestmark = pytest.mark.gpu

WALL = (0.0, 0.0, 0.0, 0.0, 0.0, 0.0)


def run_engine(plan, Uh, Vh, Wh, dt, wall=WALL, mode=0):
    import torch
    g = plan.grid
    hs = (g.nx + 2, g.nz + 2, g.ny + 2)
    dUh, dVh, dWh = to_dev(Uh), to_dev(Vh), to_dev(Wh)
    dU, dV, dW = (empty_like_dev(hs) for _ in range(3))
    dP = empty_like_dev((g.nx, g.nz, g.ny))
    st = plan.projection_step(dUh, dVh, dWh, dU, dV, dW, dP, dt, mode=mode, wall=wall)
    torch.cuda.synchronize()
    return from_dev(dU), from_dev(dV), from_dev(dW), from_dev(dP), st


@pytest.mark.parametrize("band_mode", ["reference", "consistent"])
@pytest.mark.parametrize("shape", [(64, 48, 32), (30, 17, 21), (7, 6, 5), (128, 96, 64)])
def test_projection_matches_oracle(cuda_device, oracle, band_mode, shape):
    import prj
    import workloads
    nx, ny, nz = shape
    Uh, Vh, Wh, yu, dx, dz = workloads.projection_inputs(nx, ny, nz, seed=1)
    dt = 0.37
    wall = (0.01, 0.0, -0.02, 0.03, 0.0, 0.04)
    with prj.Plan.from_yu(nx, nz, dx, dz, yu, band_mode) as plan:
        U, V, W, P, st = run_engine(plan, Uh, Vh, Wh, dt, wall)
    Uo, Vo, Wo, Po = oracle.projection(Uh, Vh, Wh, dx, dz, dt, yu, band_mode, wall)
    assert rel_l2(P, Po) <= 1e-12
    for a, b in ((U, Uo), (V, Vo), (W, Wo)):
        assert np.isfinite(a).all()
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
    idy, _, _ = prj.metrics(yu)
    d_or = oracle.div_maxabs(Uo, Vo, Wo, dx, dz, idy)
    assert st["div_maxabs"] == pytest.approx(oracle.div_maxabs(U, V, W, dx, dz, idy), rel=1e-9, abs=1e-13)
    if band_mode == "consistent":
        assert st["div_maxabs"] <= 1e-10 and d_or <= 1e-10
    assert st["p_maxabs"] == pytest.approx(np.abs(P).max(), rel=1e-15)


def test_boundary_fill_is_exact(cuda_device, oracle):
    """Halos and wall slices equal the oracle bit for bit (they are copies)."""
    import prj
    import workloads
    nx, ny, nz = 12, 8, 10
    Uh, Vh, Wh, yu, dx, dz = workloads.projection_inputs(nx, ny, nz, seed=7)
    wall = (0.5, 0.25, -0.5, 1.5, -0.25, 2.0)
    with prj.Plan.from_yu(nx, nz, dx, dz, yu) as plan:
        U, V, W, P, _ = run_engine(plan, Uh, Vh, Wh, 1.0, wall)
    assert np.all(U[:, :, 0] == 0.5) and np.all(U[:, :, -1] == 1.5)
    assert np.all(V[:, :, 0] == 0.25) and np.all(V[:, :, 1] == 0.25) and np.all(V[:, :, -1] == -0.25)
    assert np.all(W[:, :, 0] == -0.5) and np.all(W[:, :, -1] == 2.0)
    for F in (U, V, W):
        np.testing.assert_array_equal(F[0, :, 1:-1], F[nx, :, 1:-1])
        np.testing.assert_array_equal(F[nx + 1, :, 1:-1], F[1, :, 1:-1])
        np.testing.assert_array_equal(F[:, 0, 1:-1], F[:, nz, 1:-1])
        np.testing.assert_array_equal(F[:, nz + 1, 1:-1], F[:, 1, 1:-1])


def test_host_entry_equals_device_entry(cuda_device):
    import prj
    import workloads
    nx, ny, nz = 48, 32, 40
    Uh, Vh, Wh, yu, dx, dz = workloads.projection_inputs(nx, ny, nz, seed=2)
    with prj.Plan.from_yu(nx, nz, dx, dz, yu, "consistent") as plan:
        U, V, W, P, st = run_engine(plan, Uh, Vh, Wh, 0.5)
        hs = (nx + 2, nz + 2, ny + 2)
        Uh2, Vh2, Wh2 = (np.zeros(hs, order="F") for _ in range(3))
        P2 = np.zeros((nx, nz, ny), order="F")
        st2 = plan.projection_step(Uh, Vh, Wh, Uh2, Vh2, Wh2, P2, 0.5)
    np.testing.assert_array_equal(U, Uh2)
    np.testing.assert_array_equal(V, Vh2)
    np.testing.assert_array_equal(W, Wh2)
    np.testing.assert_array_equal(P, P2)
    assert st["div_maxabs"] == st2["div_maxabs"]


def test_projection_full_size_is_solenoidal(cuda_device):
    """768 x 384 x 384 with divergence-consistent bands: max|div u| <= 1e-10."""
    import prj
    import workloads
    nx, ny, nz = 768, 384, 384
    Uh, Vh, Wh, yu, dx, dz = workloads.projection_inputs(nx, ny, nz, seed=1)
    with prj.Plan.from_yu(nx, nz, dx, dz, yu, "consistent") as plan:
        U, V, W, P, st = run_engine(plan, Uh, Vh, Wh, 1.0)
    assert st["div_maxabs"] <= 1e-10, st
    assert np.isfinite(P).all()


def test_projection_rejects_bad_params(cuda_device):
    import prj
    import torch
    import workloads
    nx, ny, nz = 8, 6, 4
    Uh, Vh, Wh, yu, dx, dz = workloads.projection_inputs(nx, ny, nz)
    with prj.Plan.from_yu(nx, nz, dx, dz, yu) as plan:
        hs = (nx + 2, nz + 2, ny + 2)
        f = [to_dev(Uh), to_dev(Vh), to_dev(Wh)] + [empty_like_dev(hs) for _ in range(3)] + [empty_like_dev((nx, nz, ny))]
        with pytest.raises(prj.PrjError) as e:
            plan.projection_step(*f, dt=0.0)
        assert e.value.code == prj.PRJ_ERR_ARG
        with pytest.raises(prj.PrjError) as e:
            plan.projection_step(*f, dt=1.0, mode=7)
        assert e.value.code == prj.PRJ_ERR_ARG
    # a Poisson-only plan has no metrics for the projection
    with prj.Plan(nx, nz, ny, dx, dz, prj.bands(yu)) as plan:
        with pytest.raises(prj.PrjError) as e:
            plan.projection_step(*f, dt=1.0)
        assert e.value.code == prj.PRJ_ERR_STATE
    torch.cuda.synchronize()


def test_pipelined_host_steps_match_sync(cuda_device):
    """Three pipelined host-buffer steps (alternating staging slots) give the synchronous call's
    outputs bit for bit."""
    import prj
    import torch
    import workloads
    nx, ny, nz = 64, 48, 32
    cases = [workloads.projection_inputs(nx, ny, nz, seed=s) for s in (21, 22, 23)]
    yu, dx, dz = cases[0][3:]
    pin = lambda shape: torch.empty(tuple(reversed(shape)), dtype=torch.float64).pin_memory().numpy().T
    hs = (nx + 2, nz + 2, ny + 2)
    with prj.Plan.from_yu(nx, nz, dx, dz, yu, "consistent") as plan:
        ins, outs = [], []
        for Uh, Vh, Wh, *_ in cases:
            bufs = [pin(hs) for _ in range(3)]
            for b, a in zip(bufs, (Uh, Vh, Wh)):
                b[...] = a
            ins.append(bufs)
            outs.append([pin(hs) for _ in range(3)] + [pin((nx, nz, ny))])
        for i, o in zip(ins, outs):
            plan.projection_step_host_async(*i, *o, 0.8)
        plan.host_async_wait()
        for (Uh, Vh, Wh, *_), o in zip(cases, outs):
            want = [np.zeros(hs, order="F") for _ in range(3)] + [np.zeros((nx, nz, ny), order="F")]
            plan.projection_step(Uh, Vh, Wh, *want, 0.8, stats=False)
            for a, b in zip(o, want):
                np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("shape", [(64, 48, 32), (30, 17, 21)])
def test_basic_z_kernel_matches_oracle(cuda_device, oracle, monkeypatch, shape):
    """z_mode 2 selects the first, unpipelined per-wavenumber z kernel."""
    import prj
    import workloads
    nx, ny, nz = shape
    Uh, Vh, Wh, yu, dx, dz = workloads.projection_inputs(nx, ny, nz, seed=7)
    with prj.Plan.from_yu(nx, nz, dx, dz, yu, "consistent") as plan:
        plan.set_tuning(z_mode=2)
        assert plan.tuning["z_mode"] == 2
        U, V, W, P, st = run_engine(plan, Uh, Vh, Wh, 0.5)
    Uo, Vo, Wo, Po = oracle.projection(Uh, Vh, Wh, dx, dz, 0.5, yu, "consistent")
    assert rel_l2(P, Po) <= 1e-12
    for a, b in ((U, Uo), (V, Vo), (W, Wo)):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()

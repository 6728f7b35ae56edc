"""GPU parity of the FP64 Poisson solve (the drop-in for run_spec_poisson_multigpu).

Every case calls the engine through its C ABI (prj.py -> libprj_b200.so) and
compares with the reference's golden outputs and with the C oracle, using the
reference's acceptance criterion (max |P - P_ref| <= 1e-10 after mean removal,
tests/test_poisson_solver_and_ibm_rand/main_poi_test.f90:252-262) plus a
relative-L2 bound of 1e-12.
"""
import numpy as np
import pytest

from conftest import mean_removed_maxabs, rel_l2
from gpu_util import from_dev, to_dev

pytestmark = pytest.mark.gpu

TOL_MAXABS = 1e-10   # reference's own bound
TOL_REL = 1e-12      # FP64 engine vs FP64 oracle


def solve_dev(plan, A):
    t = to_dev(A)
    plan.poisson_fp64(t)
    import torch
    torch.cuda.synchronize()
    return from_dev(t)


@pytest.mark.parametrize("it", range(10))
def test_seed0_trials_match_reference(cuda_device, trials, oracle, it):
    import prj
    t = trials[it]
    nx, nz, ny = t["shape"]
    with prj.Plan(nx, nz, ny, t["dx"], t["dz"], t["bands"]) as plan:
        P = solve_dev(plan, t["A"])
    assert mean_removed_maxabs(P, t["B"]) <= TOL_MAXABS
    assert rel_l2(P, t["B"]) <= TOL_REL
    Po, _ = oracle.poisson(t["A"], t["dx"], t["dz"], t["bands"])
    assert rel_l2(P, Po) <= TOL_REL


def test_fortran_mirror_entry_points(cuda_device, trials, capsys):
    """init_spec / run_spec mirror the reference module (inv_dx, inv_dz, in-place P)."""
    import prj
    t = trials[5]
    nx, nz, ny = t["shape"]
    plan = prj.init_spec_poisson_multigpu(*t["bands"], nx, nz, ny, 1.0 / t["dx"], 1.0 / t["dz"])
    assert "min_abs_div_bacp" in capsys.readouterr().out
    P = t["A"].copy(order="F")
    prj.run_spec_poisson_multigpu(plan, P)  # host buffers, in place
    assert mean_removed_maxabs(P, t["B"]) <= TOL_MAXABS
    plan.close()


def test_channel_128x96x64_golden(cuda_device, channel_golden, oracle):
    import prj
    import workloads
    g = channel_golden
    nx, nz, ny = (int(v) for v in g["shape"])
    rhs, yu, dx, dz = workloads.poisson_rhs(nx, ny, nz, beta=2.0, seed=0)
    with prj.Plan.from_yu(nx, nz, dx, dz, yu) as plan:
        P = solve_dev(plan, rhs)
        Ph = rhs.copy(order="F")
        plan.poisson_fp64(Ph)  # host-buffer entry point
    s = tuple(int(v) for v in g["stride"])
    assert rel_l2(P[::s[0], ::s[1], ::s[2]], g["P_sub"]) <= TOL_REL
    assert np.isclose((P ** 2).sum(), float(g["P_sumsq"]), rtol=1e-11)
    np.testing.assert_array_equal(P, Ph)
    Po, _ = oracle.poisson(rhs, dx, dz, prj.bands(yu))
    assert rel_l2(P, Po) <= TOL_REL
    assert mean_removed_maxabs(P, Po) <= TOL_MAXABS


def test_min_pivot_matches_oracle(cuda_device, oracle):
    import prj
    import workloads
    rhs, yu, dx, dz = workloads.poisson_rhs(32, 24, 16)
    b = prj.bands(yu)
    _, mp = oracle.poisson(rhs, dx, dz, b)
    with prj.Plan(32, 16, 24, dx, dz, b) as plan:
        assert plan.min_pivot == pytest.approx(mp, rel=1e-14)


def test_mms_convergence_matches_reference(cuda_device, mms):
    """Manufactured solution of py_poi_solver.py:236-327 (second order, same errors)."""
    import prj
    from make_golden import mms_fields
    Lx, Ly, Lz = mms["L"]
    errs = []
    for N, eref in zip(mms["N"], mms["err"]):
        rhs, p, yu, dx, dz = mms_fields(str(mms["expr_p"]), str(mms["expr_rhs"]), Lx, Ly, Lz, int(N))
        nx, nz, ny = rhs.shape
        with prj.Plan(nx, nz, ny, dx, dz, prj.bands(yu)) as plan:
            P = solve_dev(plan, rhs)
        e = float(np.abs((p - p.mean()) - (P - P.mean())).max())
        assert abs(e - eref) <= 1e-9 * eref, (N, e, eref)
        errs.append(e)
    assert 3.5 < errs[-2] / errs[-1] < 4.6


@pytest.mark.parametrize("shape", [(1, 1, 2), (2, 1, 3), (1, 7, 4), (3, 3, 6), (5, 10, 10), (17, 13, 9),
                                   (37, 11, 5), (29, 31, 7), (64, 96, 33), (96, 128, 40), (250, 6, 3),
                                   (162, 125, 12), (6, 2000, 5), (2, 4000, 3)])
def test_odd_and_prime_sizes(cuda_device, oracle, shape):
    import prj
    nx, nz, ny = shape
    rng = np.random.default_rng(nx * 1000 + nz * 10 + ny)
    A = np.asfortranarray(5 * (rng.random(shape) - 0.5))
    yu = np.concatenate([[0.0], np.cumsum(rng.uniform(0.1, 0.2, ny))]) + rng.uniform(-0.2, 0.2)
    dx, dz = rng.uniform(0.1, 0.2, 2)
    for mode in ("reference", "consistent"):
        b = prj.bands(yu, mode)
        with prj.Plan(nx, nz, ny, dx, dz, b) as plan:
            P = solve_dev(plan, A)
        Po, _ = oracle.poisson(A, dx, dz, b)
        assert rel_l2(P, Po) <= TOL_REL, (shape, mode)
        assert mean_removed_maxabs(P, Po) <= TOL_MAXABS


def test_solve_is_linear_and_repeatable(cuda_device):
    import prj
    import torch
    import workloads
    nx, ny, nz = 96, 48, 64
    r1, yu, dx, dz = workloads.poisson_rhs(nx, ny, nz, seed=11)
    r2, _, _, _ = workloads.poisson_rhs(nx, ny, nz, seed=12)
    with prj.Plan.from_yu(nx, nz, dx, dz, yu) as plan:
        p1 = solve_dev(plan, r1)
        p1b = solve_dev(plan, r1)
        p2 = solve_dev(plan, r2)
        p12 = solve_dev(plan, np.asfortranarray(2.5 * r1 + r2))
    np.testing.assert_array_equal(p1, p1b)  # deterministic
    assert rel_l2(p12, 2.5 * p1 + p2) <= 1e-13


def test_residual_at_large_size(cuda_device):
    """768 x 384 x 384 (the projection benchmark grid): the solution satisfies the
    discrete pinned operator of the reference bands to round-off."""
    import prj
    import torch
    import workloads
    nx, ny, nz = 768, 384, 384
    rhs, yu, dx, dz = workloads.poisson_rhs(nx, ny, nz, seed=3)
    a, b, c, a0, b0, c0 = prj.bands(yu)
    with prj.Plan(nx, nz, ny, dx, dz, (a, b, c, a0, b0, c0)) as plan:
        t = to_dev(rhs)
        plan.poisson_fp64(t)
        p = t  # [y, z, x]
        dev = p.device
        A = torch.tensor(a, device=dev).view(-1, 1, 1)
        B = torch.tensor(b, device=dev).view(-1, 1, 1)
        C = torch.tensor(c, device=dev).view(-1, 1, 1)
        Lp = B * p
        Lp[1:] += A[1:] * p[:-1]
        Lp[:-1] += C[:-1] * p[1:]
        Lp += (torch.roll(p, 1, 2) - 2 * p + torch.roll(p, -1, 2)) / dx ** 2
        Lp += (torch.roll(p, 1, 1) - 2 * p + torch.roll(p, -1, 1)) / dz ** 2
        # pinned (0,0) mode: bottom row of the mean mode uses b00 instead of b
        Lp[0] += (b0[0] - b[0]) * p[0].mean()
        r = to_dev(rhs)
        res = float(torch.linalg.vector_norm(Lp - r) / torch.linalg.vector_norm(r))
    # round-off of the stencil itself is ~ eps * (4/dx^2) |p| / |b|
    assert res < 1e-10, res


@pytest.mark.parametrize("shape", [(64, 48, 32), (96, 130, 40), (128, 384, 64)])
def test_streamed_thomas_is_bitwise_register_thomas(cuda_device, monkeypatch, shape):
    """The cp.async-streamed Thomas kernel keeps the operation order of the register-prefetch
    kernel: FP64 solves and FP32-storage solves agree bit for bit (ny not a multiple of the
    4-plane blocks included)."""
    import prj
    import workloads
    nx, ny, nz = shape
    rhs, yu, dx, dz = workloads.poisson_rhs(nx, ny, nz, seed=12)
    out = {}
    for flag in ("0", "1"):
        with prj.Plan(nx, nz, ny, dx, dz, prj.bands(yu, "consistent")) as plan:
            plan.set_tuning(thomas_ring=int(flag))
            t = to_dev(rhs)
            plan.poisson_fp64(t)
            t2 = to_dev(rhs)
            plan.poisson_mixed(t2)
            out[flag] = (from_dev(t), from_dev(t2))
    for a, b in zip(out["0"], out["1"]):
        np.testing.assert_array_equal(a, b)

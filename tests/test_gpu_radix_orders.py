"""The compiled radix orders of the pass plans (tuning x_order / z_order).

Each order rounds differently, so a solve in another order is compared with the oracle
(FP64 tolerance 1e-12 relative L2), and within one order the kernel families must agree
bit for bit: the per-wavenumber z kernel against the split z kernels, and the persistent
batch kernel against the per-case solve.  Out-of-range orders are refused.
"""
import numpy as np
import pytest

from conftest import rel_l2
from gpu_util import from_dev, to_dev

pytestmark = pytest.mark.gpu

# (nx, ny, nz) whose nx/2 or nz has other compiled orders
ORDERED = [(128, 21, 64), (192, 17, 96), (256, 13, 128), (384, 11, 192), (512, 9, 256), (96, 15, 384)]


def _solve(plan, rhs, **tuning):
    import torch
    if tuning:
        plan.set_tuning(**tuning)
    t = to_dev(rhs)
    plan.poisson_fp64(t)
    torch.cuda.synchronize()
    return from_dev(t)


@pytest.mark.parametrize("shape", ORDERED)
def test_orders_match_oracle_and_kernel_families_agree(cuda_device, oracle, shape):
    import prj
    import workloads
    nx, ny, nz = shape
    rhs, yu, dx, dz = workloads.poisson_rhs(nx, ny, nz, seed=41)
    b6 = prj.bands(yu, "reference")
    Po, _ = oracle.poisson(rhs, dx, dz, b6)
    nxo, nzo = prj_orders(nx // 2), prj_orders(nz)
    assert nxo > 1 or nzo > 1
    with prj.Plan(nx, nz, ny, dx, dz, b6) as plan:
        t0 = plan.tuning
        for xo in range(nxo):
            for zo in range(nzo):
                split = _solve(plan, rhs, x_order=xo, z_order=zo, z_mode=0)
                assert plan.tuning["x_order"] == xo and plan.tuning["z_order"] == zo
                assert rel_l2(split, Po) <= 1e-12, (xo, zo)
                line = _solve(plan, rhs, z_mode=3)
                np.testing.assert_array_equal(line, split)
        with pytest.raises(prj.PrjError) as e:
            plan.set_tuning(z_order=nzo)
        assert e.value.code == prj.PRJ_ERR_ARG
        plan.set_tuning(**t0)


def prj_orders(n):
    """Compiled radix orders of length n (1 for the default only)."""
    alts = {64: 2, 96: 2, 128: 2, 192: 2, 256: 3, 384: 3}
    return alts.get(n, 1)


def test_batch_with_other_orders(cuda_device):
    import prj
    import workloads
    shapes = [(128, 33, 64), (256, 20, 128), (192, 25, 256)]
    cases, plans = [], []
    for i, (nx, ny, nz) in enumerate(shapes):
        rhs, yu, dx, dz = workloads.poisson_rhs(nx, ny, nz, seed=50 + i)
        p = prj.Plan(nx, nz, ny, dx, dz, prj.bands(yu, "consistent"))
        p.set_tuning(x_order=prj_orders(nx // 2) - 1, z_order=prj_orders(nz) - 1)
        cases.append(rhs)
        plans.append(p)
    singles = [_solve(p, r) for p, r in zip(plans, cases)]
    tensors = [to_dev(r) for r in cases]
    with prj.Batch(plans, tensors) as batch:
        assert batch.info["persistent"]
        batch.launch()
        batch.check_error()
        for t, want in zip(tensors, singles):
            np.testing.assert_array_equal(from_dev(t), want)
    for p in plans:
        p.close()

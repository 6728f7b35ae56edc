"""The cluster z kernel (PRJ_ZSOLVE=cluster, z_mode 4: z FFT, Thomas and inverse z FFT of
one x wavenumber on a thread-block cluster of R_0 CTAs that exchange first-pass outputs and
last-pass inputs through distributed shared memory) against the split kernels.

It runs the same pass-plan butterflies on the same elements, the same twiddle tables and
the same Thomas operation order as the split kernels, so the FP64 solve must agree bit for
bit: for every z length with a pass plan (cluster sizes 2 to 8, one to four lines per
thread), ny not a multiple of the planes per chunk, every chunk/stage shape, the pinned
(0,0) mode, and through the whole projection step against the oracle.
"""
import numpy as np
import pytest

from conftest import rel_l2
from gpu_util import from_dev, to_dev

pytestmark = pytest.mark.gpu


def _solve(monkeypatch, env, nx, ny, nz, seed, **tuning):
    import prj
    import workloads
    monkeypatch.delenv("PRJ_ZSOLVE", raising=False)
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    rhs, yu, dx, dz = workloads.poisson_rhs(nx, ny, nz, seed=seed)
    with prj.Plan(nx, nz, ny, dx, dz, prj.bands(yu, "consistent")) as plan:
        if env.get("PRJ_ZSOLVE") == "cluster":
            assert plan.tuning["z_mode"] == 4
        if tuning:
            plan.set_tuning(**tuning)
        t = to_dev(rhs)
        plan.poisson_fp64(t)
        plan.check_error()
        return from_dev(t)


@pytest.mark.parametrize("nz", [16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768, 1024, 1536])
def test_cluster_kernel_is_bitwise_split_every_plan(cuda_device, monkeypatch, nz):
    nx, ny = (32, 23) if nz <= 512 else (16, 11)
    split = _solve(monkeypatch, {"PRJ_ZSOLVE": "split"}, nx, ny, nz, seed=31)
    clus = _solve(monkeypatch, {"PRJ_ZSOLVE": "cluster"}, nx, ny, nz, seed=31)
    np.testing.assert_array_equal(split, clus)


@pytest.mark.parametrize("yb,ns", [(4, 3), (2, 3), (1, 2), (3, 2), (8, 2), (5, 4)])
def test_cluster_kernel_chunk_shapes(cuda_device, monkeypatch, yb, ns):
    nx, ny, nz = 64, 61, 384
    split = _solve(monkeypatch, {"PRJ_ZSOLVE": "split"}, nx, ny, nz, seed=32)
    clus = _solve(monkeypatch, {"PRJ_ZSOLVE": "cluster"}, nx, ny, nz, seed=32, z_planes=yb, z_stages=ns)
    np.testing.assert_array_equal(split, clus)


def test_cluster_kernel_projection_step_matches_oracle(cuda_device, monkeypatch, oracle):
    """The FP64 projection step through the cluster kernel equals the split schedule bit for
    bit and the oracle within 1e-12 (reference bands: the parity mode)."""
    import prj
    import workloads
    from test_gpu_projection import run_engine
    nx, ny, nz = 96, 64, 96
    Uh, Vh, Wh, yu, dx, dz = workloads.projection_inputs(nx, ny, nz, seed=9)
    wall = (0.01, 0.0, -0.02, 0.03, 0.0, 0.04)
    out = {}
    for mode in ("split", "cluster"):
        monkeypatch.setenv("PRJ_ZSOLVE", mode)
        with prj.Plan.from_yu(nx, nz, dx, dz, yu, "reference") as plan:
            out[mode] = run_engine(plan, Uh, Vh, Wh, 0.7, wall)
    for a, b in zip(out["split"][:4], out["cluster"][:4]):
        np.testing.assert_array_equal(a, b)
    Uo, Vo, Wo, Po = oracle.projection(Uh, Vh, Wh, dx, dz, 0.7, yu, "reference", wall)
    U, V, W, P = out["cluster"][:4]
    assert rel_l2(P, Po) <= 1e-12
    for a, b in ((U, Uo), (V, Vo), (W, Wo)):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_cluster_kernel_by_tuning(cuda_device, monkeypatch):
    """z_mode 4 through prj_plan_set_tuning on a plan made with another default gives the
    split result bit for bit, and back again."""
    import prj
    import workloads
    monkeypatch.delenv("PRJ_ZSOLVE", raising=False)
    nx, ny, nz = 48, 30, 192
    rhs, yu, dx, dz = workloads.poisson_rhs(nx, ny, nz, seed=5)
    out = {}
    with prj.Plan(nx, nz, ny, dx, dz, prj.bands(yu, "reference")) as plan:
        t = plan.tuning
        for zm in (0, 4, 3, 4):
            plan.set_tuning(t["x_rows"], t["z_rows"], zm)
            assert plan.tuning["z_mode"] == zm
            d = to_dev(rhs)
            plan.poisson_fp64(d)
            out[zm] = from_dev(d)
    np.testing.assert_array_equal(out[0], out[4])
    np.testing.assert_array_equal(out[0], out[3])

"""The per-wavenumber z kernel (z_mode 3: z FFT, Thomas and inverse z FFT of one
x wavenumber per CTA) against the split kernels.

It runs the same pass-plan butterflies, twiddle tables and Thomas operation order as the
split kernels, so the FP64 solve must agree bit for bit: for every z length with a pass
plan, ny not a multiple of the planes per stage, every ring shape, and a length without a
plan (which falls back to the split kernels).
"""
import numpy as np
import pytest

from gpu_util import from_dev, to_dev

pytestmark = pytest.mark.gpu


SPLIT, LINE = {"z_mode": 0}, {"z_mode": 3}


def _solve(monkeypatch, zsel, nx, ny, nz, seed, **tuning):
    """FP64 solve with the z kernels zsel (SPLIT or LINE; LINE falls back to the split
    kernels for a length without a pass plan); no bounded wait of the line kernel's
    tensor-map copies may have given up (the plan's error word stays clear)."""
    import prj
    import workloads
    rhs, yu, dx, dz = workloads.poisson_rhs(nx, ny, nz, seed=seed)
    with prj.Plan(nx, nz, ny, dx, dz, prj.bands(yu, "consistent")) as plan:
        plan.set_tuning(**zsel, **tuning)
        t = to_dev(rhs)
        plan.poisson_fp64(t)
        plan.check_error()
        return from_dev(t)


@pytest.mark.parametrize("shape", [(64, 48, 32), (128, 97, 384), (32, 5, 16), (24, 21, 96), (32, 9, 48),
                                   (40, 70, 768), (16, 33, 1536), (96, 130, 40)])
def test_line_kernel_is_bitwise_split(cuda_device, monkeypatch, shape):
    nx, ny, nz = shape
    split = _solve(monkeypatch, SPLIT, nx, ny, nz, seed=21)
    line = _solve(monkeypatch, LINE, nx, ny, nz, seed=21)
    np.testing.assert_array_equal(split, line)


@pytest.mark.parametrize("yb,ns", [(4, 2), (2, 3), (1, 4), (3, 2), (8, 3)])
def test_line_kernel_ring_shapes(cuda_device, monkeypatch, yb, ns):
    nx, ny, nz = 64, 61, 384
    split = _solve(monkeypatch, SPLIT, nx, ny, nz, seed=22)
    line = _solve(monkeypatch, LINE, nx, ny, nz, seed=22, z_planes=yb, z_stages=ns)
    np.testing.assert_array_equal(split, line)


def test_line_kernel_projection_step(cuda_device, monkeypatch):
    """The whole FP64 projection step (divergence, solve, correction) through the line kernel
    equals the split schedule bit for bit, and its max|div u| stays at round-off."""
    import prj
    import workloads
    from test_gpu_projection import run_engine
    nx, ny, nz = 96, 64, 48
    Uh, Vh, Wh, yu, dx, dz = workloads.projection_inputs(nx, ny, nz, seed=5)
    out = {}
    for mode, zsel in (("split", SPLIT), ("line", LINE)):
        with prj.Plan.from_yu(nx, nz, dx, dz, yu, "consistent") as plan:
            plan.set_tuning(**zsel)
            out[mode] = run_engine(plan, Uh, Vh, Wh, 0.5)
    for a, b in zip(out["split"][:4], out["line"][:4]):
        np.testing.assert_array_equal(a, b)
    assert out["line"][4]["div_maxabs"] < 1e-10


def test_default_rule_and_tuning(cuda_device, monkeypatch):
    """The per-wavenumber kernel is the default from nx/2+1 >= 2 x the SM count (the split
    kernels below); the tuning call selects either for any grid with the same results."""
    import torch
    import prj
    import workloads
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    nx_big = 2 * (2 * sms)  # nx/2+1 > 2 x SMs
    rhs, yu, dx, dz = workloads.poisson_rhs(nx_big, 8, 16, seed=3)
    with prj.Plan(nx_big, 16, 8, dx, dz, prj.bands(yu, "consistent")) as plan:
        assert plan.tuning["z_mode"] == 3
        # one z kernel per step: the driver accepted the tensor map of the row copies
        assert plan.launches_per_step(prj.MODE_FP64) == 4
    nx, ny, nz = 64, 20, 48
    rhs, yu, dx, dz = workloads.poisson_rhs(nx, ny, nz, seed=4)
    out = {}
    with prj.Plan(nx, nz, ny, dx, dz, prj.bands(yu, "consistent")) as plan:
        t = plan.tuning
        assert t["z_mode"] == 0
        for zm in (0, 3):
            plan.set_tuning(t["x_rows"], t["z_rows"], zm)
            d = to_dev(rhs)
            plan.poisson_fp64(d)
            out[zm] = from_dev(d)
    np.testing.assert_array_equal(out[0], out[3])


@pytest.mark.parametrize("scale", [2.0 ** -960, 2.0 ** -1010])
def test_line_kernel_outside_the_fast_division_window(cuda_device, monkeypatch, oracle, scale):
    """Right-hand sides so small that the forward sweeps' quotients leave the window of the
    reciprocal-and-correction division (|q| < 2^-900; subnormal inputs at 2^-1010): both
    kernels take IEEE division for those quotients and still agree bit for bit."""
    import prj
    import workloads
    nx, ny, nz = 64, 21, 384
    rhs, yu, dx, dz = workloads.poisson_rhs(nx, ny, nz, seed=23)
    rhs = np.asfortranarray(rhs * scale)
    b6 = prj.bands(yu, "consistent")
    out = {}
    for mode, zsel in (("split", SPLIT), ("line", LINE)):
        with prj.Plan(nx, nz, ny, dx, dz, b6) as plan:
            plan.set_tuning(**zsel)
            t = to_dev(rhs)
            plan.poisson_fp64(t)
            out[mode] = from_dev(t)
    np.testing.assert_array_equal(out["split"], out["line"])
    if scale == 2.0 ** -960:  # normal inputs: the oracle's plain division agrees closely
        Po, _ = oracle.poisson(rhs, dx, dz, b6)
        assert np.linalg.norm(out["line"] - Po) <= 1e-12 * np.linalg.norm(Po)

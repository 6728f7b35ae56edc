"""GPU tests of the batched form (many uneven solves in one launch: the persistent
work-queue kernel for FP64 cases of the pass-plan lengths up to 256, else one CUDA
graph) and of the launch-shape autotuner."""
import numpy as np
import pytest

from conftest import rel_l2
from gpu_util import from_dev, to_dev

pytestmark = pytest.mark.gpu

SHAPES = [(64, 48, 64), (96, 64, 128), (128, 96, 96), (256, 48, 64), (30, 17, 21), (192, 128, 256)]  # (nx, ny, nz)


def make_cases(seed=2):
    import prj
    import workloads
    rng = np.random.default_rng(seed)
    cases = []
    for nx, ny, nz in SHAPES:
        beta = rng.uniform(1.5, 2.5)
        rhs, yu, dx, dz = workloads.poisson_rhs(nx, ny, nz, beta=beta, seed=int(rng.integers(1 << 30)))
        cases.append((rhs, yu, dx, dz, prj.bands(yu, "consistent")))
    return cases


def test_batch_equals_single_solves(cuda_device):
    import prj
    import torch
    cases = make_cases()
    plans = [prj.Plan(r.shape[0], r.shape[1], r.shape[2], dx, dz, b) for r, _, dx, dz, b in cases]
    singles = []
    for p, (r, *_rest) in zip(plans, cases):
        t = to_dev(r)
        p.poisson_fp64(t)
        singles.append(t)
    tensors = [to_dev(r) for r, *_ in cases]
    with prj.Batch(plans, tensors) as batch:
        # creation ran every case once eagerly; reset the inputs and replay the graph twice
        for t, (r, *_rest) in zip(tensors, cases):
            t.copy_(to_dev(r))
        batch.launch()
        torch.cuda.synchronize()
        first = [from_dev(t) for t in tensors]
        for t, (r, *_rest) in zip(tensors, cases):
            t.copy_(to_dev(r))
        batch.launch()
        torch.cuda.synchronize()
    for a, b, c in zip(first, (from_dev(t) for t in tensors), singles):
        np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(a, from_dev(c))
    for p in plans:
        p.close()


PERSISTENT_SHAPES = [(64, 48, 64), (96, 64, 128), (128, 96, 96), (256, 48, 64), (192, 128, 256), (32, 5, 16),
                     (512, 21, 192), (48, 33, 24)]


def _cases(shapes, seed):
    import prj
    import workloads
    rng = np.random.default_rng(seed)
    out = []
    for nx, ny, nz in shapes:
        rhs, yu, dx, dz = workloads.poisson_rhs(nx, ny, nz, beta=rng.uniform(1.5, 2.5), seed=int(rng.integers(1 << 30)))
        out.append((rhs, yu, dx, dz, prj.bands(yu, "reference")))
    return out


def test_persistent_batch_equals_single_solves(cuda_device, oracle):
    """One kernel launch per batch; every case bitwise equal to its own solve, on two launches
    in a row (the work counters reset with each launch), and within 1e-12 of the oracle."""
    import prj
    import torch
    cases = _cases(PERSISTENT_SHAPES, 7)
    plans = [prj.Plan(r.shape[0], r.shape[1], r.shape[2], dx, dz, b) for r, _, dx, dz, b in cases]
    singles = []
    for p, (r, *_rest) in zip(plans, cases):
        t = to_dev(r)
        p.poisson_fp64(t)
        singles.append(from_dev(t))
    tensors = [to_dev(r) for r, *_ in cases]
    with prj.Batch(plans, tensors) as batch:
        info = batch.info
        assert info["persistent"] and info["kernels_per_launch"] == 1 and info["work_items"] > len(cases)
        for rep in range(2):
            for t, (r, *_rest) in zip(tensors, cases):
                t.copy_(to_dev(r))
            batch.launch()
            batch.check_error()
            for t, want in zip(tensors, singles):
                np.testing.assert_array_equal(from_dev(t), want)
    for (r, _, dx, dz, b), got in zip(cases, singles):
        Po, _ = oracle.poisson(r, dx, dz, b)
        assert rel_l2(got, Po) <= 1e-12
    for p in plans:
        p.close()
    torch.cuda.synchronize()


def test_forced_graph_form_equals_persistent(cuda_device):
    """mode | PRJ_BATCH_GRAPH keeps the CUDA-graph form for cases the persistent kernel could
    run; both forms give the same bits."""
    import prj
    cases = _cases(PERSISTENT_SHAPES[:5], 11)
    plans = [prj.Plan(r.shape[0], r.shape[1], r.shape[2], dx, dz, b) for r, _, dx, dz, b in cases]
    outs = {}
    for graph in (False, True):
        tensors = [to_dev(r) for r, *_ in cases]
        with prj.Batch(plans, tensors, graph=graph) as batch:
            assert batch.info["persistent"] == (not graph)
            for t, (r, *_rest) in zip(tensors, cases):
                t.copy_(to_dev(r))
            batch.launch()
            batch.check_error()
            outs[graph] = [from_dev(t) for t in tensors]
    for a, b in zip(outs[False], outs[True]):
        np.testing.assert_array_equal(a, b)
    for p in plans:
        p.close()


def test_graph_batch_for_other_lengths(cuda_device):
    """A case outside the persistent kernel's lengths (nx/2 = 15) keeps the graph form."""
    import prj
    cases = make_cases()
    plans = [prj.Plan(r.shape[0], r.shape[1], r.shape[2], dx, dz, b) for r, _, dx, dz, b in cases]
    tensors = [to_dev(r) for r, *_ in cases]
    with prj.Batch(plans, tensors) as batch:
        info = batch.info
        assert not info["persistent"] and info["kernels_per_launch"] >= len(cases)
    for p in plans:
        p.close()


def test_batch_mixed_matches_fp64(cuda_device):
    import prj
    import torch
    cases = [c for c in make_cases(5) if c[0].shape[0] != 30]  # mixed path needs radices 2,3,4,5,8
    plans = [prj.Plan(r.shape[0], r.shape[1], r.shape[2], dx, dz, b) for r, _, dx, dz, b in cases]
    ref = []
    for p, (r, *_rest) in zip(plans, cases):
        t = to_dev(r)
        p.poisson_fp64(t)
        ref.append(from_dev(t))
    tensors = [to_dev(r) for r, *_ in cases]
    with prj.Batch(plans, tensors, mode=prj.MODE_FP32_REFINE) as batch:
        for t, (r, *_rest) in zip(tensors, cases):
            t.copy_(to_dev(r))
        batch.launch()
        torch.cuda.synchronize()
    for t, want in zip(tensors, ref):
        assert rel_l2(from_dev(t), want) <= 1e-11
    for p in plans:
        p.close()


def test_batch_rejects_shared_plan(cuda_device):
    import prj
    r, yu, dx, dz, b = make_cases()[0]
    p = prj.Plan(r.shape[0], r.shape[1], r.shape[2], dx, dz, b)
    with pytest.raises(prj.PrjError) as e:
        prj.Batch([p, p], [to_dev(r), to_dev(r)])
    assert e.value.code == prj.PRJ_ERR_ARG
    p.close()


def test_autotune_keeps_results(cuda_device, tmp_path, monkeypatch):
    import autotune
    import prj
    import torch
    monkeypatch.setattr(autotune, "CACHE", str(tmp_path / "tune.json"))
    r, yu, dx, dz, b = make_cases()[2]
    with prj.Plan(r.shape[0], r.shape[1], r.shape[2], dx, dz, b) as plan:
        t0 = to_dev(r)
        plan.poisson_fp64(t0)
        best = autotune.tune(plan, reps=2)
        assert best["ms"] > 0 and not best["cached"]
        t = plan.tuning
        assert {k: t[k] for k in ("x_rows", "z_rows", "z_mode")} == {k: best[k] for k in ("x_rows", "z_rows", "z_mode")}
        t1 = to_dev(r)
        plan.poisson_fp64(t1)
        torch.cuda.synchronize()
        assert rel_l2(from_dev(t1), from_dev(t0)) <= 1e-12
        again = autotune.tune(plan, reps=2)
        assert again["cached"]
        with pytest.raises(prj.PrjError):
            plan.set_tuning(3, 0, 0)


def test_misaligned_array_keeps_graph_form(cuda_device):
    """An array that is not 16-byte aligned (the persistent kernel reads P in 16-byte pairs)
    makes the batch use the graph form, with the bits of the per-case solve of the same
    array."""
    import prj
    import torch
    cases = _cases(PERSISTENT_SHAPES[:2], 13)
    plans = [prj.Plan(r.shape[0], r.shape[1], r.shape[2], dx, dz, b) for r, _, dx, dz, b in cases]

    def misaligned(r):
        d = to_dev(r)
        store = torch.zeros(d.numel() + 1, dtype=torch.float64, device=d.device)
        t = store[1:].view(d.shape)  # 8 bytes past a 16-byte boundary
        t.copy_(d)
        assert t.data_ptr() % 16 == 8
        return t

    single0 = misaligned(cases[0][0])
    plans[0].poisson_fp64(single0)
    single1 = to_dev(cases[1][0])
    plans[1].poisson_fp64(single1)
    singles = [from_dev(single0), from_dev(single1)]
    tensors = [misaligned(cases[0][0]), to_dev(cases[1][0])]
    with prj.Batch(plans, tensors) as batch:
        assert not batch.info["persistent"]
        for t, (r, *_rest) in zip(tensors, cases):
            t.copy_(to_dev(r))
        batch.launch()
        torch.cuda.synchronize()
        for t, want in zip(tensors, singles):
            np.testing.assert_array_equal(from_dev(t), want)
    for p in plans:
        p.close()

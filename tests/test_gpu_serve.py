"""GPU tests of the served form: continuous batching of mixed-size projection
requests that carry their own data, with resident per-size plans and HBM-budget
admission.

Every request brings its predictor, either as host arrays copied in (results
copied back into its host arrays) or as a seed from which its predictor is
produced on the device (results read from the slot by the completion callback).
Each result served in the overlapping mix must equal the oracle on that
request's own field (FP64 tolerance 1e-12) and the same request solved alone,
bit for bit.
"""
import numpy as np
import pytest

from conftest import rel_l2
from gpu_util import from_dev

pytestmark = pytest.mark.gpu

SMALL = ((64, 48, 32), (96, 32, 64), (128, 96, 64), (48, 40, 96))


def _pinned(shape):
    import torch
    return torch.empty(tuple(reversed(shape)), dtype=torch.float64).pin_memory().numpy().T


def _solo(size, Uh, Vh, Wh, dt):
    """The same request alone: a fresh plan, the predictor tensors given, one step."""
    import torch
    import prj
    import workloads
    nx, ny, nz = size
    yu = workloads.tanh_faces(ny, 2.0)
    dx, dz = workloads.channel_spacing(nx, nz)
    out = [torch.full_like(Uh, float("nan")) for _ in range(3)]
    out.append(torch.full((ny, nz, nx), float("nan"), dtype=torch.float64, device=Uh.device))
    with prj.Plan.from_yu(nx, nz, dx, dz, yu, "consistent") as plan:
        plan.projection_step(Uh, Vh, Wh, *out, dt, stats=False)
        torch.cuda.synchronize()
    return [from_dev(t) for t in out]


def test_served_requests_with_their_own_data(cuda_device, oracle):
    import serve
    import torch
    import workloads
    arrivals = serve.poisson_arrivals(20000.0, 0.004, seed=7, sizes=SMALL, probs=(0.25,) * 4)
    assert len(arrivals) >= 40
    reqs = []
    for i, (t, size) in enumerate(arrivals):
        r = serve.Request(i, size, t, seed=500 + i)
        if i % 2 == 0:  # host data in, results back to host arrays
            nx, ny, nz = size
            Uh, Vh, Wh, yu, dx, dz = workloads.projection_inputs(nx, ny, nz, seed=700 + i)
            hs = (nx + 2, nz + 2, ny + 2)
            r.fields = tuple(_pinned(hs) for _ in range(3))
            for dst, src in zip(r.fields, (Uh, Vh, Wh)):
                dst[...] = src
            r.want = "host"
            r.out = tuple(_pinned(hs) for _ in range(3)) + (_pinned((nx, nz, ny)),)
        reqs.append(r)
    srv = serve.ProjectionServer(hbm_budget=8e9)
    kept = {}

    def on_complete(r):
        if r.want == "device" and r.rid % 3 == 1:
            kept[r.rid] = [from_dev(t) for t in r.slot.fields[3:]]

    done = srv.run(None, on_complete=on_complete, requests=reqs)
    assert len(done) == len(reqs)
    assert srv.max_inflight > 1  # requests overlapped on the device
    assert kept
    dt = srv.dt
    checked = 0
    for r in reqs:
        nx, ny, nz = r.size
        if r.want == "host":
            Uh, Vh, Wh = r.fields
            yu = workloads.tanh_faces(ny, 2.0)
            dx, dz = workloads.channel_spacing(nx, nz)
            want = oracle.projection(Uh, Vh, Wh, dx, dz, dt, yu, "consistent")
            U, V, W, P = r.out
            assert rel_l2(P, want[3]) <= 1e-12
            for a, b in zip((U, V, W), want[:3]):
                assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
            if r.rid % 4 == 0:
                dev = [torch.from_numpy(np.ascontiguousarray(a.T)).cuda() for a in (Uh, Vh, Wh)]
                for a, b in zip(_solo(r.size, *dev, dt), r.out):
                    np.testing.assert_array_equal(a, b)
            checked += 1
        elif r.rid in kept:
            hs = (ny + 2, nz + 2, nx + 2)
            dev = [torch.zeros(hs, dtype=torch.float64, device="cuda") for _ in range(3)]
            yu = workloads.tanh_faces(ny, 2.0)
            yp = torch.tensor((yu[:-1] + yu[1:]) / 2, dtype=torch.float64, device="cuda")
            serve.device_predictor(*dev, yp, r.seed)
            for a, b in zip(_solo(r.size, *dev, dt), kept[r.rid]):
                np.testing.assert_array_equal(a, b)
            checked += 1
    assert checked >= len(reqs) // 2
    srv.close()
    torch.cuda.synchronize()


def test_device_predictor_matches_host_workload_distribution(cuda_device):
    """The per-request device predictor has the channel case's profile and noise level."""
    import serve
    import torch
    import workloads
    nx, ny, nz = 64, 48, 32
    hs = (ny + 2, nz + 2, nx + 2)
    f = [torch.zeros(hs, dtype=torch.float64, device="cuda") for _ in range(3)]
    yu = workloads.tanh_faces(ny, 2.0)
    yp = (yu[:-1] + yu[1:]) / 2
    serve.device_predictor(*f, torch.tensor(yp, device="cuda"), 11)
    U = f[0][1:-1, 1:-1, 1:-1].cpu().numpy()
    prof = 1.5 * (1 - (yp - 1) ** 2)
    assert np.abs(U.mean(axis=(1, 2)) - prof).max() < 0.05
    assert abs(f[1][2:-1, 1:-1, 1:-1].std().item() - 0.1) < 0.01
    assert float(f[1][1].abs().max()) == 0.0
    g = [torch.zeros_like(t) for t in f]
    serve.device_predictor(*g, torch.tensor(yp, device="cuda"), 11)
    for a, b in zip(f, g):
        assert torch.equal(a, b)


def test_budget_limits_resident_memory(cuda_device):
    """A budget that holds about one large slot still serves every request, without exceeding it."""
    import serve
    sizes = ((128, 96, 64), (256, 128, 128))
    one = serve.ProjectionServer()._slot_bytes(sizes[1])
    budget = 1.6 * one
    arrivals = serve.poisson_arrivals(2000.0, 0.02, seed=9, sizes=sizes, probs=(0.5, 0.5))
    srv = serve.ProjectionServer(hbm_budget=budget)
    done = srv.run(arrivals, warm=False)
    assert len(done) == len(arrivals)
    assert srv.peak_used <= budget
    s = serve.summarize(done, 0.02)
    assert s["p99_ms"] >= s["p50_ms"] > 0
    srv.close()


def test_slot_streams_prefer_smaller_grids(cuda_device):
    """Each slot's stream gets a priority by its grid size's rank among the sizes the server
    knows: under the default policy the smaller grid's stream has the higher priority (a lower
    number), "large" reverses it, "none" is flat; an unknown policy is refused."""
    import torch
    import serve
    least, greatest = torch.cuda.Stream.priority_range()
    small, big = serve.SERVED_SIZES[0], serve.SERVED_SIZES[1]
    pr = {}
    for pol in ("small", "large", "none"):
        srv = serve.ProjectionServer(hbm_budget=8e9, priority=pol)
        try:
            pr[pol] = [srv._acquire(size, 0.0).stream.priority for size in (small, big)]
        finally:
            srv.close()
    assert pr["small"][0] < pr["small"][1] and pr["large"][0] > pr["large"][1]
    assert pr["none"] == [0, 0]
    assert all(greatest <= p <= least for v in pr.values() for p in v)
    with pytest.raises(ValueError):
        serve.ProjectionServer(priority="fifo")

"""GPU tests of the served form: continuous batching of mixed-size projection
requests with resident per-size plans and HBM-budget admission."""
import numpy as np
import pytest

from gpu_util import from_dev

pytestmark = pytest.mark.gpu

SMALL = ((64, 48, 32), (96, 32, 64), (128, 96, 64), (48, 40, 96))


def test_served_results_equal_solo(cuda_device):
    """Each result computed in the overlapping mix is bit-identical to the same request alone."""
    import serve
    import torch
    arrivals = serve.poisson_arrivals(20000.0, 0.004, seed=7, sizes=SMALL, probs=(0.25,) * 4)
    assert len(arrivals) >= 40
    srv = serve.ProjectionServer(hbm_budget=8e9)
    kept = {}

    def on_complete(r):
        if r.rid % 3 == 0:
            r.slot.stream.synchronize()
            kept[r.rid] = (r.slot, from_dev(r.slot.fields[6]), from_dev(r.slot.fields[3]))

    done = srv.run(arrivals, on_complete=on_complete)
    assert len(done) == len(arrivals)
    assert srv.max_inflight > 1  # requests overlapped on the device
    for rid, (slot, P, U) in kept.items():
        Uh, Vh, Wh, dU, dV, dW, dP = slot.fields
        dP.fill_(float("nan"))
        dU.fill_(float("nan"))
        slot.plan.projection_step(Uh, Vh, Wh, dU, dV, dW, dP, srv.dt, stats=False, stream=slot.stream)
        slot.stream.synchronize()
        np.testing.assert_array_equal(from_dev(dP), P)
        np.testing.assert_array_equal(from_dev(dU), U)
    srv.close()
    torch.cuda.synchronize()


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

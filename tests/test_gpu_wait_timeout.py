"""The bounded device waits give up and report instead of hanging: a wait on an mbarrier that
nothing arrives on (budget ~1 ms of SM clock) must come back as PRJ_ERR_TIMEOUT, and the context
must stay usable for the next solve."""
import numpy as np
import pytest

from conftest import rel_l2
from gpu_util import from_dev, to_dev

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout_and_context_survives(cuda_device, oracle):
    import prj
    import workloads
    rc = prj.load_library().prj_selftest_wait_timeout(0, 2_000_000)
    assert rc == prj.PRJ_ERR_TIMEOUT
    assert b"gave up" in prj.load_library().prj_last_error_string()
    rhs, yu, dx, dz = workloads.poisson_rhs(32, 24, 16, seed=2)
    b = prj.bands(yu)
    with prj.Plan(32, 16, 24, dx, dz, b) as plan:
        t = to_dev(rhs)
        plan.poisson_fp64(t)
        P = from_dev(t)
    Po, _ = oracle.poisson(rhs, dx, dz, b)
    assert rel_l2(P, Po) <= 1e-12

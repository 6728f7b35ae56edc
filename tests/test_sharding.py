"""CPU tests of the multi-rank host logic (replicas over torch.distributed): case partition,
max-over-ranks timing and the whole-job value, with two gloo ranks."""
import os

import pytest


def test_partition_cases_balances_and_covers():
    import sharding
    pts = [a * b * c for a, b, c in [(64, 48, 64), (256, 128, 256), (96, 64, 96), (192, 96, 128),
                                      (128, 48, 64), (256, 128, 192), (64, 64, 64), (128, 128, 128)]]
    parts = sharding.partition_cases(pts, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(pts)))
    loads = [sum(pts[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(pts)  # LPT bound
    assert parts == sharding.partition_cases(pts, 3)  # deterministic: every rank agrees
    assert sharding.partition_cases(pts, 1) == [list(range(len(pts)))]
    with pytest.raises(ValueError):
        sharding.partition_cases(pts, 0)


def test_job_throughput():
    import sharding
    assert sharding.job_throughput(1e9, 10, 4, 1000.0) == pytest.approx(40.0)


def _rank_main(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "dns-supercritical-ibm_b200"))
    import datetime
    import torch.distributed as dist
    import sharding
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms_local = [5.0, 7.5][rank]  # rank 1 is the slow one
        ms = sharding.max_over_ranks(ms_local, dist)
        value = sharding.job_throughput(768 * 384 * 384, 50, world, ms)
        parts = sharding.partition_cases([10, 9, 8, 7, 6, 5, 4], world)
        dist.barrier()
        q.put((rank, ms, value, parts[rank]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_max_and_value():
    import socket
    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got[0][1] == got[1][1] == 7.5
    assert got[0][2] == got[1][2] == pytest.approx(2 * 768 * 384 * 384 * 50 / 7.5e-3 / 1e9)
    assert sorted(got[0][3] + got[1][3]) == list(range(7)) and not set(got[0][3]) & set(got[1][3])

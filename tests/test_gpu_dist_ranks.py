"""The projection step over ranks with the real engine in separate processes.

Two (and three) processes each create a plan on the one GPU of this harness and run
``prj_dist.DistSolve.project`` on their own planes: divergence, forward transforms,
the all-to-all of the spectrum, Thomas on their own x wavenumbers, the all-to-all
back, inverse transforms, the neighbour P plane and the correction.  The exchanges
go through host memory over a gloo process group (``host_staged_exchange``), so no
kernel of one process waits on another's.  The assembled U, V, W, P must equal the
single-GPU step bit for bit and the oracle within 1e-12.
"""
import os
import socket
import sys

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(os.path.dirname(HERE), "dns-supercritical-ibm_b200")
SHAPE = (96, 30, 48)  # nx, ny, nz: uneven plane and wavenumber splits for 2 and 3 ranks
DT = 0.6
WALL = (0.01, 0.0, -0.02, 0.03, 0.0, 0.04)


def _inputs():
    sys.path.insert(0, PKG)
    import workloads
    nx, ny, nz = SHAPE
    Uh, Vh, Wh, yu, dx, dz = workloads.projection_inputs(nx, ny, nz, seed=13)
    for F in (Uh, Vh, Wh):
        workloads.fill_halos(F)
    return Uh, Vh, Wh, yu, dx, dz


def _rank_main(rank, world, port, q):
    sys.path.insert(0, PKG)
    import datetime
    import torch
    import torch.distributed as dist
    import prj
    import prj_dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        nx, ny, nz = SHAPE
        Uh, Vh, Wh, yu, dx, dz = _inputs()
        with prj.Plan.from_yu(nx, nz, dx, dz, yu, "consistent") as plan:
            rk = prj_dist.DistSolve((nx, nz, ny), rank, world, prj_dist.Engine(plan), torch.device("cuda", 0))
            # this rank's halo'd planes y0-1 .. y1 of the inputs ([y+2, z+2, x+2] memory)
            t = lambda A: torch.from_numpy(np.ascontiguousarray(A.transpose(2, 1, 0)[rk.y0:rk.y1 + 2])).cuda()
            fields = (t(Uh), t(Vh), t(Wh))
            outs = tuple(torch.full_like(fields[0], float("nan")) for _ in range(3))
            P_ext = torch.zeros((rk.y1 - rk.y0 + 1, nz, nx), dtype=torch.float64, device="cuda")
            params = prj.StepParams(DT, *WALL, 0)
            rk.project(fields, outs, P_ext, params, prj_dist.host_staged_exchange(dist),
                       prj_dist.host_staged_plane_exchange(dist, rank, world))
            torch.cuda.synchronize()
            lo = 0 if rank == 0 else 1                      # the bottom wall plane on the first rank
            hi = rk.y1 - rk.y0 + (2 if rank == world - 1 else 1)  # the top wall plane on the last rank
            res = [o[lo:hi].cpu().numpy() for o in outs] + [P_ext[1:].cpu().numpy()]
        dist.barrier()
        q.put((rank, rk.y0, rk.y1, lo, res))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_processes_with_host_staged_exchange(cuda_device, oracle, world):
    import torch.multiprocessing as mp
    import prj
    from test_gpu_projection import run_engine
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in range(world)), key=lambda r: r[0])
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    nx, ny, nz = SHAPE
    got = [np.full((ny + 2, nz + 2, nx + 2), np.nan) for _ in range(3)] + [np.full((ny, nz, nx), np.nan)]
    for rank, y0, y1, lo, arrs in res:
        for G, a in zip(got[:3], arrs[:3]):
            G[y0 + lo:y0 + lo + a.shape[0]] = a
        got[3][y0:y1] = arrs[3]
    got = [g.transpose(2, 1, 0) for g in got]  # back to the reference's [x, z, y] order
    Uh, Vh, Wh, yu, dx, dz = _inputs()
    with prj.Plan.from_yu(nx, nz, dx, dz, yu, "consistent") as plan:
        ref = run_engine(plan, Uh, Vh, Wh, DT, WALL)
    for a, b in zip(got, ref[:4]):
        np.testing.assert_array_equal(a, b)
    Uo, Vo, Wo, Po = oracle.projection(Uh, Vh, Wh, dx, dz, DT, yu, "consistent", WALL)
    assert rel_l2(got[3], Po) <= 1e-12
    for a, b in zip(got[:3], (Uo, Vo, Wo)):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()

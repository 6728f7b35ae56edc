"""CPU tests of the host side of the one-solve-over-several-GPUs path (prj_dist.py): the
range splits, and the two all-to-all exchanges with real gloo ranks.  A stand-in engine
writes every spectrum value as a code of its (y, kx, z) position in the documented block
layout, checks that the line buffer it receives holds every plane of its own x wavenumbers
in order, marks the values, and checks that the marked values come back to the planes'
owners.  The GPU stages themselves are tested in tests/test_gpu_dist.py."""
import os

import pytest


def test_split_bounds():
    import prj_dist
    assert prj_dist.split_bounds(10, 3) == [0, 4, 7, 10]
    assert prj_dist.split_bounds(2, 3) == [0, 1, 2, 2]
    assert prj_dist.split_bounds(7, 1) == [0, 7]
    with pytest.raises(ValueError):
        prj_dist.split_bounds(5, 0)


def code(y, kx, z):
    return 1e6 * y + 1e3 * kx + z


class FakeEngine:
    """Stages on CPU tensors with the C-ABI's layouts (two doubles per complex value)."""

    def __init__(self, nh, nz, ny):
        import torch
        self.nh, self.nz, self.ny = nh, nz, ny
        self.spec = torch.zeros((ny, nh, nz, 2), dtype=torch.float64)
        self.errors = []

    def forward(self, P_local, y0, y1, stream=None):
        for y in range(y0, y1):
            for kx in range(self.nh):
                for z in range(self.nz):
                    self.spec[y, kx, z, 0] = code(y, kx, z)
                    self.spec[y, kx, z, 1] = -code(y, kx, z)

    def pack(self, y0, y1, kxb, send, stream=None):
        blocks = [self.spec[y0:y1, kxb[q]:kxb[q + 1]].reshape(-1) for q in range(len(kxb) - 1)]
        import torch
        flat = torch.cat(blocks)
        send[:flat.numel()] = flat

    def thomas(self, lines, kx0, kx1, stream=None):
        nk = kx1 - kx0
        v = lines[:self.ny * nk * self.nz * 2].view(self.ny, nk, self.nz, 2)
        for y in range(self.ny):
            for k in range(nk):
                for z in range(self.nz):
                    if v[y, k, z, 0] != code(y, kx0 + k, z) or v[y, k, z, 1] != -code(y, kx0 + k, z):
                        self.errors.append(("lines", y, kx0 + k, z))
        v[..., 0] += 0.5

    def unpack(self, y0, y1, kxb, recv, stream=None):
        off = 0
        for q in range(len(kxb) - 1):
            n = (y1 - y0) * (kxb[q + 1] - kxb[q]) * self.nz * 2
            self.spec[y0:y1, kxb[q]:kxb[q + 1]] = recv[off:off + n].view(y1 - y0, kxb[q + 1] - kxb[q], self.nz, 2)
            off += n

    def inverse(self, P_local, y0, y1, stream=None):
        for y in range(y0, y1):
            for kx in range(self.nh):
                for z in range(self.nz):
                    if self.spec[y, kx, z, 0] != code(y, kx, z) + 0.5:
                        self.errors.append(("back", y, kx, z))


def _rank_main(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "dns-supercritical-ibm_b200"))
    import datetime
    import torch
    import torch.distributed as dist
    import prj_dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        nx, nz, ny = 10, 3, 7  # nh = 6 x wavenumbers, uneven splits
        eng = FakeEngine(nx // 2 + 1, nz, ny)
        rk = prj_dist.DistSolve((nx, nz, ny), rank, world, eng, "cpu")

        def ex(out, inp, out_splits, in_splits):
            dist.all_to_all_single(out[:sum(out_splits)], inp[:sum(in_splits)], out_splits, in_splits)
        P_local = torch.zeros((rk.y1 - rk.y0, nz, nx), dtype=torch.float64)
        rk.solve(P_local, ex)
        dist.barrier()
        q.put((rank, (rk.y0, rk.y1, rk.kx0, rk.kx1), eng.errors[:5]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_exchange_spectrum_blocks(world):
    import socket
    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    ys = [r[1][:2] for r in res]
    kxs = [r[1][2:] for r in res]
    assert ys[0][0] == 0 and ys[-1][1] == 7 and all(ys[i][1] == ys[i + 1][0] for i in range(world - 1))
    assert kxs[0][0] == 0 and kxs[-1][1] == 6 and all(kxs[i][1] == kxs[i + 1][0] for i in range(world - 1))
    for r in res:
        assert r[2] == [], r


def _plane_main(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "dns-supercritical-ibm_b200"))
    import datetime
    import torch
    import torch.distributed as dist
    import prj_dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        b = prj_dist.split_bounds(7, world)
        y0, y1 = b[rank], b[rank + 1]
        P_ext = torch.full((y1 - y0 + 1, 3, 4), -1.0, dtype=torch.float64)
        for y in range(y0, y1):
            P_ext[y - y0 + 1] = float(y)
        prj_dist.nccl_plane_exchange(dist, rank, world)(P_ext)
        dist.barrier()
        q.put((rank, float(P_ext[0].min()), float(P_ext[0].max()), y0))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_neighbour_plane_exchange(world):
    """The P plane below each rank's first plane arrives from the rank below (rank 0 keeps
    its unused plane)."""
    import socket
    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_plane_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    for rank, lo, hi, y0 in sorted(q.get(timeout=10) for _ in range(world)):
        if rank == 0:
            assert lo == hi == -1.0
        else:
            assert lo == hi == float(y0 - 1)

"""One FP64 Poisson solve spread over several GPUs (ranks).

The reference spreads a solve over MPI ranks and moves the spectrum between pencil
ownerships with diezDecomp transposes (src/poisson_solver_mgpu_dtdma/
poisson_solver_multigpu.f90:328-554).  Here rank r owns the y planes ``y_bounds[r] ..
y_bounds[r+1]`` of P for the x and z transforms and the x wavenumbers ``kx_bounds[r] ..
kx_bounds[r+1]`` for the Thomas lines, and one all-to-all each way moves the spectrum
between the two ownerships:

    forward x, z (own planes) -> pack by destination kx range -> all-to-all ->
    Thomas (own lines, all planes) -> all-to-all back -> unpack -> inverse z, x.

The stages are the engine's C-ABI calls ``prj_dist_*`` (the single-GPU kernels on plane
and line subsets), so the assembled P equals the one-GPU solve bit for bit.  The
exchange is a callable ``exchange(out, inp, out_splits, in_splits)`` with the meaning of
``torch.distributed.all_to_all_single``: ``nccl_exchange`` between GPUs, or the in-process
copy of ``solve_emulated``, which runs all ranks' stages on one device.
"""
from __future__ import annotations

import ctypes

import prj


def split_bounds(n: int, parts: int):
    """Bounds of ``parts`` contiguous ranges tiling [0, n), sizes differing by at most one."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    q, r = divmod(n, parts)
    b = [0]
    for p in range(parts):
        b.append(b[-1] + q + (1 if p < r else 0))
    return b


class Engine:
    """The stage calls of one rank on its plan (ctypes into libprj_b200.so)."""

    def __init__(self, plan):
        self.plan = plan
        self.L = prj.load_library()

    def _s(self, stream):
        return prj._stream_ptr(stream)

    def forward(self, P_local, y0, y1, stream=None):
        prj._check(self.L.prj_dist_forward(self.plan.handle, ctypes.c_void_p(P_local.data_ptr()), y0, y1,
                                           self._s(stream)))

    def pack(self, y0, y1, kx_bounds, send, stream=None):
        kb = (ctypes.c_int * len(kx_bounds))(*kx_bounds)
        prj._check(self.L.prj_dist_pack(self.plan.handle, y0, y1, kb, len(kx_bounds) - 1,
                                        ctypes.c_void_p(send.data_ptr()), self._s(stream)))

    def thomas(self, lines, kx0, kx1, stream=None):
        prj._check(self.L.prj_dist_thomas(self.plan.handle, ctypes.c_void_p(lines.data_ptr()), kx0, kx1,
                                          self._s(stream)))

    def unpack(self, y0, y1, kx_bounds, recv, stream=None):
        kb = (ctypes.c_int * len(kx_bounds))(*kx_bounds)
        prj._check(self.L.prj_dist_unpack(self.plan.handle, y0, y1, kb, len(kx_bounds) - 1,
                                          ctypes.c_void_p(recv.data_ptr()), self._s(stream)))

    def inverse(self, P_local, y0, y1, stream=None):
        prj._check(self.L.prj_dist_inverse(self.plan.handle, ctypes.c_void_p(P_local.data_ptr()), y0, y1,
                                           self._s(stream)))

    def divergence(self, Uh, Vh, Wh, y0, y1, params, stream=None):
        p = lambda t: ctypes.c_void_p(t.data_ptr())
        prj._check(self.L.prj_dist_divergence(self.plan.handle, p(Uh), p(Vh), p(Wh), y0, y1, ctypes.byref(params),
                                              self._s(stream)))

    def correct(self, P_ext, Uh, Vh, Wh, U, V, W, y0, y1, params, stream=None):
        p = lambda t: ctypes.c_void_p(t.data_ptr())
        prj._check(self.L.prj_dist_correct(self.plan.handle, p(P_ext), p(Uh), p(Vh), p(Wh), p(U), p(V), p(W), y0, y1,
                                           ctypes.byref(params), self._s(stream)))


class DistSolve:
    """Rank ``rank`` of ``world`` in a solve of the grid ``(nx, nz, ny)``.  Buffers are
    float64 tensors on ``device`` (two doubles per complex spectrum value)."""

    def __init__(self, grid, rank: int, world: int, engine, device):
        import torch
        nx, nz, ny = grid
        self.rank, self.world, self.engine = rank, world, engine
        self.nz, self.ny = nz, ny
        self.nh = nx // 2 + 1
        self.y_bounds = split_bounds(ny, world)
        self.kx_bounds = split_bounds(self.nh, world)
        self.y0, self.y1 = self.y_bounds[rank], self.y_bounds[rank + 1]
        self.kx0, self.kx1 = self.kx_bounds[rank], self.kx_bounds[rank + 1]
        rows, nkx = self.y1 - self.y0, self.kx1 - self.kx0
        z2 = 2 * nz
        # forward exchange: blocks [q][y - y0][kx - kxb[q]][z] out, lines [y][kx - kx0][z] in
        self.fwd_in = [rows * (self.kx_bounds[q + 1] - self.kx_bounds[q]) * z2 for q in range(world)]
        self.fwd_out = [(self.y_bounds[p + 1] - self.y_bounds[p]) * nkx * z2 for p in range(world)]
        self.send = torch.empty(max(1, sum(self.fwd_in)), dtype=torch.float64, device=device)
        self.lines = torch.empty(max(1, sum(self.fwd_out)), dtype=torch.float64, device=device)
        self.back = torch.empty(max(1, sum(self.fwd_in)), dtype=torch.float64, device=device)

    # the three phases between the exchanges
    def phase_forward(self, P_local, stream=None):
        self.engine.forward(P_local, self.y0, self.y1, stream)
        self.engine.pack(self.y0, self.y1, self.kx_bounds, self.send, stream)

    def phase_lines(self, stream=None):
        self.engine.thomas(self.lines, self.kx0, self.kx1, stream)

    def phase_inverse(self, P_local, stream=None):
        self.engine.unpack(self.y0, self.y1, self.kx_bounds, self.back, stream)
        self.engine.inverse(P_local, self.y0, self.y1, stream)

    def phase_divergence(self, fields, params, stream=None):
        Uh, Vh, Wh = fields
        self.engine.divergence(Uh, Vh, Wh, self.y0, self.y1, params, stream)
        self.engine.pack(self.y0, self.y1, self.kx_bounds, self.send, stream)

    def project(self, fields, outs, P_ext, params, exchange, plane_exchange, stream=None):
        """Projection step of this rank's planes.  ``fields`` = (Uh, Vh, Wh) and ``outs`` =
        (U, V, W): local halo'd arrays of halo'd planes y0 .. y1+1 ((y1-y0+2) x (nz+2) x
        (nx+2)), ghost planes of the inputs filled by the caller.  ``P_ext`` holds P planes
        y0-1 .. y1-1 ((y1-y0+1) x nz x nx); its own planes receive P.  ``plane_exchange(
        P_ext)`` must copy the last own plane of every rank into plane 0 of the next rank's
        ``P_ext`` (send/recv with the neighbours); ``exchange`` is the all-to-all."""
        P_own = P_ext[1:]
        self.phase_divergence(fields, params, stream)
        exchange(self.lines, self.send, self.fwd_out, self.fwd_in)
        self.phase_lines(stream)
        exchange(self.back, self.lines, self.fwd_in, self.fwd_out)
        self.phase_inverse(P_own, stream)
        plane_exchange(P_ext)
        self.engine.correct(P_ext, *fields, *outs, self.y0, self.y1, params, stream)

    def solve(self, P_local, exchange, stream=None):
        """In-place solve of this rank's planes ``P_local`` ((y1-y0) x nz x nx, x fastest).
        Every rank calls it; ``exchange`` is collective."""
        self.phase_forward(P_local, stream)
        exchange(self.lines, self.send, self.fwd_out, self.fwd_in)
        self.phase_lines(stream)
        exchange(self.back, self.lines, self.fwd_in, self.fwd_out)
        self.phase_inverse(P_local, stream)


def nccl_exchange(dist, stream=None):
    """all_to_all_single over the default process group (NCCL between GPUs), ordered after
    the work queued on ``stream`` (the current stream if None)."""
    import torch

    def ex(out, inp, out_splits, in_splits):
        s = stream or torch.cuda.current_stream()
        with torch.cuda.stream(s):
            dist.all_to_all_single(out[:sum(out_splits)], inp[:sum(in_splits)], out_splits, in_splits)
    return ex


def nccl_plane_exchange(dist, rank: int, world: int, stream=None):
    """The neighbour exchange of ``DistSolve.project``: rank r sends its last P plane to
    rank r+1 and receives plane y0-1 from rank r-1 (point-to-point over the process group).
    For CUDA tensors the sends, receives and the copy into ``P_ext[0]`` are ordered on
    ``stream`` (the current stream if None), the stream the inverse transform wrote P on
    and the correction reads it on."""
    import contextlib

    def ex(P_ext):
        ctx = contextlib.nullcontext()
        if P_ext.is_cuda:
            import torch
            ctx = torch.cuda.stream(stream or torch.cuda.current_stream(P_ext.device))
        with ctx:
            ops = []
            if rank + 1 < world:
                ops.append(dist.P2POp(dist.isend, P_ext[-1].contiguous(), rank + 1))
            recv = None
            if rank > 0:
                recv = P_ext[0].new_empty(P_ext[0].shape)
                ops.append(dist.P2POp(dist.irecv, recv, rank - 1))
            if ops:
                for w in dist.batch_isend_irecv(ops):
                    w.wait()
            if recv is not None:
                P_ext[0].copy_(recv)
    return ex


def host_staged_exchange(dist, stream=None):
    """The all-to-all of ``DistSolve`` through host memory: the device send buffer is copied
    to the host, exchanged with ``all_to_all_single`` over the process group (gloo between
    processes that may share a GPU, or hosts without a GPU interconnect), and the received
    blocks are copied back; the copies are ordered on ``stream`` (the current stream if
    None) and the collective waits for them on the host."""
    import torch

    def ex(out, inp, out_splits, in_splits):
        s = stream or torch.cuda.current_stream(out.device)
        with torch.cuda.stream(s):
            h_in = inp[:sum(in_splits)].to("cpu")  # synchronous: the collective needs the data
            h_out = torch.empty(sum(out_splits), dtype=out.dtype)
            dist.all_to_all_single(h_out, h_in, out_splits, in_splits)
            out[:sum(out_splits)].copy_(h_out)
    return ex


def host_staged_plane_exchange(dist, rank: int, world: int, stream=None):
    """``nccl_plane_exchange`` through host memory (see ``host_staged_exchange``)."""
    import torch

    def ex(P_ext):
        s = stream or torch.cuda.current_stream(P_ext.device)
        with torch.cuda.stream(s):
            h = P_ext[[0, -1]].to("cpu")
            prev = h[0].clone()
            ops = []
            if rank + 1 < world:
                ops.append(dist.P2POp(dist.isend, h[1].contiguous(), rank + 1))
            if rank > 0:
                ops.append(dist.P2POp(dist.irecv, prev, rank - 1))
            if ops:
                for w in dist.batch_isend_irecv(ops):
                    w.wait()
            if rank > 0:
                P_ext[0].copy_(prev)
    return ex


def project_emulated(plans, Uh, Vh, Wh, U, V, W, P, params, world: int):
    """The projection step of ``world`` ranks emulated on one device (one plan per rank,
    in-process exchanges).  Halo'd tensors are (ny+2, nz+2, nx+2) with filled halos, P is
    (ny, nz, nx); U, V, W and P are written."""
    import torch
    g = plans[0].grid
    ranks = [DistSolve((g.nx, g.nz, g.ny), r, world, Engine(plans[r]), P.device) for r in range(world)]
    fields = [tuple(F[rk.y0:rk.y1 + 2] for F in (Uh, Vh, Wh)) for rk in ranks]
    outs = [tuple(F[rk.y0:rk.y1 + 2] for F in (U, V, W)) for rk in ranks]
    pext = [torch.zeros((rk.y1 - rk.y0 + 1, g.nz, g.nx), dtype=torch.float64, device=P.device) for rk in ranks]
    for rk, f in zip(ranks, fields):
        rk.phase_divergence(f, params)
    _exchange_all(ranks, world, forward=True)
    for rk in ranks:
        rk.phase_lines()
    _exchange_all(ranks, world, forward=False)
    for rk, pe in zip(ranks, pext):
        rk.phase_inverse(pe[1:])
    for r in range(1, world):
        pext[r][0].copy_(pext[r - 1][-1])
    # the correction writes its own planes of the shared output tensors; the local halo'd
    # views of neighbouring ranks overlap only in ghost planes that neither writes
    for rk, pe, f, o in zip(ranks, pext, fields, outs):
        rk.engine.correct(pe, *f, *o, rk.y0, rk.y1, params)
    for rk, pe in zip(ranks, pext):
        P[rk.y0:rk.y1].copy_(pe[1:])
    return U, V, W, P


def _exchange_all(ranks, world, forward):
    """In-process all-to-all between emulated ranks (rank p's input chunk q goes to rank
    q's output chunk p)."""
    if forward:
        outs, inps = [rk.lines for rk in ranks], [rk.send for rk in ranks]
        out_splits, in_splits = [rk.fwd_out for rk in ranks], [rk.fwd_in for rk in ranks]
    else:
        outs, inps = [rk.back for rk in ranks], [rk.lines for rk in ranks]
        out_splits, in_splits = [rk.fwd_in for rk in ranks], [rk.fwd_out for rk in ranks]
    for p in range(world):
        for q in range(world):
            n = in_splits[p][q]
            assert n == out_splits[q][p]
            if n:
                i0 = sum(in_splits[p][:q])
                o0 = sum(out_splits[q][:p])
                outs[q][o0:o0 + n].copy_(inps[p][i0:i0 + n])


def solve_emulated(plans, P, world: int):
    """Run the ``world`` ranks of one solve on a single device, one plan per rank, with an
    in-process exchange (for tests: the data movement of the distributed solve without
    NCCL).  ``P`` is the whole (ny, nz, nx) tensor, solved in place; returns it."""
    g = plans[0].grid
    ranks = [DistSolve((g.nx, g.nz, g.ny), r, world, Engine(plans[r]), P.device) for r in range(world)]
    locs = [P[rk.y0:rk.y1] for rk in ranks]

    def exchange_all(outs, inps, out_splits, in_splits):
        # rank p's input chunk q goes to rank q's output chunk p
        in_off = [[sum(in_splits[p][:q]) for q in range(world)] for p in range(world)]
        out_off = [[sum(out_splits[q][:p]) for p in range(world)] for q in range(world)]
        for p in range(world):
            for q in range(world):
                n = in_splits[p][q]
                assert n == out_splits[q][p]
                if n:
                    outs[q][out_off[q][p]:out_off[q][p] + n].copy_(inps[p][in_off[p][q]:in_off[p][q] + n])

    for rk, Pl in zip(ranks, locs):
        rk.phase_forward(Pl)
    exchange_all([rk.lines for rk in ranks], [rk.send for rk in ranks],
                 [rk.fwd_out for rk in ranks], [rk.fwd_in for rk in ranks])
    for rk in ranks:
        rk.phase_lines()
    exchange_all([rk.back for rk in ranks], [rk.lines for rk in ranks],
                 [rk.fwd_in for rk in ranks], [rk.fwd_out for rk in ranks])
    for rk, Pl in zip(ranks, locs):
        rk.phase_inverse(Pl)
    return P

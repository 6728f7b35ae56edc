"""Served projection solves: a continuous-batching request loop on one GPU.

Requests (one projection step of a channel case of some size) arrive on an
open-loop schedule.  The server keeps, per grid size, a pool of resident
*slots*: a solver plan plus the device fields of one request (predictor u_hat,
outputs u, v, w, p) and a CUDA stream.  A queued request is admitted as soon as
a slot of its size is idle; if none exists, a new slot is created when it fits
the HBM budget, evicting idle slots of other sizes (least recently used) when
needed.  Admitted requests run asynchronously on their slot's stream, so
requests of different sizes overlap on the device; completion is detected with
CUDA events.  Latency is completion time minus arrival time (host clock).

Predictor fields are synthetic (a channel profile plus seeded noise), generated
once per slot; a request uses its slot's field, so a result can be replayed
alone and compared bit for bit (see tests/test_gpu_serve.py).
"""
from __future__ import annotations

import collections
import math
import time
from dataclasses import dataclass, field

import numpy as np

import prj
import workloads

# sizes (nx, ny, nz) and their probabilities of the served channel workload
SERVED_SIZES = ((128, 96, 64), (256, 128, 128), (384, 192, 192), (768, 384, 384))
SERVED_PROBS = (0.4, 0.3, 0.2, 0.1)


@dataclass
class Request:
    rid: int
    size: tuple
    arrival: float           # seconds since the start of the run
    start: float = -1.0
    done: float = -1.0
    slot: object = None


@dataclass
class Slot:
    size: tuple
    plan: object
    fields: tuple            # Uh, Vh, Wh, U, V, W, P (torch, device)
    stream: object
    event: object
    nbytes: int
    seed: int
    busy: bool = False
    last_used: float = 0.0
    current: Request = None


def poisson_arrivals(rate_hz: float, duration_s: float, seed: int = 3, sizes=SERVED_SIZES, probs=SERVED_PROBS):
    """Open-loop schedule: exponential inter-arrival times and i.i.d. sizes."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t >= duration_s:
            break
        out.append((t, sizes[int(rng.choice(len(sizes), p=probs))]))
    return out


class ProjectionServer:
    def __init__(self, device: int = 0, hbm_budget: float = 150e9, max_slots: int = 64, slots_per_size: int = 4,
                 mode: int = prj.MODE_FP64, band_mode: str = "consistent", dt: float = 1.0):
        import torch
        self.torch = torch
        self.device = device
        self.budget = float(hbm_budget)
        self.max_slots = max_slots
        self.slots_per_size = slots_per_size
        self.mode = mode
        self.band_mode = band_mode
        self.dt = dt
        self.slots: list[Slot] = []
        self.used = 0
        self.peak_used = 0
        self.max_inflight = 0
        self.seed = 100

    # ------------------------------------------------------------------ slots
    def _slot_bytes(self, size):
        nx, ny, nz = size
        nh = (nx + 2) * (nz + 2) * (ny + 2)
        fields = 8 * (6 * nh + nx * ny * nz)
        plan = 16 * (nx // 2 + 1) * nz * ny + 8 * (nx // 2 + 1) * (nz // 2 + 2) * ny
        return fields + plan

    def _new_slot(self, size):
        torch = self.torch
        nx, ny, nz = size
        dev = torch.device("cuda", self.device)
        yu = workloads.tanh_faces(ny, 2.0)
        dx, dz = workloads.channel_spacing(nx, nz)
        plan = prj.Plan.from_yu(nx, nz, dx, dz, yu, self.band_mode, device=self.device)
        self.seed += 1
        g = torch.Generator(device=dev)
        g.manual_seed(self.seed)
        hs = (ny + 2, nz + 2, nx + 2)
        yp = torch.tensor((yu[:-1] + yu[1:]) / 2, dtype=torch.float64, device=dev)
        Uh = torch.zeros(hs, dtype=torch.float64, device=dev)
        Vh = torch.zeros_like(Uh)
        Wh = torch.zeros_like(Uh)
        inner = (slice(1, -1), slice(1, -1), slice(1, -1))
        Uh[inner] = 1.5 * (1 - (yp.view(-1, 1, 1) - 1) ** 2) + 0.1 * torch.randn((ny, nz, nx), generator=g,
                                                                                dtype=torch.float64, device=dev)
        Vh[inner] = 0.1 * torch.randn((ny, nz, nx), generator=g, dtype=torch.float64, device=dev)
        Wh[inner] = 0.1 * torch.randn((ny, nz, nx), generator=g, dtype=torch.float64, device=dev)
        Vh[1] = 0.0
        U, V, W = (torch.empty_like(Uh) for _ in range(3))
        P = torch.empty((ny, nz, nx), dtype=torch.float64, device=dev)
        s = torch.cuda.Stream(device=dev)
        torch.cuda.synchronize(dev)
        nbytes = plan.device_bytes + 8 * (6 * Uh.numel() + P.numel())
        slot = Slot(size, plan, (Uh, Vh, Wh, U, V, W, P), s, torch.cuda.Event(), nbytes, self.seed)
        self.slots.append(slot)
        self.used += nbytes
        self.peak_used = max(self.peak_used, self.used)
        return slot

    def _evict_for(self, need):
        """Free idle slots of least recent use until `need` more bytes fit."""
        idle = sorted((s for s in self.slots if not s.busy), key=lambda s: s.last_used)
        for s in idle:
            if self.used + need <= self.budget:
                break
            self.slots.remove(s)
            self.used -= s.nbytes
            s.plan.close()
            s.fields = None
        return self.used + need <= self.budget

    def _acquire(self, size, now):
        mine = 0
        for s in self.slots:
            if s.size == size:
                if not s.busy:
                    return s
                mine += 1
        if mine >= self.slots_per_size:
            return None
        if len(self.slots) >= self.max_slots and not self._evict_for(0):
            return None
        need = self._slot_bytes(size)
        if self.used + need > self.budget and not self._evict_for(need):
            return None
        if len(self.slots) >= self.max_slots:
            return None
        return self._new_slot(size)

    def launch(self, slot, req):
        Uh, Vh, Wh, U, V, W, P = slot.fields
        slot.plan.projection_step(Uh, Vh, Wh, U, V, W, P, self.dt, mode=self.mode, stats=False, stream=slot.stream)
        slot.event.record(slot.stream)

    # ------------------------------------------------------------------- loop
    def run(self, arrivals, on_complete=None, warm=True):
        """Serve `arrivals` [(t, size)], return the list of completed requests."""
        sizes = sorted({s for _, s in arrivals})
        if warm:  # the per-size slots that fit the budget, created before the clock starts
            for k in range(self.slots_per_size):
                for size in sizes:
                    if sum(sl.size == size for sl in self.slots) <= k:
                        if self._acquire(size, 0.0) is None:
                            break
                        self.slots[-1].busy = True  # keep _acquire from returning it again
            for sl in self.slots:
                sl.busy = False
        reqs = [Request(i, size, t) for i, (t, size) in enumerate(arrivals)]
        queues = {size: collections.deque() for size in sizes}
        queued = 0
        inflight = []
        done = []
        nxt = 0
        t0 = time.perf_counter()
        while nxt < len(reqs) or queued or inflight:
            now = time.perf_counter() - t0
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                queues[reqs[nxt].size].append(reqs[nxt])
                queued += 1
                nxt += 1
            still = []
            for r in inflight:
                if r.slot.event.query():
                    r.done = time.perf_counter() - t0
                    r.slot.busy = False
                    r.slot.last_used = r.done
                    if on_complete:
                        on_complete(r)
                    done.append(r)
                else:
                    still.append(r)
            inflight = still
            # admit the oldest waiting request of each size while that size has a free slot;
            # sizes go in order of their oldest request, and a size without a slot blocks no other
            blocked = False
            for q in sorted((q for q in queues.values() if q), key=lambda q: q[0].arrival):
                while q:
                    slot = self._acquire(q[0].size, now)
                    if slot is None:
                        blocked = True
                        break
                    r = q.popleft()
                    queued -= 1
                    slot.busy = True
                    slot.current = r
                    r.slot = slot
                    r.start = time.perf_counter() - t0
                    self.launch(slot, r)
                    inflight.append(r)
                    self.max_inflight = max(self.max_inflight, len(inflight))
            if blocked and not inflight:
                raise RuntimeError("requests cannot be admitted within the HBM budget")
            if nxt < len(reqs) and not inflight and not queued:
                time.sleep(max(0.0, min(1e-3, reqs[nxt].arrival - (time.perf_counter() - t0))))
        return done

    def close(self):
        for s in self.slots:
            s.plan.close()
        self.slots = []
        self.used = 0


def summarize(done, duration_s):
    lat = np.array([r.done - r.arrival for r in done]) * 1e3
    pts = sum(s[0] * s[1] * s[2] for s in (r.size for r in done))
    span = max(r.done for r in done) if done else 0.0
    return {
        "requests": len(done),
        "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
        "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
        "mean_ms": float(lat.mean()) if len(lat) else None,
        "solves_per_s": len(done) / span if span else None,
        "gpts_per_s": pts / span / 1e9 if span else None,
        "offered_window_s": duration_s,
        "drain_s": span - duration_s,
    }

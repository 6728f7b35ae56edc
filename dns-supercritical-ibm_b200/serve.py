"""Served projection solves: a continuous-batching request loop on one GPU.

Requests arrive on an open-loop schedule.  Each request is one projection step of
a channel case of some size and carries its own predictor field, in one of two
forms:

* ``seed``: the predictor u_hat is produced on the device from the request's
  seed in one pass (prj_synth_channel_predictor: a channel profile plus N(0, 0.1)
  noise that is a fixed function of the seed, v = 0 on the bottom wall face).  This
  is how a DNS time loop hands the projection its input: the momentum step leaves
  u_hat in device memory (src/main.f90:386-393 calls the projection on it);
* ``fields``: host arrays (Uh, Vh, Wh) in the reference's halo'd Fortran layout,
  copied to the device inside the request's timed work (pinned memory makes the
  copy asynchronous).

The result is handed back either as a device handle (``want="device"``: the
completion callback reads the slot's U, V, W, P while the slot is still held for
it) or copied into host arrays the request brings (``want="host"``: the
device-to-host copies are part of the request's work and latency).

The server keeps, per grid size, a pool of resident *slots*: a solver plan, the
device fields of one request and a CUDA stream (of higher priority for smaller grids,
so a short request's kernels do not queue behind a long one's).  A queued request is admitted as
soon as a slot of its size is idle; if none exists, a new slot is created when it
fits the HBM budget, evicting idle slots of other sizes (least recently used)
when needed.  Admitted requests run asynchronously on their slot's stream (input,
projection, output), so requests of different sizes overlap on the device.  One
waiter thread per slot blocks on the slot's completion event (a blocking-sync
event, so the thread sleeps) and stamps the completion time; the admission loop
sleeps on the completion queue between arrivals instead of polling.  Latency is
completion time minus arrival time (host clock).
"""
from __future__ import annotations

import collections
import queue
import threading
import time
from dataclasses import dataclass

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
    seed: int = 0            # predictor produced on the device from this seed (when fields is None)
    fields: tuple = None     # or host (Uh, Vh, Wh), halo'd Fortran-ordered [x+2, z+2, y+2]
    want: str = "device"     # "device": result handle; "host": U, V, W, P copied into `out`
    out: tuple = None        # host (U, V, W, P) for want == "host" (P Fortran-ordered [x, z, y])
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
    yp: object               # cell-centre coordinates (device) of the predictor profile
    busy: bool = False
    last_used: float = 0.0
    current: Request = None
    waiter: object = None
    jobs: object = None


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


def device_predictor(Uh, Vh, Wh, yp, seed, stream=None):
    """The channel predictor of one request in place on the device, a fixed function of
    `seed` (prj_synth_channel_predictor: U = 1.5 (1 - (y-1)^2) + N(0, 0.1), V, W = N(0, 0.1),
    V = 0 on the bottom wall face); halo'd [y+2, z+2, x+2] tensors, interior only (the
    projection reads no halo of its inputs)."""
    prj.synth_predictor(Uh, Vh, Wh, yp, seed, 0.1, stream=stream)


class ProjectionServer:
    def __init__(self, device: int = 0, hbm_budget: float = 150e9, max_slots: int = 64, slots_per_size: int = 4,
                 mode: int = prj.MODE_FP64, band_mode: str = "consistent", dt: float = 1.0, priority: str = "small"):
        import torch
        self.torch = torch
        self.device = device
        self.budget = float(hbm_budget)
        self.max_slots = max_slots
        self.slots_per_size = slots_per_size
        self.mode = mode
        self.band_mode = band_mode
        self.dt = dt
        # stream priority of a slot: "small" (smaller grids first, the default), "large" or
        # "none" (all equal); the GPU's block scheduler prefers the CTAs of higher-priority
        # streams when both have work ready.  Measured at 1000 requests/s of the served mix:
        # "small" p50 0.9 ms / p99 36 ms, "none" 5.3 / 92 ms (small requests' kernels queued
        # behind the 768^3 ones: 133 ms p99 at 128x96x64), "large" 5.3 / 131 ms
        if priority not in ("none", "large", "small"):
            raise ValueError(f"priority {priority!r}")
        self.priority = priority
        self.known_points = {sz[0] * sz[1] * sz[2] for sz in SERVED_SIZES}
        self.slots: list[Slot] = []
        self.used = 0
        self.peak_used = 0
        self.max_inflight = 0
        self._done_q = queue.Queue()
        self._t0 = time.perf_counter()

    # ------------------------------------------------------------------ slots
    def _slot_bytes(self, size):
        nx, ny, nz = size
        nh = (nx + 2) * (nz + 2) * (ny + 2)
        fields = 8 * (6 * nh + nx * ny * nz)
        plan = 16 * (nx // 2 + 1) * nz * ny + 8 * (nx // 2 + 1) * (nz // 2 + 2) * ny
        return fields + plan

    def _waiter_loop(self, slot):
        """Blocks on the slot's completion events in order; stamps and reports completions."""
        while True:
            job = slot.jobs.get()
            if job is None:
                return
            req, ev = job
            ev.synchronize()
            req.done = time.perf_counter() - self._t0
            self._done_q.put(req)

    def _new_slot(self, size):
        torch = self.torch
        nx, ny, nz = size
        dev = torch.device("cuda", self.device)
        yu = workloads.tanh_faces(ny, 2.0)
        dx, dz = workloads.channel_spacing(nx, nz)
        plan = prj.Plan.from_yu(nx, nz, dx, dz, yu, self.band_mode, device=self.device)
        hs = (ny + 2, nz + 2, nx + 2)
        Uh = torch.zeros(hs, dtype=torch.float64, device=dev)
        Vh, Wh = torch.zeros_like(Uh), torch.zeros_like(Uh)
        U, V, W = (torch.empty_like(Uh) for _ in range(3))
        P = torch.empty((ny, nz, nx), dtype=torch.float64, device=dev)
        yp = torch.tensor((yu[:-1] + yu[1:]) / 2, dtype=torch.float64, device=dev)
        s = torch.cuda.Stream(device=dev, priority=self._stream_priority(size))
        torch.cuda.synchronize(dev)
        nbytes = plan.device_bytes + 8 * (6 * Uh.numel() + P.numel())
        slot = Slot(size, plan, (Uh, Vh, Wh, U, V, W, P), s, None, nbytes, yp)
        slot.jobs = queue.Queue()
        slot.waiter = threading.Thread(target=self._waiter_loop, args=(slot,), daemon=True)
        slot.waiter.start()
        self.slots.append(slot)
        self.used += nbytes
        self.peak_used = max(self.peak_used, self.used)
        return slot

    def _stream_priority(self, size):
        if self.priority == "none":
            return 0
        least, greatest = self.torch.cuda.Stream.priority_range()  # e.g. (0, -5): lower is higher
        # rank among the sizes the server knows (the served mix, the run's requests, resident
        # slots): the most preferred gets the greatest priority
        pts = lambda sz: sz[0] * sz[1] * sz[2]
        known = self.known_points | {pts(s.size) for s in self.slots} | {pts(size)}
        order = sorted(known, reverse=(self.priority == "large"))
        return max(greatest, least - (len(order) - 1 - order.index(pts(size))))

    def _drop(self, s):
        s.jobs.put(None)
        s.waiter.join()
        s.plan.close()
        s.fields = None

    def _evict_for(self, need):
        """Free idle slots of least recent use until `need` more bytes fit."""
        idle = sorted((s for s in self.slots if not s.busy), key=lambda s: s.last_used)
        for s in idle:
            if self.used + need <= self.budget:
                break
            self.slots.remove(s)
            self.used -= s.nbytes
            self._drop(s)
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
        """The request's work on the slot's stream: its input, the projection step, its output."""
        torch = self.torch
        Uh, Vh, Wh, U, V, W, P = slot.fields
        if req.fields is not None:
            with torch.cuda.stream(slot.stream):
                for d, h in zip((Uh, Vh, Wh), req.fields):
                    d.copy_(torch.from_numpy(h.T), non_blocking=True)
        else:
            device_predictor(Uh, Vh, Wh, slot.yp, req.seed, stream=slot.stream)
        slot.plan.projection_step(Uh, Vh, Wh, U, V, W, P, self.dt, mode=self.mode, stats=False, stream=slot.stream)
        if req.want == "host":
            with torch.cuda.stream(slot.stream):
                for h, d in zip(req.out, (U, V, W, P)):
                    torch.from_numpy(h.T).copy_(d, non_blocking=True)
        ev = torch.cuda.Event(blocking=True)
        ev.record(slot.stream)
        slot.jobs.put((req, ev))

    # ------------------------------------------------------------------- loop
    def run(self, arrivals, on_complete=None, warm=True, requests=None):
        """Serve `arrivals` [(t, size)] (or ready Request objects in arrival order); return the
        completed requests.  Requests made from `arrivals` carry seed = 1000 + index."""
        if requests is None:
            requests = [Request(i, size, t, seed=1000 + i) for i, (t, size) in enumerate(arrivals)]
        sizes = sorted({r.size for r in requests})
        self.known_points |= {sz[0] * sz[1] * sz[2] for sz in sizes}
        if warm:  # the per-size slots that fit the budget, created before the clock starts
            for k in range(self.slots_per_size):
                for size in sizes:
                    if sum(sl.size == size for sl in self.slots) <= k:
                        if self._acquire(size, 0.0) is None:
                            break
                        self.slots[-1].busy = True  # keep _acquire from returning it again
            for sl in self.slots:
                sl.busy = False
        queues = {size: collections.deque() for size in sizes}
        queued = 0
        inflight = 0
        done = []
        nxt = 0
        self._t0 = t0 = time.perf_counter()

        def finish(r):
            nonlocal inflight
            inflight -= 1
            if on_complete:
                on_complete(r)  # the slot stays held while the callback reads its outputs
            r.slot.busy = False
            r.slot.last_used = r.done
            done.append(r)

        while nxt < len(requests) or queued or inflight:
            now = time.perf_counter() - t0
            while nxt < len(requests) and requests[nxt].arrival <= now:
                queues[requests[nxt].size].append(requests[nxt])
                queued += 1
                nxt += 1
            while True:
                try:
                    finish(self._done_q.get_nowait())
                except queue.Empty:
                    break
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
                    inflight += 1
                    self.max_inflight = max(self.max_inflight, inflight)
            if blocked and not inflight:
                raise RuntimeError("requests cannot be admitted within the HBM budget")
            # sleep until the next completion or the next arrival
            wait = 0.05
            if nxt < len(requests):
                wait = max(0.0, requests[nxt].arrival - (time.perf_counter() - t0))
            if inflight:
                try:
                    finish(self._done_q.get(timeout=wait if wait > 0 else 1e-4))
                except queue.Empty:
                    pass
            elif wait > 0 and not queued:
                time.sleep(wait)
        return done

    def close(self):
        for s in self.slots:
            self._drop(s)
        self.slots = []
        self.used = 0


def summarize(done, duration_s):
    lat = np.array([r.done - r.arrival for r in done]) * 1e3
    by_size = {}
    for size in sorted({r.size for r in done}):
        ls = np.array([r.done - r.arrival for r in done if r.size == size]) * 1e3
        by_size["x".join(map(str, size))] = {"requests": int(len(ls)), "p50_ms": float(np.percentile(ls, 50)),
                                             "p99_ms": float(np.percentile(ls, 99))}
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
        "by_size": by_size,
    }

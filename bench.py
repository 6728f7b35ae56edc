#!/usr/bin/env python
"""Benchmark of the B200 pressure projection (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
                    [--mode fp64|mixed] [--no-cpu-baseline]

Workload: one projection step of the channel case 768 x 384 x 384 (Lx = 2 pi,
Lz = pi, tanh faces with beta = 2, Poiseuille predictor plus N(0, 0.1) noise,
v = 0 at the walls), divergence-consistent bands so that max|div u| reaches
round-off.  Seeded synthetic inputs are generated on the device (no dataset
exists for this path).  The three input fields (0.92 GB each) are larger than
the 126 MB L2, so no flush is needed between steps.

value: Gpts/s = (points of all ranks x K) / (max over ranks of the device time
of K steps), CUDA events on the launching stream.  e2e: the same metric through
the host-buffer C-ABI (H2D of u_hat, projection, D2H of u, v, w, p inside the
timed region): prj_projection_step_host_async, steps pipelined over two staging
slots, with the synchronous drop-in prj_projection_step_host beside it.  The
pipelined time of K steps is the first copy-in, K-1 periods of one step's
copy-out overlapping the next step's copy-in (PCIe both ways at once), and the
last copy-out, so K (16 by default) amortises the fill and drain as a time loop
that calls the projection every step does.
Multi-GPU runs are independent replicas (one solve fits one GPU; the API for one
solve over several GPUs, prj_dist_*, is not timed here): weak scaling, no
collective on the data path.

roofline: the dominant kernel (algorithmic bytes per launch / its CUDA-event
duration against the measured HBM peak, and its DRAM traffic from the committed
ncu summary); roofline_kernels: the same for every step kernel; roofline_step:
the whole step at 88 B per point.

--impl reference times the CPU restatement of the reference's FFTW path
(oracle/, all host threads) on the same workload, per step a bounded sample
(768 x ny_s x 384, ny_s chosen so that the warm-up and timed steps together take about
--ref-budget-s seconds, 100 by default).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "dns-supercritical-ibm_b200")
sys.path.insert(0, PKG)

METRIC = "projection Gpts/s 768x384x384: FP32+refine vs FP64 @div<1e-10; served p99 ms"
NX, NY, NZ = 768, 384, 384
ALG_BYTES_PER_POINT = 88  # projection: 56 B/pt compulsory FP64 I/O + 32 B/pt spectrum round trips


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """Samples SM clock and clock-event reasons of one GPU through NVML while running."""

    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
               0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}

    def __init__(self, index: int, period_s: float = 0.01):
        self.index, self.period = index, period_s
        self.samples, self.reasons = [], 0
        self.max_mhz = None
        self._stop = threading.Event()
        self._thr = None
        self.ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.nv = None

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                self.reasons |= nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            except Exception:
                pass
            time.sleep(self.period)

    def __enter__(self):
        if self.ok:
            self._thr = threading.Thread(target=self._run, daemon=True)
            self._thr.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thr:
            self._thr.join()

    def summary(self):
        if not self.ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"], "samples": 0}
        names = [v for k, v in self.REASONS.items() if self.reasons & k]
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.max_mhz,
                "reasons": names, "samples": len(self.samples)}


# ----------------------------------------------------------------------------- workload
def device_inputs(nx, ny, nz, seed, device):
    """Channel predictor on the device: halo'd [y+2, z+2, x+2] tensors (interior filled)."""
    import torch
    import workloads
    yu = workloads.tanh_faces(ny, 2.0)
    yp = torch.tensor((yu[:-1] + yu[1:]) / 2, dtype=torch.float64, device=device)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    hs = (ny + 2, nz + 2, nx + 2)
    Uh = torch.zeros(hs, dtype=torch.float64, device=device)
    Vh = torch.zeros(hs, dtype=torch.float64, device=device)
    Wh = torch.zeros(hs, dtype=torch.float64, device=device)
    inner = (slice(1, -1), slice(1, -1), slice(1, -1))
    Uh[inner] = 1.5 * (1.0 - (yp.view(-1, 1, 1) - 1.0) ** 2) + 0.1 * torch.randn((ny, nz, nx), generator=g,
                                                                                 dtype=torch.float64, device=device)
    Vh[inner] = 0.1 * torch.randn((ny, nz, nx), generator=g, dtype=torch.float64, device=device)
    Wh[inner] = 0.1 * torch.randn((ny, nz, nx), generator=g, dtype=torch.float64, device=device)
    Vh[1] = 0.0  # bottom wall face V(k=0)
    return Uh, Vh, Wh, yu


def kernel_alg_bytes(nx, ny, nz):
    """Algorithmic bytes per launch of each kernel (what crosses its boundary)."""
    N = nx * ny * nz
    Nh = (nx + 2) * (nz + 2) * (ny + 2)
    S = (nx // 2 + 1) * nz * ny * 16  # one pass over the complex half-spectrum
    return {"k_fwd_x": 24 * N + S, "k_zsolve": 2 * S, "k_bwd_x": S + 8 * N, "k_correct": 32 * N + 24 * Nh,
            "k_zfft_fwd": 2 * S, "k_thomas": 2 * S, "k_zfft_inv": 2 * S, "k_stats": 32 * N}


def read_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", f"dram_traffic_projection_{NX}x{NY}x{NZ}.txt")
    try:
        for line in open(path):
            parts = line.split()
            if len(parts) >= 2 and parts[0] == kernel:
                return float(parts[1])
    except OSError:
        pass
    return None


# ----------------------------------------------------------------------------- reference arm
def run_reference(args, rank):
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import pyoracle
    import workloads
    C = pyoracle.COracle()
    cores = os.cpu_count() or 1
    # probe the per-point cost on a thin slab, then size the per-step sample
    probe_ny = 16
    Uh, Vh, Wh, yu, dx, dz = workloads.projection_inputs(NX, probe_ny, NZ, seed=1)
    t0 = time.perf_counter()
    C.projection(Uh, Vh, Wh, dx, dz, 1.0, yu, "consistent", nthreads=cores)
    per_pt = (time.perf_counter() - t0) / (NX * probe_ny * NZ)
    budget = args.ref_budget_s
    nsteps = args.steps + args.warmup
    ny_s = int(budget / max(nsteps, 1) / (per_pt * NX * NZ))
    ny_s = max(8, min(NY, ny_s - ny_s % 2))
    Uh, Vh, Wh, yu, dx, dz = workloads.projection_inputs(NX, ny_s, NZ, seed=1)
    for _ in range(args.warmup):
        C.projection(Uh, Vh, Wh, dx, dz, 1.0, yu, "consistent", nthreads=cores)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        C.projection(Uh, Vh, Wh, dx, dz, 1.0, yu, "consistent", nthreads=cores)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = NX * ny_s * NZ * args.steps / total / 1e9
    sample = f"{NX}x{ny_s}x{NZ} projection per step (nx, nz and the stretching of the full case; ny reduced to bound the run)"
    line = {"metric": METRIC, "value": value, "unit": "Gpts/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "pressure projection step 768x384x384 (channel, tanh beta=2)", "nx": NX, "ny": NY,
                       "nz": NZ, "bands": "consistent", "sample_ny": ny_s},
            "cpu_baseline": {"value": value, "unit": "Gpts/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "Gpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference FFTW/MPI build unavailable (no Fortran/MPI/FFTW on the box); the C restatement "
                    "of its FFTW path (oracle/prj_oracle.c, OpenMP) is timed instead"}
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- engine arm
def cpu_baseline_engine_workload(Uh_h, Vh_h, Wh_h, yu, dx, dz):
    """Time the oracle projection once on the bench workload (host copies of the inputs).
    Returns the baseline record and the oracle's (U, V, W, P), the parity check of the
    engine's step on the same input."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    C = pyoracle.COracle()
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    out = C.projection(Uh_h, Vh_h, Wh_h, dx, dz, 1.0, yu, "consistent", nthreads=cores)
    dt = time.perf_counter() - t0
    return {"value": NX * NY * NZ / dt / 1e9, "unit": "Gpts/s", "cores": cores, "kind": "port",
            "sample": f"one full {NX}x{NY}x{NZ} projection step ({dt:.2f} s)"}, out


def parity_vs_oracle(dev_out, oracle_out):
    """rel-L2 of P and max |u - u_oracle| / max |u_oracle| over U, V, W: the engine's device
    tensors ([y, z, x] memory) against the oracle's Fortran-ordered [x, z, y] arrays."""
    import numpy as np
    U, V, W, P = (t.cpu().numpy() for t in dev_out)
    Uo, Vo, Wo, Po = (a.T for a in oracle_out)
    p_rel = float(np.linalg.norm((P - Po).ravel()) / np.linalg.norm(Po.ravel()))
    u_rel = max(float(np.abs(a - b).max()) / float(np.abs(b).max()) for a, b in ((U, Uo), (V, Vo), (W, Wo)))
    return {"p_rel_l2_vs_oracle": p_rel, "u_maxabs_vs_oracle": u_rel}


def parity_reference_bands(Uh, Vh, Wh, Uh_h, Vh_h, Wh_h, yu, dx, dz, device, stream):
    """The same step with the reference's own bands (mk_P_abc), the parity mode, against the
    oracle with the same bands (outside every timed region)."""
    import torch
    import prj
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    out = [torch.empty_like(Uh) for _ in range(3)] + [torch.empty((NY, NZ, NX), dtype=torch.float64, device=device)]
    with prj.Plan.from_yu(NX, NZ, dx, dz, yu, "reference", device=device.index or 0) as plan:
        plan.projection_step(Uh, Vh, Wh, *out, 1.0, stats=False, stream=stream)
        torch.cuda.synchronize()
    ref = pyoracle.COracle().projection(Uh_h, Vh_h, Wh_h, dx, dz, 1.0, yu, "reference", nthreads=os.cpu_count() or 1)
    res = parity_vs_oracle(out, ref)
    del out, ref
    torch.cuda.empty_cache()
    return res


# ----------------------------------------------------------------------------- extra legs
def timed_steps(fn, stream, steps):
    """Sum of CUDA-event durations of `steps` calls of fn() on `stream`."""
    import torch
    total = 0.0
    for _ in range(steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    return total


def run_batched(device, steps, warmup, rank=0, world=1, dist=None, tune=True):
    """64 independent Poisson solves of uneven sizes in one launch: sizes from default_rng(2)
    (Nx, Nz in {64,96,128,192,256}, Ny in {48,64,96,128}, tanh beta ~ U[1.5,2.5]), uniform[-1,1]
    right-hand sides minus their dy-weighted mean; launch shapes from the autotuner.  FP64: the
    persistent work-queue kernel (one kernel per batch; its plans at the default tuning, since it
    sets its own tile shapes), and beside it the CUDA-graph form of the autotuned per-case
    kernels (fp64_graph); FP32-storage + FP64 refinement: one CUDA graph of the per-case
    kernels."""
    import numpy as np
    import torch
    import autotune
    import prj
    import workloads
    import sharding
    rng = np.random.default_rng(2)
    specs_all = []
    for _ in range(64):
        nx, nz = (int(v) for v in rng.choice([64, 96, 128, 192, 256], 2))
        ny = int(rng.choice([48, 64, 96, 128]))
        specs_all.append((nx, ny, nz, float(rng.uniform(1.5, 2.5))))
    # the 64 cases are split over the ranks by size (no data-path collective)
    mine = sharding.partition_cases([a * b * c for a, b, c, _ in specs_all], world)[rank]
    specs = [specs_all[i] for i in mine]
    seeds = [1000 + i for i in mine]
    plans, rhs, defaults = [], [], []
    t_tune = time.perf_counter()
    tuned = {}
    for i, (nx, ny, nz, beta) in enumerate(specs):
        yu = workloads.tanh_faces(ny, beta)
        dx, dz = workloads.channel_spacing(nx, nz)
        p = prj.Plan(nx, nz, ny, dx, dz, prj.bands(yu, "consistent"), device=device.index or 0)
        defaults.append(p.tuning)
        if not tune:
            tuned[(nx, ny, nz)] = {}
        elif (nx, ny, nz) in tuned:
            p.set_tuning(**tuned[(nx, ny, nz)])
        else:
            best = autotune.tune(p, reps=3)
            tuned[(nx, ny, nz)] = {k: best.get(k, 0) for k in autotune.FIELDS}
        plans.append(p)
        g = torch.Generator(device=device)
        g.manual_seed(seeds[i])
        r = torch.rand((ny, nz, nx), generator=g, dtype=torch.float64, device=device) * 2 - 1
        w = torch.tensor(np.diff(yu), dtype=torch.float64, device=device).view(-1, 1, 1)
        r -= (r * w).sum() / (w.sum() * nx * nz)
        rhs.append(r)
    t_tune = time.perf_counter() - t_tune
    pts = sum(nx * ny * nz for nx, ny, nz, _ in specs_all)
    out = {"cases": 64, "points": pts, "distinct_sizes": len(tuned), "setup_s": t_tune,
           "sharding": f"{world} rank(s), cases partitioned by size"}
    stream = torch.cuda.current_stream(device)
    tuned_t = [p.tuning for p in plans]
    for name, mode, graph in (("fp64", prj.MODE_FP64, False), ("fp64_graph", prj.MODE_FP64, True),
                              ("mixed", prj.MODE_FP32_REFINE, False)):
        # the persistent kernel sets its own tile shapes: its plans keep the default tuning
        # (radix orders included); the graph forms run the autotuned per-case kernels
        for p, t in zip(plans, defaults if name == "fp64" else tuned_t):
            p.set_tuning(**t)
        if mode == prj.MODE_FP32_REFINE:  # the mixed path runs the split z kernels
            for p in plans:
                t = p.tuning
                if t["z_mode"] != 0:
                    p.set_tuning(t["x_rows"], 0, 0)
        work = [r.clone() for r in rhs]
        with prj.Batch(plans, work, mode=mode, graph=graph) as batch:
            def reset():
                for w_, r_ in zip(work, rhs):
                    w_.copy_(r_)
            for _ in range(warmup):
                reset()
                batch.launch(stream)
            torch.cuda.synchronize()
            total = 0.0
            for _ in range(steps):
                reset()
                total += timed_steps(lambda: batch.launch(stream), stream, 1)
            if dist is not None:
                dist.barrier()
            total = sharding.max_over_ranks(total, dist, device)
            info = batch.info
            out[name] = {"gpts_per_s": pts * steps / (total / 1e3) / 1e9, "ms_per_batch": total / steps,
                         "launches": steps, "persistent_kernel": info["persistent"],
                         "kernels_per_launch": info["kernels_per_launch"], "work_items": info["work_items"]}
            if info["persistent"]:
                batch.check_error(stream)
    for p in plans:
        p.close()
    return out


def fluid_div_maxabs(U, V, W, solid, inv_dy_p, dx, dz, vbot=0.0, vtop=0.0):
    """max |div u| over the fluid cells of corrected halo'd [y+2, z+2, x+2] fields, in the
    engine's discrete divergence (periodic x and z halos, wall faces V(0) and V(ny))."""
    import torch
    ny = U.shape[0] - 2
    out = 0.0
    for j0 in range(0, ny, 64):  # plane blocks bound the temporaries
        j1 = min(ny, j0 + 64)
        sl = slice(j0 + 1, j1 + 1)
        d = (U[sl, 1:-1, 2:] - U[sl, 1:-1, 1:-1]) / dx
        d += (W[sl, 2:, 1:-1] - W[sl, 1:-1, 1:-1]) / dz
        v1 = V[j0 + 2:j1 + 2, 1:-1, 1:-1].clone()
        v0 = V[sl, 1:-1, 1:-1].clone()
        if j1 == ny:
            v1[-1] = vtop
        if j0 == 0:
            v0[0] = vbot
        d += (v1 - v0) * inv_dy_p[j0:j1].view(-1, 1, 1)
        d.masked_fill_(solid[j0:j1], 0.0)
        out = max(out, float(d.abs().max()))
    return out


def run_rough(device, nx, ny, nz, steps, warmup):
    """Rough-wall projection: wall-refined faces (uniform below y = 0.1, 1.5% growth per
    cell), the channel predictor zeroed inside a Gaussian k^-2 height field (peak 0.08,
    RMS 0.02, default_rng(5), both walls), FP64 and FP32 storage + FP64 refinement."""
    import numpy as np
    import torch
    import prj
    import workloads
    yu = workloads.wall_refined_faces(ny)
    h = workloads.rough_height_field(nx, nz, seed=5)
    yp = torch.tensor((yu[:-1] + yu[1:]) / 2, dtype=torch.float64, device=device).view(-1, 1, 1)
    ht = torch.tensor(h.T.copy(), dtype=torch.float64, device=device).unsqueeze(0)  # [1, z, x]
    solid = (yp < ht) | (yp > 2.0 - ht)                                              # [y, z, x]
    g = torch.Generator(device=device)
    g.manual_seed(6)
    hs = (ny + 2, nz + 2, nx + 2)
    fields = []
    for comp in range(3):
        f = torch.zeros(hs, dtype=torch.float64, device=device)
        inner = f[1:-1, 1:-1, 1:-1]
        inner.normal_(0.0, 0.1, generator=g)
        if comp == 0:
            inner += 1.5 * (1.0 - (yp - 1.0) ** 2)
        inner.masked_fill_(solid, 0.0)
        if comp == 1:
            f[1] = 0.0
        fields.append(f)
    Uh, Vh, Wh = fields
    U, V, W = (torch.empty_like(Uh) for _ in range(3))
    P = torch.empty((ny, nz, nx), dtype=torch.float64, device=device)
    dx, dz = 2 * math.pi / nx, math.pi / nz
    inv_dy_p = torch.tensor(prj.metrics(yu)[0], dtype=torch.float64, device=device)
    out = {"grid": f"{nx}x{ny}x{nz}", "solid_fraction": float(solid.float().mean()),
           "dy_wall": float(yu[1] - yu[0]), "dy_max": float(np.diff(yu).max())}
    stream = torch.cuda.current_stream(device)
    # immersed-boundary column forcing of the predictor ahead of the step (prj_rough_force,
    # ibm_part_2): per column the last bottom cell and the first top cell inside the roughness
    cnt_bot = (yp < ht).sum(dim=0).to(torch.int32)          # [z, x]
    cnt_top = (yp > 2.0 - ht).sum(dim=0).to(torch.int32)
    bot = (cnt_bot - 1).contiguous()
    top = (ny - cnt_top).contiguous()
    inds = {"U_bot": bot, "U_top": top, "V_bot": bot, "V_top": top, "W_bot": bot, "W_top": top}
    Uf, Vf, Wf = Uh.clone(), Vh.clone(), Wh.clone()
    force = lambda: prj.rough_force(Uf, Vf, Wf, inds, stream=stream)
    for _ in range(warmup):
        force()
    f_ms = timed_steps(force, stream, steps) / steps
    out["ibm_column_forcing"] = {"ms": f_ms, "cells_forced": int(3 * (cnt_bot.sum() + cnt_top.sum())),
                                 "call": "prj_rough_force on the three predictor components"}
    del Uf, Vf, Wf
    with prj.Plan.from_yu(nx, nz, dx, dz, yu, "consistent", device=device.index or 0) as plan:
        P64 = None
        for name, mode, graph in (("fp64", prj.MODE_FP64, False), ("fp64_graph", prj.MODE_FP64, True),
                              ("mixed", prj.MODE_FP32_REFINE, False)):
            fn = lambda: plan.projection_step(Uh, Vh, Wh, U, V, W, P, 1.0, mode=mode, stats=False, stream=stream)
            for _ in range(warmup):
                fn()
            ms = timed_steps(fn, stream, steps) / steps
            st = plan.projection_step(Uh, Vh, Wh, U, V, W, P, 1.0, mode=mode, stats=True, stream=stream)
            rec = {"gpts_per_s": nx * ny * nz / (ms / 1e3) / 1e9, "ms_per_step": ms,
                   "div_maxabs_all": st["div_maxabs"],
                   "div_maxabs_fluid": fluid_div_maxabs(U, V, W, solid, inv_dy_p, dx, dz)}
            if P64 is None:
                P64 = P.clone()
            else:
                rec["p_rel_l2_vs_fp64"] = float(torch.linalg.vector_norm(P - P64) / torch.linalg.vector_norm(P64))
                rec.update({k: st[k] for k in ("refine_iters", "fp64_lines", "last_update_rel")})
            out[name] = rec
        del P64
    return out


def run_vd(device, nx, ny, nz, steps, warmup):
    """Variable-density step (rho_min splitting) on the channel case: the predictor of the
    main workload, rho(y) = 1 - 0.6 (1 - (y-1)^2) times 1 + N(0, 0.05), P_now, P_old and
    div_now ~ N(0, 0.01), halos filled periodically / by wall ghost copies; FP64."""
    import torch
    import prj
    Uh, Vh, Wh, yu = device_inputs(nx, ny, nz, seed=11, device=device)
    yp = torch.tensor((yu[:-1] + yu[1:]) / 2, dtype=torch.float64, device=device).view(-1, 1, 1)
    g = torch.Generator(device=device)
    g.manual_seed(12)
    hs = (ny + 2, nz + 2, nx + 2)

    def halo(f):  # periodic x/z images, wall ghost planes copied from the first/last plane
        f[:, :, 0] = f[:, :, -2]
        f[:, :, -1] = f[:, :, 1]
        f[:, 0, :] = f[:, -2, :]
        f[:, -1, :] = f[:, 1, :]
        f[0] = f[1]
        f[-1] = f[-2]
        return f

    rho = torch.zeros(hs, dtype=torch.float64, device=device)
    rho[1:-1, 1:-1, 1:-1].normal_(1.0, 0.05, generator=g).mul_(1.0 - 0.6 * (1.0 - (yp - 1.0) ** 2))
    extra = []
    for _ in range(3):
        f = torch.zeros(hs, dtype=torch.float64, device=device)
        f[1:-1, 1:-1, 1:-1].normal_(0.0, 0.01, generator=g)
        extra.append(halo(f))
    halo(rho)
    Pn, Po, div = extra
    U, V, W, Pnext = (torch.empty(hs, dtype=torch.float64, device=device) for _ in range(4))
    P = torch.empty((ny, nz, nx), dtype=torch.float64, device=device)
    dx, dz = 2 * math.pi / nx, math.pi / nz
    stream = torch.cuda.current_stream(device)
    with prj.Plan.from_yu(nx, nz, dx, dz, yu, "consistent", device=device.index or 0) as plan:
        fn = lambda: plan.projection_step_vd(Uh, Vh, Wh, rho, Pn, Po, div, U, V, W, P, Pnext, 1.0, stats=False,
                                             stream=stream)
        for _ in range(warmup):
            fn()
        plan.enable_stage_timing(True)
        ms = timed_steps(fn, stream, steps) / steps
        plan.enable_stage_timing(False)
        stages = plan.stage_times()
        st = plan.projection_step_vd(Uh, Vh, Wh, rho, Pn, Po, div, U, V, W, P, Pnext, 1.0, stream=stream)
    return {"grid": f"{nx}x{ny}x{nz}", "gpts_per_s": nx * ny * nz / (ms / 1e3) / 1e9, "ms_per_step": ms,
            "div_maxabs": st["div_maxabs"], "rho_min": st["rho_min"],
            "stages_ms_per_launch": {k: v[0] / v[1] for k, v in stages.items()}}


def run_served(device, seconds, rate, budget, io="device"):
    """Open-loop Poisson arrivals (rate per second, default_rng(3)) of projection requests of
    sizes (128,96,64)/(256,128,128)/(384,192,192)/(768,384,384) with p = 0.4/0.3/0.2/0.1.
    io "device": every request's predictor is produced on the device from its own seed and its
    U, V, W, P are left on the device for the caller (a result handle); io "host": every
    request's predictor is copied in from pinned host memory (a pool of one field set per
    size, the requests of a size taking turns) and its U, V, W, P are copied back to pinned
    host memory, both inside the request's latency."""
    import torch
    import serve
    import workloads
    arrivals = serve.poisson_arrivals(rate, seconds, seed=3)
    reqs = [serve.Request(i, size, t, seed=1000 + i) for i, (t, size) in enumerate(arrivals)]
    h2d = d2h = 0
    if io == "host":
        pin = lambda shape: torch.empty(tuple(reversed(shape)), dtype=torch.float64).pin_memory().numpy().T
        pool = {}
        for size in sorted({r.size for r in reqs}):
            nx, ny, nz = size
            Uh, Vh, Wh, *_ = workloads.projection_inputs(nx, ny, nz, seed=17)
            hs = (nx + 2, nz + 2, ny + 2)
            ins = tuple(pin(hs) for _ in range(3))
            for dst, src in zip(ins, (Uh, Vh, Wh)):
                dst[...] = src
            pool[size] = (ins, tuple(pin(hs) for _ in range(3)) + (pin((nx, nz, ny)),))
        for r in reqs:
            r.fields, r.out = pool[r.size]
            r.want = "host"
            nx, ny, nz = r.size
            h2d += 3 * 8 * (nx + 2) * (nz + 2) * (ny + 2)
            d2h += 3 * 8 * (nx + 2) * (nz + 2) * (ny + 2) + 8 * nx * ny * nz
    srv = serve.ProjectionServer(device=device.index or 0, hbm_budget=budget)
    t0 = time.perf_counter()
    done = srv.run(None, requests=reqs)
    wall = time.perf_counter() - t0
    out = serve.summarize(done, seconds)
    offered = sum(a * b * c for _, (a, b, c) in arrivals) / seconds / 1e9
    out.update({"rate_hz": rate, "offered_gpts_per_s": offered, "wall_s": wall,
                "max_inflight": srv.max_inflight, "peak_resident_gb": srv.peak_used / 1e9,
                "sustained": bool(out["drain_s"] is not None and out["drain_s"] < 0.05 * seconds),
                "io": ("predictor produced on the device per request from its seed; U, V, W, P left on the "
                       "device (result handle)") if io == "device" else
                      ("predictor copied in from pinned host memory and U, V, W, P copied back to pinned host "
                       "memory inside each request"),
                "h2d_bytes_per_request": h2d / max(1, len(reqs)), "d2h_bytes_per_request": d2h / max(1, len(reqs))})
    srv.close()
    return out


def main():
    global NX, NY, NZ
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--mode", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--e2e-steps", type=int, default=16, help="0 skips the end-to-end leg")
    ap.add_argument("--grid", default=f"{NX}x{NY}x{NZ}", help="nx x ny x nz (profiling of smaller cases)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the mixed, batched and served legs")
    ap.add_argument("--legs", default="mixed,batched,served,vd,rough",
                    help="comma list of the extra legs to run (mixed, batched, served, vd, rough)")
    ap.add_argument("--batch-tune", default="auto", choices=["auto", "default"],
                    help="batched leg: autotuned tunings, or the plans' defaults (profiling runs)")
    ap.add_argument("--served-seconds", type=float, default=30.0)
    ap.add_argument("--served-rate", type=float, default=2000.0)
    ap.add_argument("--served-budget-gb", type=float, default=150.0)
    ap.add_argument("--rough-grid", default="1536x512x768", help="rough-wall leg nx x ny x nz ('' skips it)")
    ap.add_argument("--ref-budget-s", type=float, default=100.0,
                    help="reference arm: host seconds for its warm-up and timed steps together")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    NX, NY, NZ = (int(v) for v in args.grid.lower().split("x"))

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)

    import numpy as np
    import torch
    import prj
    import sharding

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=device)

    def barrier():
        if dist is not None:
            dist.barrier()

    mode = prj.MODE_FP64 if args.mode == "fp64" else prj.MODE_FP32_REFINE
    Uh, Vh, Wh, yu = device_inputs(NX, NY, NZ, seed=1 + rank, device=device)
    dx, dz = 2 * math.pi / NX, math.pi / NZ
    hs = (NY + 2, NZ + 2, NX + 2)
    U = torch.empty(hs, dtype=torch.float64, device=device)
    V = torch.empty_like(U)
    W = torch.empty_like(U)
    P = torch.empty((NY, NZ, NX), dtype=torch.float64, device=device)
    plan = prj.Plan.from_yu(NX, NZ, dx, dz, yu, "consistent", device=local)
    stream = torch.cuda.current_stream(device)

    def step(stats=False):
        return plan.projection_step(Uh, Vh, Wh, U, V, W, P, 1.0, mode=mode, stats=stats, stream=stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches_per_step = plan.launches_per_step(mode)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ms_max = sharding.max_over_ranks(ms, dist, device)
    value = sharding.job_throughput(NX * NY * NZ, args.steps, world, ms_max)
    # per-kernel CUDA-event times: a separate run with stage timing (events around every
    # kernel, which the timed run above does without)
    plan.enable_stage_timing(True)
    for _ in range(max(3, args.steps // 5)):
        step()
    torch.cuda.synchronize()
    plan.enable_stage_timing(False)
    stages = plan.stage_times()

    # accuracy record of the same step (outside the timed region)
    st = step(stats=True)

    # e2e through the host-buffer C-ABI call
    Uh_h = np.asfortranarray(Uh.cpu().numpy().T)
    Vh_h = np.asfortranarray(Vh.cpu().numpy().T)
    Wh_h = np.asfortranarray(Wh.cpu().numpy().T)
    e2e = None
    if args.e2e_steps > 0:
        pin = lambda shape: torch.empty(tuple(reversed(shape)), dtype=torch.float64).pin_memory().numpy().T
        hshape = (NX + 2, NZ + 2, NY + 2)
        pUh, pVh, pWh, pU, pV, pW = (pin(hshape) for _ in range(6))
        pP = pin((NX, NZ, NY))
        pUh[...] = Uh_h
        pVh[...] = Vh_h
        pWh[...] = Wh_h
        plan.projection_step(pUh, pVh, pWh, pU, pV, pW, pP, 1.0, mode=mode, stats=False)  # warm (staging alloc)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            plan.projection_step(pUh, pVh, pWh, pU, pV, pW, pP, 1.0, mode=mode, stats=False)
        sync_s = sharding.max_over_ranks((time.perf_counter() - t0) / args.e2e_steps, dist, device)
        # pipelined host-buffer steps: one step's copy-out overlaps the next step's copy-in
        plan.projection_step_host_async(pUh, pVh, pWh, pU, pV, pW, pP, 1.0, mode=mode)  # warm (slot alloc)
        plan.host_async_wait()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            plan.projection_step_host_async(pUh, pVh, pWh, pU, pV, pW, pP, 1.0, mode=mode)
        plan.host_async_wait()
        e2e_s = sharding.max_over_ranks((time.perf_counter() - t0) / args.e2e_steps, dist, device)
        nh = (NX + 2) * (NZ + 2) * (NY + 2)
        e2e = {"value": world * NX * NY * NZ / e2e_s / 1e9, "unit": "Gpts/s", "h2d_bytes_per_step": 3 * 8 * nh,
               "d2h_bytes_per_step": 3 * 8 * nh + 8 * NX * NY * NZ, "ms_per_step": 1e3 * e2e_s,
               "call": f"prj_projection_step_host_async, {args.e2e_steps} steps pipelined (pinned host buffers)",
               "steps": args.e2e_steps,
               "sync_call": {"value": world * NX * NY * NZ / sync_s / 1e9, "ms_per_step": 1e3 * sync_s,
                             "call": "prj_projection_step_host"}}

    # roofline of the dominant kernel
    peak, peak_kind = peaks()
    alg = kernel_alg_bytes(NX, NY, NZ)
    dom = max(stages, key=lambda k: stages[k][0])
    dom_ms = stages[dom][0] / stages[dom][1]
    achieved = alg[dom] / (dom_ms / 1e3) / 1e9
    traffic = read_traffic(dom)
    # every step kernel: algorithmic bytes, achieved GB/s and fraction of the peak, and the DRAM
    # traffic of the committed ncu summary with the GB/s it implies at this duration
    per_kernel = {}
    for k, (tot_ms, cnt) in stages.items():
        if k not in alg or cnt == 0:
            continue
        k_ms = tot_ms / cnt
        tr = read_traffic(k)
        gbs = alg[k] / (k_ms / 1e3) / 1e9
        per_kernel[k] = {"alg_bytes": alg[k], "ms": k_ms, "achieved": gbs, "frac": gbs / peak, "traffic": tr,
                         "traffic_gbs": (tr / (k_ms / 1e3) / 1e9) if tr else None,
                         "traffic_frac": (tr / (k_ms / 1e3) / 1e9 / peak) if tr else None}
    step_ms = ms_max / args.steps
    roof_step = ALG_BYTES_PER_POINT * NX * NY * NZ / (step_ms / 1e3) / 1e9
    launches = launches_per_step * args.steps

    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, orc = cpu_baseline_engine_workload(Uh_h, Vh_h, Wh_h, yu, dx, dz)
        if mode == prj.MODE_FP64:  # U, V, W, P still hold the accuracy step's outputs
            parity = {"consistent_bands": parity_vs_oracle((U, V, W, P), orc)}
            parity["reference_bands"] = parity_reference_bands(Uh, Vh, Wh, Uh_h, Vh_h, Wh_h, yu, dx, dz, device,
                                                               stream)
        del orc

    legs = set() if args.no_extra else {v.strip() for v in args.legs.split(",") if v.strip()}
    extra = {}
    if "mixed" in legs:
        # FP32 spectral storage + FP64 refinement on the same step
        other = prj.MODE_FP32_REFINE if mode == prj.MODE_FP64 else prj.MODE_FP64
        P_main = P.clone()
        for _ in range(args.warmup):
            plan.projection_step(Uh, Vh, Wh, U, V, W, P, 1.0, mode=other, stats=False, stream=stream)
        ms_other = timed_steps(lambda: plan.projection_step(Uh, Vh, Wh, U, V, W, P, 1.0, mode=other, stats=False,
                                                            stream=stream), stream, max(3, args.steps // 4))
        ms_other = sharding.max_over_ranks(ms_other, dist, device)
        st_o = plan.projection_step(Uh, Vh, Wh, U, V, W, P, 1.0, mode=other, stats=True, stream=stream)
        rel = float(torch.linalg.vector_norm(P - P_main) / torch.linalg.vector_norm(P_main))
        nsteps_o = max(3, args.steps // 4)
        extra["other_precision"] = {
            "mode": "mixed" if other == prj.MODE_FP32_REFINE else "fp64",
            "gpts_per_s": world * NX * NY * NZ * nsteps_o / (ms_other / 1e3) / 1e9, "ms_per_step": ms_other / nsteps_o,
            "p_rel_l2_vs_this_mode": rel, "div_maxabs": st_o["div_maxabs"], "refine_iters": st_o["refine_iters"],
            "fp64_lines": st_o["fp64_lines"], "last_update_rel": st_o["last_update_rel"]}
        del P_main
    plan.close()
    del Uh, Vh, Wh, U, V, W, P
    torch.cuda.empty_cache()
    if "batched" in legs:
        extra["batched"] = run_batched(device, steps=max(3, args.steps // 4), warmup=args.warmup, rank=rank,
                                       world=world, dist=dist, tune=args.batch_tune == "auto")
        torch.cuda.empty_cache()
    if world == 1:
        if "served" in legs and args.served_seconds > 0:  # --served-seconds 0 leaves the served legs out
            extra["served"] = run_served(device, args.served_seconds, args.served_rate, args.served_budget_gb * 1e9)
            torch.cuda.empty_cache()
            # the same request mix at a rate one GPU sustains: latency without queue growth
            extra["served_sustainable"] = run_served(device, min(10.0, args.served_seconds), 1000.0,
                                                     args.served_budget_gb * 1e9)
            torch.cuda.empty_cache()
            # requests that bring their fields from host memory and take their results back there
            # (PCIe-bound: about 0.9 GB of copies per request of the mix)
            extra["served_host_io"] = run_served(device, min(10.0, args.served_seconds), 40.0,
                                                 args.served_budget_gb * 1e9, io="host")
            torch.cuda.empty_cache()
        if "vd" in legs:
            extra["variable_density"] = run_vd(device, NX, NY, NZ, steps=max(3, args.steps // 4),
                                               warmup=args.warmup)
            torch.cuda.empty_cache()
        if "rough" in legs and args.rough_grid:
            rx, ry, rz = (int(v) for v in args.rough_grid.lower().split("x"))
            extra["rough_wall"] = run_rough(device, rx, ry, rz, steps=max(3, args.steps // 10), warmup=args.warmup)
            torch.cuda.empty_cache()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Gpts/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"pressure projection step {NX}x{NY}x{NZ} (channel Lx=2pi Lz=pi, tanh beta=2, "
                                   "Poiseuille + N(0,0.1) predictor)", "nx": NX, "ny": NY, "nz": NZ,
                       "mode": args.mode, "bands": "consistent", "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (3 x 0.92 GB fields), no flush"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                         "alg_bytes_per_launch": alg[dom], "avg_launch_ms": dom_ms},
            "roofline_step": {"alg_bytes_per_point": ALG_BYTES_PER_POINT, "achieved": roof_step, "peak": peak,
                              "unit": "GB/s", "frac": roof_step / peak},
            "roofline_kernels": per_kernel,
            "stages_ms_per_launch": {k: v[0] / v[1] for k, v in stages.items()},
            "stage_share": {k: v[0] / sum(x[0] for x in stages.values()) for k, v in stages.items()},
            "gpu_launches": launches,
            "accuracy": {"div_maxabs": st["div_maxabs"], "p_maxabs": st["p_maxabs"], "min_pivot": st["min_pivot"],
                         **(parity["consistent_bands"] if parity else {}), "vs_oracle": parity},
            "clocks": clk.summary(),
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""Autotuner of the pressure-Poisson engine: launch shapes and FFT radix plans.

For one grid size it times candidate tunings of a plan (prj_tuning,
include/projection.h) on an in-place FP64 solve with CUDA events, in two phases:
first the launch shapes -- x-rows per CTA of the x transforms, spectral rows per
CTA of the z transforms, split versus fused z kernels -- in the default radix
orders; then, with the best shapes, every compiled radix order of the x and z
transform lengths (the pass plans of fft_pass.cuh, where the reference lets
FFTW/cuFFT pick a factorisation at plan time, poisson_solver_multigpu.f90:77-129).
The fastest is applied and cached in a JSON file keyed by grid size and device name
(PRJ_AUTOTUNE_CACHE, default ~/.cache/prj_b200/autotune.json).
"""
from __future__ import annotations

import json
import os

import prj

CACHE = os.environ.get("PRJ_AUTOTUNE_CACHE",
                       os.path.join(os.path.expanduser("~"), ".cache", "prj_b200", "autotune.json"))


def _load_cache():
    try:
        with open(CACHE) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save_cache(d):
    try:
        os.makedirs(os.path.dirname(CACHE), exist_ok=True)
        tmp = CACHE + ".tmp"
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, CACHE)
    except OSError:
        pass


def key(plan) -> str:
    import torch
    g = plan.grid
    return f"{g.nx}x{g.nz}x{g.ny}:{torch.cuda.get_device_name(plan.device)}"


def candidates(plan):
    out = []
    for z_mode in (0, 1, 3):
        for x_rows in (2, 4, 8, 16):
            for z_rows in ((0, 4, 8, 16) if z_mode == 0 else (0,)):
                if z_mode == 3 and x_rows not in (4, 8):
                    continue
                out.append(dict(x_rows=x_rows, z_rows=z_rows, z_mode=z_mode))
    return out


# compiled radix orders per transform length (fft_pass.cuh PRJ_PASS_PLANS + PRJ_PASS_ALTS)
RADIX_ORDERS = {64: 2, 96: 2, 128: 2, 192: 2, 256: 3, 384: 3}


def order_candidates(plan, shape):
    """The best launch shape in every combination of the compiled radix orders."""
    g = plan.grid
    nxo = RADIX_ORDERS.get(g.nx // 2, 1) if g.nx % 2 == 0 else 1
    nzo = RADIX_ORDERS.get(g.nz, 1)
    return [dict(shape, x_order=xo, z_order=zo) for xo in range(nxo) for zo in range(nzo) if xo or zo]


def time_solve(plan, P, reps):
    import torch
    s = torch.cuda.current_stream(plan.device)
    plan.poisson_fp64(P, stream=s)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        plan.poisson_fp64(P, stream=s)
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


FIELDS = ("x_rows", "z_rows", "z_mode", "x_order", "z_order")


def _apply(plan, t):
    plan.set_tuning(**{k: t.get(k, 0) for k in FIELDS})


def tune(plan, reps: int = 5, use_cache: bool = True) -> dict:
    """Apply the fastest tuning for this plan's grid (cached) and return it with its time."""
    import torch
    k = key(plan)
    cache = _load_cache() if use_cache else {}
    if k in cache:
        t = cache[k]
        _apply(plan, t)
        return dict(t, cached=True)
    g = plan.grid
    P = torch.randn((g.ny, g.nz, g.nx), dtype=torch.float64, device=f"cuda:{plan.device}")
    best = None
    default = plan.tuning
    for phase in (0, 1):
        cands = candidates(plan) if phase == 0 else order_candidates(plan, {f: best[f] for f in FIELDS})
        for c in cands:
            c = dict({"x_order": 0, "z_order": 0}, **c)
            try:
                _apply(plan, c)
            except prj.PrjError:
                continue
            ms = time_solve(plan, P, reps)
            if best is None or ms < best["ms"]:
                best = dict(c, ms=ms)
        if best is None:
            _apply(plan, default)
            return dict(default, ms=None, cached=False)
    _apply(plan, best)
    if use_cache:
        cache = _load_cache()
        cache[k] = best
        _save_cache(cache)
    return dict(best, cached=False)

"""ctypes harness of the B200 pressure-projection engine (libprj_b200.so).

Two faces over the same C ABI (include/projection.h):

* ``Plan`` -- Pythonic: build from the face grid ``yu`` (or explicit band
  arrays), then ``poisson_fp64(P)`` / ``projection_step(...)`` on torch CUDA
  tensors (device-resident, asynchronous on the current stream) or on numpy
  arrays (host buffers; copies in and out).
* ``init_spec_poisson_multigpu`` / ``run_spec_poisson_multigpu`` -- the two
  entry points of the reference's Fortran module ``poisson_solver_multigpu``
  (src/poisson_solver_mgpu_dtdma/poisson_solver_multigpu.f90:33, :328) with
  their argument meaning kept for the single-rank case: the first builds the
  solver from the bands and grid spacings, the second overwrites P (RHS in,
  solution out).

Layouts follow the reference: numpy arrays are Fortran-ordered ``[x, z, y]``;
torch tensors use the same memory as C-contiguous ``[y, z, x]``.

The engine has no CPU fallback: if the library is missing or no GPU is
visible, creating a plan raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libprj_b200.so")

PRJ_OK = 0
PRJ_ERR_ARG = -1
PRJ_ERR_UNSUPPORTED = -2
PRJ_ERR_CUDA = -3
PRJ_ERR_OOM = -4
PRJ_ERR_NUMERIC = -5
PRJ_ERR_TIMEOUT = -6
PRJ_ERR_STATE = -7

MODE_FP64 = 0
MODE_FP32_REFINE = 1
BATCH_GRAPH = 0x10  # or-ed into a batch's mode: the CUDA-graph form

# every symbol include/projection.h declares
EXPORTS = (
    "prj_plan_create", "prj_plan_destroy", "prj_poisson_fp64", "prj_projection_step",
    "prj_poisson_fp64_host", "prj_projection_step_host", "prj_plan_min_pivot",
    "prj_plan_device_bytes", "prj_last_error_string", "prj_version",
    "prj_bands_from_yu", "prj_metrics_from_yu",
    "prj_plan_enable_stage_timing", "prj_plan_stage_times", "prj_stage_name",
    "prj_poisson_fp64_noalloc", "prj_poisson_mixed",
    "prj_batch_create", "prj_batch_launch", "prj_batch_destroy", "prj_batch_info", "prj_batch_check_error",
    "prj_plan_get_tuning", "prj_plan_set_tuning",
    "prj_vd_metric_from_yu", "prj_plan_set_vd_metric", "prj_projection_step_vd",
    "prj_field_read_header", "prj_field_read", "prj_field_write", "prj_field_read_device",
    "prj_field_write_device", "prj_rough_force", "prj_ibm_interp", "prj_plan_schedule",
    "prj_projection_step_host_async", "prj_host_async_wait", "prj_selftest_wait_timeout",
    "prj_dist_forward", "prj_dist_pack", "prj_dist_thomas", "prj_dist_unpack", "prj_dist_inverse",
    "prj_dist_divergence", "prj_dist_correct", "prj_selftest_division", "prj_plan_check_error",
    "prj_geom_read_column", "prj_geom_read_bands", "prj_geom_read_metrics", "prj_geom_read_base_params",
    "prj_synth_channel_predictor",
)

BANDS_REFERENCE = 0
BANDS_CONSISTENT = 1


class PrjError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"prj error {code}: {msg}")
        self.code = code


class Stats(ctypes.Structure):
    _fields_ = [("div_maxabs", ctypes.c_double), ("p_maxabs", ctypes.c_double),
                ("min_pivot", ctypes.c_double), ("refine_iters", ctypes.c_int),
                ("fp64_lines", ctypes.c_int), ("last_update_rel", ctypes.c_double),
                ("rho_min", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tuning(ctypes.Structure):
    _fields_ = [("x_rows", ctypes.c_int), ("z_rows", ctypes.c_int), ("z_mode", ctypes.c_int),
                ("z_planes", ctypes.c_int), ("z_stages", ctypes.c_int), ("thomas_ring", ctypes.c_int),
                ("mixed_iters", ctypes.c_int), ("mixed_tau", ctypes.c_double), ("x_order", ctypes.c_int),
                ("z_order", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class VdFields(ctypes.Structure):
    _fields_ = [("rho", ctypes.c_void_p), ("P_now", ctypes.c_void_p), ("P_old", ctypes.c_void_p),
                ("div_now", ctypes.c_void_p), ("P_next", ctypes.c_void_p)]


class RoughInds(ctypes.Structure):
    _fields_ = [(f"{c}_{w}", ctypes.c_void_p) for c in "UVW" for w in ("bot", "top")]


class CaseParams(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("nz", ctypes.c_int), ("ny", ctypes.c_int), ("use_rough_surf", ctypes.c_int),
                ("nstep", ctypes.c_longlong), ("dtmax", ctypes.c_double), ("dx", ctypes.c_double),
                ("dz", ctypes.c_double),
                ("wall_U_bot", ctypes.c_double), ("wall_V_bot", ctypes.c_double), ("wall_W_bot", ctypes.c_double),
                ("wall_U_top", ctypes.c_double), ("wall_V_top", ctypes.c_double), ("wall_W_top", ctypes.c_double),
                ("use_incompressible", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class StepParams(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double),
                ("wall_U_bot", ctypes.c_double), ("wall_V_bot", ctypes.c_double), ("wall_W_bot", ctypes.c_double),
                ("wall_U_top", ctypes.c_double), ("wall_V_top", ctypes.c_double), ("wall_W_top", ctypes.c_double),
                ("compute_stats", ctypes.c_int)]


_lib = None
_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p


def load_library(path: str | None = None) -> ctypes.CDLL:
    """Load libprj_b200.so (building it first if the sources are newer)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    path = path or LIB_PATH
    if path == LIB_PATH:
        import importlib.util
        spec = importlib.util.spec_from_file_location("_prj_build", os.path.join(HERE, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        if mod.needs_build():
            mod.build()
    if not os.path.exists(path):
        raise RuntimeError(f"engine library missing: {path} (run dns-supercritical-ibm_b200/build.py)")
    L = ctypes.CDLL(path)
    i, d, u = ctypes.c_int, ctypes.c_double, ctypes.c_uint
    L.prj_plan_create.argtypes = [i, i, i, d, d, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, u, i, ctypes.POINTER(_vp)]
    L.prj_plan_destroy.argtypes = [_vp]
    L.prj_poisson_fp64.argtypes = [_vp, _vp, _vp]
    L.prj_projection_step.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(StepParams), i,
                                      ctypes.POINTER(Stats), _vp]
    L.prj_poisson_fp64_host.argtypes = [_vp, _dp]
    L.prj_projection_step_host.argtypes = [_vp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, ctypes.POINTER(StepParams), i,
                                           ctypes.POINTER(Stats)]
    L.prj_plan_min_pivot.argtypes = [_vp, _dp]
    L.prj_plan_check_error.argtypes = [_vp, _vp]
    L.prj_synth_channel_predictor.argtypes = [i, i, i, _vp, ctypes.c_ulonglong, d, _vp, _vp, _vp, _vp]
    L.prj_geom_read_column.argtypes = [ctypes.c_char_p, i, i, i, _dp]
    L.prj_geom_read_bands.argtypes = [ctypes.c_char_p, i, _dp, _dp, _dp, _dp, _dp, _dp]
    L.prj_geom_read_metrics.argtypes = [ctypes.c_char_p, i, _dp, _dp, _dp]
    L.prj_geom_read_base_params.argtypes = [ctypes.c_char_p, ctypes.POINTER(CaseParams)]
    L.prj_plan_device_bytes.argtypes = [_vp, ctypes.POINTER(ctypes.c_size_t)]
    L.prj_bands_from_yu.argtypes = [i, _dp, i, _dp, _dp, _dp, _dp, _dp, _dp]
    L.prj_metrics_from_yu.argtypes = [i, _dp, _dp, _dp, _dp]
    L.prj_plan_enable_stage_timing.argtypes = [_vp, i]
    L.prj_plan_stage_times.argtypes = [_vp, _dp, ctypes.POINTER(ctypes.c_int), i, ctypes.POINTER(ctypes.c_int)]
    L.prj_stage_name.argtypes = [i]
    L.prj_poisson_fp64_noalloc.argtypes = [i, i, i, d, d, _dp, _dp, _dp, _dp, _dp, _dp, _vp, _vp]
    L.prj_poisson_mixed.argtypes = [_vp, _vp, _vp]
    L.prj_batch_create.argtypes = [ctypes.POINTER(_vp), ctypes.POINTER(_vp), i, i, ctypes.POINTER(_vp)]
    L.prj_batch_launch.argtypes = [_vp, _vp]
    L.prj_batch_destroy.argtypes = [_vp]
    L.prj_batch_info.argtypes = [_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                 ctypes.POINTER(ctypes.c_longlong)]
    L.prj_batch_check_error.argtypes = [_vp, _vp]
    L.prj_plan_get_tuning.argtypes = [_vp, ctypes.POINTER(Tuning)]
    L.prj_plan_set_tuning.argtypes = [_vp, ctypes.POINTER(Tuning)]
    L.prj_vd_metric_from_yu.argtypes = [i, _dp, _dp]
    L.prj_plan_schedule.argtypes = [_vp, i, ctypes.POINTER(i)]
    L.prj_projection_step_host_async.argtypes = [_vp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, ctypes.POINTER(StepParams), i]
    L.prj_host_async_wait.argtypes = [_vp]
    L.prj_selftest_wait_timeout.argtypes = [i, ctypes.c_longlong]
    L.prj_rough_force.argtypes = [i, i, i, _vp, _vp, _vp, ctypes.POINTER(RoughInds), ctypes.POINTER(StepParams), _vp]
    ll = ctypes.c_longlong
    L.prj_ibm_interp.argtypes = [_vp, ll, i, _vp, _vp, _vp, _vp, _vp, _vp, i, _vp, _vp, _vp, _vp]
    cp, ip = ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)
    L.prj_field_read_header.argtypes = [cp, ip, ip, ip]
    L.prj_field_read.argtypes = [cp, i, i, i, _dp, i]
    L.prj_field_write.argtypes = [cp, i, i, i, _dp, i]
    L.prj_field_read_device.argtypes = [cp, i, i, i, _vp, i, i]
    L.prj_field_write_device.argtypes = [cp, i, i, i, _vp, i, i]
    L.prj_plan_set_vd_metric.argtypes = [_vp, _dp]
    L.prj_projection_step_vd.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(StepParams),
                                         ctypes.POINTER(VdFields), i, ctypes.POINTER(Stats), _vp]
    L.prj_dist_forward.argtypes = [_vp, _vp, i, i, _vp]
    L.prj_dist_pack.argtypes = [_vp, i, i, ip, i, _vp, _vp]
    L.prj_dist_thomas.argtypes = [_vp, _vp, i, i, _vp]
    L.prj_dist_unpack.argtypes = [_vp, i, i, ip, i, _vp, _vp]
    L.prj_dist_inverse.argtypes = [_vp, _vp, i, i, _vp]
    L.prj_selftest_division.argtypes = [i, ctypes.c_longlong, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_longlong),
                                        ctypes.POINTER(d), ctypes.POINTER(d)]
    L.prj_dist_divergence.argtypes = [_vp, _vp, _vp, _vp, i, i, ctypes.POINTER(StepParams), _vp]
    L.prj_dist_correct.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, i, i, ctypes.POINTER(StepParams), _vp]
    for name in EXPORTS:
        getattr(L, name).restype = ctypes.c_int
    L.prj_last_error_string.restype = ctypes.c_char_p
    L.prj_version.restype = ctypes.c_char_p
    L.prj_stage_name.restype = ctypes.c_char_p
    if path == LIB_PATH:
        _lib = L
    return L


def _check(rc: int):
    if rc != PRJ_OK:
        raise PrjError(rc, load_library().prj_last_error_string().decode())


def _arr(v, n=None):
    a = np.ascontiguousarray(v, dtype=np.float64)
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _torch():
    import torch
    return torch


def _is_tensor(x):
    try:
        torch = _torch()
    except ImportError:  # pragma: no cover
        return False
    return isinstance(x, torch.Tensor)


def _stream_ptr(stream):
    if stream is not None:
        return ctypes.c_void_p(int(stream.cuda_stream) if hasattr(stream, "cuda_stream") else int(stream))
    torch = _torch()
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def bands(yu, mode="reference"):
    """(a, b, c, a00, b00, c00) from the face grid (prj_bands_from_yu; host-only).

    mode "reference": calc_bands.mk_P_abc; "consistent": div(grad p) bands."""
    yu = _arr(yu)
    ny = yu.size - 1
    out = [np.zeros(ny) for _ in range(6)]
    m = {"reference": BANDS_REFERENCE, "consistent": BANDS_CONSISTENT}[mode]
    _check(load_library().prj_bands_from_yu(ny, _p(yu), m, *[_p(v) for v in out]))
    return tuple(out)


def synth_predictor(Uh, Vh, Wh, yp, seed, sigma=0.1, stream=None):
    """Channel predictor of `seed` in place on halo'd [y+2, z+2, x+2] CUDA tensors
    (prj_synth_channel_predictor): Poiseuille profile over the cell centres yp (CUDA
    tensor, ny values) plus N(0, sigma) noise, v = 0 on the bottom wall face."""
    ny, nz, nx = Uh.shape[0] - 2, Uh.shape[1] - 2, Uh.shape[2] - 2
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    _check(load_library().prj_synth_channel_predictor(nx, nz, ny, p(yp), int(seed) & (2 ** 64 - 1), float(sigma),
                                                      p(Uh), p(Vh), p(Wh), _stream_ptr(stream)))


def vd_metric(yu):
    """inv_dy_p_pad (ny+1) of the variable-density step (prj_vd_metric_from_yu; host-only)."""
    yu = _arr(yu)
    out = np.zeros(yu.size)
    _check(load_library().prj_vd_metric_from_yu(yu.size - 1, _p(yu), _p(out)))
    return out


def metrics(yu):
    """(inv_dy_p, dPdy_lo, dPdy_hi) from the face grid (prj_metrics_from_yu; host-only)."""
    yu = _arr(yu)
    ny = yu.size - 1
    out = [np.zeros(ny) for _ in range(3)]
    _check(load_library().prj_metrics_from_yu(ny, _p(yu), *[_p(v) for v in out]))
    return tuple(out)


def read_geom(geom_dir):
    """A reference case's geometry folder (geom_data written by calc_bands.py): the
    base_params.txt records of this path, the six band arrays and the three metrics
    (prj_geom_read_*; host-only)."""
    L = load_library()
    enc = os.fsencode(geom_dir)
    cp = CaseParams()
    _check(L.prj_geom_read_base_params(os.path.join(enc, b"base_params.txt"), ctypes.byref(cp)))
    ny = cp.ny
    b6 = [np.zeros(ny) for _ in range(6)]
    m3 = [np.zeros(ny) for _ in range(3)]
    _check(L.prj_geom_read_bands(enc, ny, *[_p(v) for v in b6]))
    _check(L.prj_geom_read_metrics(enc, ny, *[_p(v) for v in m3]))
    return {"params": cp.as_dict(), "bands": tuple(b6), "metrics": tuple(m3)}


@dataclass
class Grid:
    nx: int
    nz: int
    ny: int
    dx: float
    dz: float


class Plan:
    """A solver plan on one GPU (prj_plan_create / prj_plan_destroy)."""

    def __init__(self, nx, nz, ny, dx, dz, bands6, metrics3=None, device=0):
        L = load_library()
        b = [_arr(v, ny) for v in bands6]
        m = [_arr(v, ny) for v in metrics3] if metrics3 is not None else [None, None, None]
        h = _vp()
        _check(L.prj_plan_create(nx, nz, ny, float(dx), float(dz), *[_p(v) for v in b], *[_p(v) for v in m], 0,
                                 device, ctypes.byref(h)))
        self._h = h
        self.grid = Grid(nx, nz, ny, float(dx), float(dz))
        self.device = device
        self.has_metrics = metrics3 is not None

    @classmethod
    def from_yu(cls, nx, nz, dx, dz, yu, band_mode="reference", device=0):
        """Build bands and metrics from the face grid ``yu`` (ny+1 values)."""
        yu = np.asarray(yu, dtype=np.float64)
        plan = cls(nx, nz, len(yu) - 1, dx, dz, bands(yu, band_mode), metrics(yu), device)
        plan.set_vd_metric(vd_metric(yu))
        return plan

    @classmethod
    def from_geom(cls, geom_dir, device=0):
        """A plan for a reference case's geometry folder (base_params.txt, P_band_abc(_00).dat,
        inv_dy_p.dat, dPdy_ddy_lh.dat); ``plan.case`` holds its base parameters."""
        geo = read_geom(geom_dir)
        c = geo["params"]
        plan = cls(c["nx"], c["nz"], c["ny"], c["dx"], c["dz"], geo["bands"], geo["metrics"], device)
        plan.case = c
        return plan

    def projection_step_host_async(self, Uh, Vh, Wh, U, V, W, P, dt, mode=MODE_FP64, wall=(0.0,) * 6):
        """Enqueue one pipelined host-buffer step (prj_projection_step_host_async); numpy
        Fortran-ordered arrays as for projection_step, ideally in pinned memory.  Call
        host_async_wait() before reading the outputs or reusing the buffers."""
        g = self.grid
        hs = (g.nx + 2, g.nz + 2, g.ny + 2)
        for a in (Uh, Vh, Wh, U, V, W):
            if not (a.dtype == np.float64 and a.flags.f_contiguous and a.shape == hs):
                raise ValueError(f"halo'd fields must be Fortran-ordered float64 arrays of shape {hs}")
        if not (P.dtype == np.float64 and P.flags.f_contiguous and P.shape == (g.nx, g.nz, g.ny)):
            raise ValueError("P must be a Fortran-ordered float64 array of shape (nx, nz, ny)")
        par = StepParams(float(dt), *[float(w) for w in wall], 0)
        _check(load_library().prj_projection_step_host_async(self.handle, _p(Uh), _p(Vh), _p(Wh), _p(U), _p(V),
                                                             _p(W), _p(P), ctypes.byref(par), mode))

    def host_async_wait(self):
        _check(load_library().prj_host_async_wait(self.handle))

    def launches_per_step(self, mode=MODE_FP64):
        """Kernel launches of one projection step of ``mode`` (prj_plan_schedule)."""
        n = ctypes.c_int()
        _check(load_library().prj_plan_schedule(self.handle, mode, ctypes.byref(n)))
        return n.value

    def set_vd_metric(self, inv_dy_p_pad):
        """inv_dy_p_pad (ny+1) for projection_step_vd (prj_plan_set_vd_metric)."""
        _check(load_library().prj_plan_set_vd_metric(self.handle, _p(_arr(inv_dy_p_pad, self.grid.ny + 1))))

    def close(self):
        if getattr(self, "_h", None):
            load_library().prj_plan_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover - best effort
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        if not self._h:
            raise PrjError(PRJ_ERR_STATE, "plan destroyed")
        return self._h

    @property
    def min_pivot(self) -> float:
        v = ctypes.c_double()
        _check(load_library().prj_plan_min_pivot(self.handle, ctypes.byref(v)))
        return v.value

    def check_error(self, stream=None):
        """Raise PrjError(PRJ_ERR_TIMEOUT) if a bounded device-side wait gave up since the last
        check (prj_plan_check_error; waits for the stream and clears the word)."""
        _check(load_library().prj_plan_check_error(self.handle, _stream_ptr(stream)))

    @property
    def device_bytes(self) -> int:
        v = ctypes.c_size_t()
        _check(load_library().prj_plan_device_bytes(self.handle, ctypes.byref(v)))
        return v.value

    def enable_stage_timing(self, on=True):
        _check(load_library().prj_plan_enable_stage_timing(self.handle, 1 if on else 0))

    def stage_times(self):
        """{kernel name: (total ms, launches)} recorded since the last call (synchronises)."""
        L = load_library()
        n = 12
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_int * n)()
        ns = ctypes.c_int()
        _check(L.prj_plan_stage_times(self.handle, ms, cnt, n, ctypes.byref(ns)))
        return {L.prj_stage_name(i).decode(): (ms[i], cnt[i]) for i in range(ns.value) if cnt[i]}

    @property
    def tuning(self) -> dict:
        t = Tuning()
        _check(load_library().prj_plan_get_tuning(self.handle, ctypes.byref(t)))
        return t.as_dict()

    def set_tuning(self, x_rows=None, z_rows=None, z_mode=None, **kw):
        """Change some fields of the plan's tuning (prj_plan_set_tuning); the others keep their
        current values.  Fields: x_rows, z_rows, z_mode, z_planes, z_stages, thomas_ring,
        mixed_iters, mixed_tau, x_order, z_order."""
        t = self.tuning
        for k, v in (("x_rows", x_rows), ("z_rows", z_rows), ("z_mode", z_mode), *kw.items()):
            if k not in t:
                raise TypeError(f"unknown tuning field {k!r}")
            if v is not None:
                t[k] = v
        _check(load_library().prj_plan_set_tuning(self.handle, ctypes.byref(Tuning(**t))))

    # ---------------------------------------------------------------- solve
    def poisson_mixed(self, P, stream=None):
        """In-place Poisson solve with FP32 spectral storage and FP64 refinement (torch CUDA tensor)."""
        g = self.grid
        torch = _torch()
        if not (_is_tensor(P) and P.is_cuda and P.dtype == torch.float64 and P.is_contiguous()
                and tuple(P.shape) == (g.ny, g.nz, g.nx)):
            raise ValueError("P must be a contiguous float64 CUDA tensor of shape (ny, nz, nx)")
        _check(load_library().prj_poisson_mixed(self.handle, ctypes.c_void_p(P.data_ptr()), _stream_ptr(stream)))
        return P

    def poisson_fp64(self, P, stream=None):
        """In-place FP64 solve.  torch CUDA tensor [y, z, x] (async) or numpy [x, z, y] F-order (sync)."""
        g = self.grid
        L = load_library()
        if _is_tensor(P):
            torch = _torch()
            if not (P.is_cuda and P.dtype == torch.float64 and P.is_contiguous() and tuple(P.shape) == (g.ny, g.nz, g.nx)):
                raise ValueError("P must be a contiguous float64 CUDA tensor of shape (ny, nz, nx)")
            _check(L.prj_poisson_fp64(self.handle, ctypes.c_void_p(P.data_ptr()), _stream_ptr(stream)))
            return P
        if not (isinstance(P, np.ndarray) and P.dtype == np.float64 and P.flags.f_contiguous and P.shape == (g.nx, g.nz, g.ny)):
            raise ValueError("P must be a Fortran-ordered float64 array of shape (nx, nz, ny)")
        _check(L.prj_poisson_fp64_host(self.handle, _p(P)))
        return P

    def projection_step(self, Uh, Vh, Wh, U, V, W, P, dt, mode=MODE_FP64, wall=(0.0,) * 6, stats=True, stream=None):
        """One projection.  All torch CUDA tensors (halo'd [y+2, z+2, x+2], P [y, z, x]) or all numpy
        (halo'd F-order [x+2, z+2, y+2], P [x, z, y]).  Returns a Stats dict (or None if stats=False)."""
        g = self.grid
        L = load_library()
        par = StepParams(float(dt), *[float(w) for w in wall], 1 if stats else 0)
        st = Stats()
        sp = ctypes.byref(st) if stats else None
        if _is_tensor(Uh):
            torch = _torch()
            hs = (g.ny + 2, g.nz + 2, g.nx + 2)
            for t in (Uh, Vh, Wh, U, V, W):
                if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous() and tuple(t.shape) == hs):
                    raise ValueError(f"halo'd fields must be contiguous float64 CUDA tensors of shape {hs}")
            if not (P.is_cuda and P.dtype == torch.float64 and P.is_contiguous() and tuple(P.shape) == (g.ny, g.nz, g.nx)):
                raise ValueError("P must be a contiguous float64 CUDA tensor of shape (ny, nz, nx)")
            ptr = lambda t: ctypes.c_void_p(t.data_ptr())
            _check(L.prj_projection_step(self.handle, ptr(Uh), ptr(Vh), ptr(Wh), ptr(U), ptr(V), ptr(W), ptr(P),
                                         ctypes.byref(par), mode, sp, _stream_ptr(stream)))
        else:
            hs = (g.nx + 2, g.nz + 2, g.ny + 2)
            for a in (Uh, Vh, Wh, U, V, W):
                if not (a.dtype == np.float64 and a.flags.f_contiguous and a.shape == hs):
                    raise ValueError(f"halo'd fields must be Fortran-ordered float64 arrays of shape {hs}")
            if not (P.dtype == np.float64 and P.flags.f_contiguous and P.shape == (g.nx, g.nz, g.ny)):
                raise ValueError("P must be a Fortran-ordered float64 array of shape (nx, nz, ny)")
            _check(L.prj_projection_step_host(self.handle, _p(Uh), _p(Vh), _p(Wh), _p(U), _p(V), _p(W), _p(P),
                                              ctypes.byref(par), mode, sp))
        return st.as_dict() if stats else None


    def projection_step_vd(self, Uh, Vh, Wh, rho, P_now, P_old, div_now, U, V, W, P, P_next, dt, mode=MODE_FP64,
                           wall=(0.0,) * 6, stats=True, stream=None):
        """Variable-density projection (prj_projection_step_vd).  Torch CUDA tensors: halo'd
        [y+2, z+2, x+2] for Uh..W, rho, P_now, P_old, div_now, P_next; P [y, z, x].  The caller
        rotates P_old <- P_now <- P_next afterwards.  Returns a Stats dict (or None)."""
        g = self.grid
        L = load_library()
        torch = _torch()
        hs = (g.ny + 2, g.nz + 2, g.nx + 2)
        for t in (Uh, Vh, Wh, rho, P_now, P_old, div_now, U, V, W, P_next):
            if not (_is_tensor(t) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous() and tuple(t.shape) == hs):
                raise ValueError(f"halo'd fields must be contiguous float64 CUDA tensors of shape {hs}")
        if not (P.is_cuda and P.dtype == torch.float64 and P.is_contiguous() and tuple(P.shape) == (g.ny, g.nz, g.nx)):
            raise ValueError("P must be a contiguous float64 CUDA tensor of shape (ny, nz, nx)")
        par = StepParams(float(dt), *[float(w) for w in wall], 1 if stats else 0)
        st = Stats()
        ptr = lambda t: ctypes.c_void_p(t.data_ptr())
        f = VdFields(rho.data_ptr(), P_now.data_ptr(), P_old.data_ptr(), div_now.data_ptr(), P_next.data_ptr())
        _check(L.prj_projection_step_vd(self.handle, ptr(Uh), ptr(Vh), ptr(Wh), ptr(U), ptr(V), ptr(W), ptr(P),
                                        ctypes.byref(par), ctypes.byref(f), mode,
                                        ctypes.byref(st) if stats else None, _stream_ptr(stream)))
        return st.as_dict() if stats else None


# ----------------------------------------------------------------- IBM forcing
def rough_force(Uh, Vh, Wh, inds, wall=(0.0,) * 6, stream=None):
    """ibm_part_2 forcing in place (prj_rough_force).  Uh, Vh, Wh: halo'd torch CUDA tensors
    [y+2, z+2, x+2]; inds: dict with keys U_bot, U_top, V_bot, V_top, W_bot, W_top of contiguous
    int32 CUDA tensors [nz, nx] (column (i, j) at [j, i])."""
    torch = _torch()
    ny, nz, nx = (d - 2 for d in Uh.shape)
    keys = [f"{c}_{w}" for c in "UVW" for w in ("bot", "top")]
    for k in keys:
        t = inds[k]
        if not (t.is_cuda and t.dtype == torch.int32 and t.is_contiguous() and tuple(t.shape) == (nz, nx)):
            raise ValueError(f"{k} must be a contiguous int32 CUDA tensor of shape {(nz, nx)}")
    ri = RoughInds(*[inds[k].data_ptr() for k in keys])
    par = StepParams(1.0, *[float(w) for w in wall], 0)
    _check(load_library().prj_rough_force(nx, nz, ny, ctypes.c_void_p(Uh.data_ptr()), ctypes.c_void_p(Vh.data_ptr()),
                                          ctypes.c_void_p(Wh.data_ptr()), ctypes.byref(ri), ctypes.byref(par),
                                          _stream_ptr(stream)))


def ibm_interp(A, pos, src1, src2, c0, c1, c2, dst=None, src=None, stream=None):
    """Interpolated forcing points in place on torch CUDA tensor A (prj_ibm_interp):
    A[pos] = c1 A[src1] + c2 A[src2] + c0 (sources read first), then A[dst] = A[src].
    Offsets are int64 CUDA tensors into A's flat storage; coefficients float64 CUDA tensors."""
    torch = _torch()
    n = int(pos.numel())
    ncopy = int(dst.numel()) if dst is not None else 0
    scratch = torch.empty(2 * n + 1, dtype=torch.float64, device=A.device)
    vp = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None
    _check(load_library().prj_ibm_interp(vp(A), A.numel(), n, vp(pos), vp(src1), vp(src2), vp(c0), vp(c1), vp(c2),
                                         ncopy, vp(dst), vp(src), vp(scratch), _stream_ptr(stream)))


# ----------------------------------------------------------------- field files
def field_header(path):
    """(nx, nz, ny) of a field file (prj_field_read_header)."""
    v = [ctypes.c_int() for _ in range(3)]
    _check(load_library().prj_field_read_header(os.fsencode(path), *[ctypes.byref(x) for x in v]))
    return tuple(x.value for x in v)


def _field_dims(a, halo):
    if _is_tensor(a):
        ny, nz, nx = a.shape
    else:
        nx, nz, ny = a.shape
    return (nx - 2, nz - 2, ny - 2) if halo else (nx, nz, ny)


def write_field(path, a, halo=False):
    """Write a field in the reference's file format (src/mod_io.f90: int32 nx, nz, ny + float64
    interior, x fastest).  a: numpy Fortran-ordered [x, z, y] or a contiguous torch CUDA tensor
    [y, z, x]; halo=True for halo'd arrays (interior written)."""
    L = load_library()
    nx, nz, ny = _field_dims(a, halo)
    if _is_tensor(a):
        if not (a.is_cuda and a.is_contiguous() and str(a.dtype) == "torch.float64"):
            raise ValueError("tensor fields must be contiguous float64 CUDA tensors")
        _check(L.prj_field_write_device(os.fsencode(path), nx, nz, ny, ctypes.c_void_p(a.data_ptr()), int(halo),
                                        a.device.index or 0))
    else:
        if not (a.dtype == np.float64 and a.flags.f_contiguous):
            raise ValueError("numpy fields must be Fortran-ordered float64 arrays")
        _check(L.prj_field_write(os.fsencode(path), nx, nz, ny, _p(a), int(halo)))


def read_field(path, out=None, halo=False):
    """Read a field file into `out` (same conventions as write_field) or, when out is None, into
    a new numpy Fortran-ordered (nx, nz, ny) array.  A grid differing from out's raises PrjError."""
    L = load_library()
    if out is None:
        nx, nz, ny = field_header(path)
        out = np.empty((nx, nz, ny), order="F")
        halo = False
    nx, nz, ny = _field_dims(out, halo)
    if _is_tensor(out):
        if not (out.is_cuda and out.is_contiguous() and str(out.dtype) == "torch.float64"):
            raise ValueError("tensor fields must be contiguous float64 CUDA tensors")
        _check(L.prj_field_read_device(os.fsencode(path), nx, nz, ny, ctypes.c_void_p(out.data_ptr()), int(halo),
                                       out.device.index or 0))
    else:
        if not (out.dtype == np.float64 and out.flags.f_contiguous):
            raise ValueError("numpy fields must be Fortran-ordered float64 arrays")
        _check(L.prj_field_read(os.fsencode(path), nx, nz, ny, _p(out), int(halo)))
    return out


class Batch:
    """Many independent in-place Poisson solves in one launch (prj_batch_create /
    prj_batch_launch): one persistent kernel over a work queue for FP64 cases of the
    pass-plan lengths up to 256, else (or with graph=True) one CUDA graph.  Case i
    solves plans[i] on tensors[i]."""

    def __init__(self, plans, tensors, mode=MODE_FP64, graph=False):
        if len(plans) != len(tensors) or not plans:
            raise ValueError("need one tensor per plan")
        L = load_library()
        n = len(plans)
        hp = (_vp * n)(*[p.handle for p in plans])
        hd = (_vp * n)(*[ctypes.c_void_p(t.data_ptr()) for t in tensors])
        h = _vp()
        _check(L.prj_batch_create(hp, hd, n, mode | (BATCH_GRAPH if graph else 0), ctypes.byref(h)))
        self._h = h
        self._keep = (list(plans), list(tensors))  # the graph holds their addresses

    def launch(self, stream=None):
        _check(load_library().prj_batch_launch(self._h, _stream_ptr(stream)))

    @property
    def info(self) -> dict:
        """{"persistent", "kernels_per_launch", "work_items"} (prj_batch_info)."""
        p, k, w = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        _check(load_library().prj_batch_info(self._h, ctypes.byref(p), ctypes.byref(k), ctypes.byref(w)))
        return {"persistent": bool(p.value), "kernels_per_launch": k.value, "work_items": w.value}

    def check_error(self, stream=None):
        """Raise PrjError(PRJ_ERR_TIMEOUT) if a bounded wait of the persistent kernel gave up
        (prj_batch_check_error; waits for the stream)."""
        _check(load_library().prj_batch_check_error(self._h, _stream_ptr(stream)))

    def close(self):
        if getattr(self, "_h", None):
            load_library().prj_batch_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ------------------------------------------------------------------------------
# Mirror of the reference's Fortran module interface (single rank)
# ------------------------------------------------------------------------------

def init_spec_poisson_multigpu(P_band_a, P_band_b, P_band_c, P_band_a_00, P_band_b_00, P_band_c_00,
                               nx_glob, nz_glob, ny_loc, inv_dx, inv_dz, mpi_divs_z=1, mpi_divs_y=1, device=0):
    """Build the solver (init_spec_poisson_multigpu, poisson_solver_multigpu.f90:33-326).

    Arguments keep the reference's meaning; the FFT plans, a_x/a_z tables and
    the pivot table live inside the returned plan.  More than one rank is
    rejected (the reference would run its DTDMA path; the engine holds all of
    y on one GPU).  Prints the reference's min_abs_div_bacp INFO line.
    """
    if mpi_divs_z * mpi_divs_y != 1:
        raise PrjError(PRJ_ERR_UNSUPPORTED, "the engine runs one rank per solve (mpi_divs_z = mpi_divs_y = 1)")
    plan = Plan(nx_glob, nz_glob, ny_loc, 1.0 / inv_dx, 1.0 / inv_dz,
                (P_band_a, P_band_b, P_band_c, P_band_a_00, P_band_b_00, P_band_c_00), None, device)
    print(f"{'INFO: init_spec_poisson_multigpu, min_abs_div_bacp: ':>52}{plan.min_pivot:14.6E}", flush=True)
    return plan


def run_spec_poisson_multigpu(plan: Plan, P):
    """Solve in place (run_spec_poisson_multigpu, poisson_solver_multigpu.f90:328-554)."""
    return plan.poisson_fp64(P)

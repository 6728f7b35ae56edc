"""CPU oracle for the pressure projection -- TEST INFRASTRUCTURE ONLY.

Two independent restatements of the reference's algorithm live here:

* ``COracle`` -- ctypes bindings to ``libprj_oracle.so`` (``prj_oracle.c``), the
  plain-C restatement of the reference's FFTW path (halfcomplex R2HC/HC2R
  transforms, the ``poi_C`` Thomas sweep of
  src/poisson_solver_mgpu_dtdma/poisson_solver_multigpu.f90:395-422, the
  1/(nx*nz) scale of :540-551, the divergence of src/mod_cfd_subroutines.f90:527-537
  and the correction of :1086-1152, :1223-1243).
* ``np_poisson`` -- a NumPy restatement of the same solve in the complex
  rfft2 formulation that the reference's own Python checker uses
  (tests/test_poisson_solver_and_ibm_rand/py_poi_solver.py:96-131).

Only tests, the smoke check and the CPU-baseline leg of the benchmark import
this module, and only as the checker.  The CUDA engine never calls it.

Array convention: numpy arrays indexed ``[i, j, k]`` = (x, z, y) stored in
Fortran order (x fastest), exactly the reference's ``P(i, j, k)``.  Halo'd
fields have shape (nx+2, nz+2, ny+2) with index offset 1.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libprj_oracle.so")


# --------------------------------------------------------------------------
# geometry helpers (calc_bands.py restatements, NumPy)
# --------------------------------------------------------------------------

def yp_ext_from_yu(yu: np.ndarray) -> list:
    """[yu_0, yp_0 .. yp_{ny-1}, yu_ny], calc_bands.py:226-227."""
    yu = [float(v) for v in np.asarray(yu).reshape(-1)]
    ny = len(yu) - 1
    yp = [(yu[i] + yu[i + 1]) / 2 for i in range(ny)]
    return [yu[0]] + yp + [yu[-1]]


def mk_P_abc(yp_ext, is_dirich_first=False):
    """Restatement of calc_bands.py:181-201; returns three arrays (a, b, c)."""
    yp_ext = [float(v) for v in yp_ext]
    ny = len(yp_ext) - 2
    pad = list(yp_ext)
    pad[0] = 2 * yp_ext[0] - yp_ext[1]
    pad[-1] = 2 * yp_ext[-1] - yp_ext[-2]
    a = np.zeros(ny)
    b = np.zeros(ny)
    c = np.zeros(ny)
    for i in range(ny):
        x0, x1, x2 = pad[i], pad[i + 1], pad[i + 2]
        dy = 0.5 * (x2 - x0)
        a[i] = 1.0 / ((x1 - x0) * dy)
        c[i] = 1.0 / ((x2 - x1) * dy)
        b[i] = -(a[i] + c[i])
    if is_dirich_first:
        b[0] -= a[0]
    else:
        b[0] += a[0]
    b[-1] += c[-1]
    a[0] = 0.0
    c[-1] = 0.0
    return a, b, c


def bands(yu, mode="reference"):
    """(a, b, c, a00, b00, c00) for the wall-normal Laplacian.

    mode "reference": the reference's bands (mk_P_abc, plain and pinned).
    mode "consistent": the bands of div(grad p) built from the same 1-D metrics
    that the divergence and correction use, so max|div u| reaches round-off.
    """
    yu = np.asarray(yu, dtype=np.float64).reshape(-1)
    ny = len(yu) - 1
    if mode == "reference":
        ext = yp_ext_from_yu(yu)
        return (*mk_P_abc(ext, False), *mk_P_abc(ext, True))
    if mode != "consistent":
        raise ValueError(mode)
    yp = (yu[:-1] + yu[1:]) / 2
    idy = 1.0 / (yu[1:] - yu[:-1])
    a = np.zeros(ny)
    c = np.zeros(ny)
    a[1:] = idy[1:] / (yp[1:] - yp[:-1])
    c[:-1] = idy[:-1] / (yp[1:] - yp[:-1])
    b = -(a + c)
    b00 = b.copy()
    ghost = 2 * yu[0] - yp[0]
    b00[0] -= 2.0 * (1.0 / (yu[1] - yu[0])) / (yp[0] - ghost)
    return a, b, c, a.copy(), b00, c.copy()


def metrics(yu):
    """(inv_dy_p, dPdy_lo, dPdy_hi), each ny long: calc_bands.py:274, :336-343."""
    yu = np.asarray(yu, dtype=np.float64).reshape(-1)
    ny = len(yu) - 1
    inv_dy_p = 1.0 / (yu[1:] - yu[:-1])
    yp = (yu[:-1] + yu[1:]) / 2
    lo = np.zeros(ny)
    hi = np.zeros(ny)
    dy = yp[1:] - yp[:-1]
    lo[1:] = -1 / dy
    hi[1:] = 1 / dy
    return inv_dy_p, lo, hi


# --------------------------------------------------------------------------
# NumPy restatement of the solve (complex rfft2 formulation)
# --------------------------------------------------------------------------

def np_poisson(rhs, dx, dz, bands6):
    """Solve with numpy's FFT; rhs indexed [x, z, y].  Returns a new array."""
    a, b, c, a00, b00, c00 = [np.asarray(v, dtype=np.float64) for v in bands6]
    nx, nz, ny = rhs.shape
    kx = np.arange(nx // 2 + 1)
    kz = np.fft.fftfreq(nz, d=1.0 / nz)
    ax = -4.0 / (dx * dx) * np.sin(kx * np.pi / nx) ** 2
    az = -4.0 / (dz * dz) * np.sin(kz * np.pi / nz) ** 2
    lam = ax[:, None] + az[None, :]
    spec = np.fft.rfft2(rhs, axes=(1, 0))  # [kx, kz, y]
    A = np.broadcast_to(a, lam.shape + (ny,)).copy()
    B = b[None, None, :] + lam[:, :, None]
    C = np.broadcast_to(c, lam.shape + (ny,)).copy()
    A[0, 0] = a00
    B[0, 0] = b00 + lam[0, 0]
    C[0, 0] = c00
    cp = np.empty_like(B)
    den = np.empty_like(B)
    den[..., 0] = B[..., 0]
    cp[..., 0] = C[..., 0] / den[..., 0]
    for k in range(1, ny):
        den[..., k] = B[..., k] - A[..., k] * cp[..., k - 1]
        cp[..., k] = C[..., k] / den[..., k]
    spec[..., 0] /= den[..., 0]
    for k in range(1, ny):
        spec[..., k] = (spec[..., k] - A[..., k] * spec[..., k - 1]) / den[..., k]
    for k in range(ny - 2, -1, -1):
        spec[..., k] -= cp[..., k] * spec[..., k + 1]
    return np.fft.irfft2(spec, s=(nz, nx), axes=(1, 0))


# --------------------------------------------------------------------------
# ctypes bindings to the C restatement
# --------------------------------------------------------------------------

def build_c_oracle(force: bool = False) -> str:
    """Compile libprj_oracle.so with the committed Makefile (gcc + OpenMP)."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "prj_oracle.c"))
    ):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_dp = ctypes.POINTER(ctypes.c_double)


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim == 1), "need float64 F-order"
    return a.ctypes.data_as(_dp)


class COracle:
    """ctypes front-end of the C oracle."""

    def __init__(self, path: str | None = None):
        path = path or build_c_oracle()
        self.lib = ctypes.CDLL(path)
        L = self.lib
        i, d = ctypes.c_int, ctypes.c_double
        L.orc_poisson.argtypes = [i, i, i, d, d, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, i]
        L.orc_divergence.argtypes = [i, i, i, d, d, d, _dp, _dp, _dp, _dp, d, d, _dp, i]
        L.orc_correction.argtypes = [i, i, i, d, d, d, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, i]
        L.orc_div_maxabs.argtypes = [i, i, i, d, d, _dp, _dp, _dp, _dp, i]
        L.orc_div_maxabs.restype = d
        L.orc_r2hc.argtypes = [i, _dp, _dp]
        L.orc_hc2r.argtypes = [i, _dp, _dp]
        L.orc_bands_from_yu.argtypes = [i, _dp, i, _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_metrics_from_yu.argtypes = [i, _dp, _dp, _dp, _dp]
        L.orc_mk_P_abc.argtypes = [i, _dp, i, _dp, _dp, _dp]
        L.orc_rho_min.argtypes = [i, i, i, _dp, i]
        L.orc_rho_min.restype = d
        L.orc_vd_metric_from_yu.argtypes = [i, _dp, _dp]
        L.orc_vd_rhs.argtypes = [i, i, i, d, d, d, _dp, _dp, _dp, _dp, _dp, d, d, _dp, _dp, _dp, _dp, d, _dp, i]
        L.orc_vd_correction.argtypes = [i, i, i, d, d, d, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, d,
                                        _dp, _dp, _dp, _dp, i]

    def poisson(self, rhs, dx, dz, bands6, nthreads=0):
        """Returns (P, min_pivot); rhs [x, z, y] is not modified."""
        P = np.array(rhs, dtype=np.float64, order="F", copy=True)
        nx, nz, ny = P.shape
        bb = [np.ascontiguousarray(v, dtype=np.float64) for v in bands6]
        mp = ctypes.c_double(0.0)
        rc = self.lib.orc_poisson(nx, nz, ny, dx, dz, *[_ptr(v) for v in bb], _ptr(P), ctypes.byref(mp), nthreads)
        if rc:
            raise RuntimeError(f"orc_poisson failed: {rc}")
        return P, mp.value

    def divergence(self, Uh, Vh, Wh, dx, dz, dt, inv_dy_p, vbot=0.0, vtop=0.0, nthreads=0):
        nx, nz, ny = Uh.shape[0] - 2, Uh.shape[1] - 2, Uh.shape[2] - 2
        P = np.zeros((nx, nz, ny), order="F")
        idy = np.ascontiguousarray(inv_dy_p, dtype=np.float64)
        rc = self.lib.orc_divergence(nx, nz, ny, dx, dz, dt, _ptr(idy), _ptr(Uh), _ptr(Vh), _ptr(Wh), vbot, vtop, _ptr(P), nthreads)
        if rc:
            raise RuntimeError(f"orc_divergence failed: {rc}")
        return P

    def correction(self, P, Uh, Vh, Wh, dx, dz, dt, dPdy_lo, dPdy_hi, wall=(0.0,) * 6, nthreads=0):
        nx, nz, ny = P.shape
        U = np.zeros_like(Uh, order="F")
        V = np.zeros_like(Vh, order="F")
        W = np.zeros_like(Wh, order="F")
        lo = np.ascontiguousarray(dPdy_lo, dtype=np.float64)
        hi = np.ascontiguousarray(dPdy_hi, dtype=np.float64)
        w = np.ascontiguousarray(wall, dtype=np.float64)
        P = np.asfortranarray(P, dtype=np.float64)
        rc = self.lib.orc_correction(nx, nz, ny, dx, dz, dt, _ptr(lo), _ptr(hi), _ptr(P), _ptr(Uh), _ptr(Vh), _ptr(Wh),
                                     _ptr(w), _ptr(U), _ptr(V), _ptr(W), nthreads)
        if rc:
            raise RuntimeError(f"orc_correction failed: {rc}")
        return U, V, W

    def div_maxabs(self, U, V, W, dx, dz, inv_dy_p, nthreads=0):
        nx, nz, ny = U.shape[0] - 2, U.shape[1] - 2, U.shape[2] - 2
        idy = np.ascontiguousarray(inv_dy_p, dtype=np.float64)
        return self.lib.orc_div_maxabs(nx, nz, ny, dx, dz, _ptr(idy), _ptr(U), _ptr(V), _ptr(W), nthreads)

    def projection(self, Uh, Vh, Wh, dx, dz, dt, yu, band_mode="reference", wall=(0.0,) * 6, nthreads=0):
        """divergence -> Poisson -> correction; returns (U, V, W, P)."""
        b6 = bands(yu, band_mode)
        idy, lo, hi = metrics(yu)
        P = self.divergence(Uh, Vh, Wh, dx, dz, dt, idy, wall[1], wall[4], nthreads)
        P, _ = self.poisson(P, dx, dz, b6, nthreads)
        U, V, W = self.correction(P, Uh, Vh, Wh, dx, dz, dt, lo, hi, wall, nthreads)
        return U, V, W, P

    # ------------------------------------------------ variable-density projection
    def vd_metric(self, yu):
        """inv_dy_p_pad (ny+1) from the faces (calc_bands.py:273, :276)."""
        yu = np.ascontiguousarray(yu, dtype=np.float64)
        out = np.zeros(len(yu))
        assert self.lib.orc_vd_metric_from_yu(len(yu) - 1, _ptr(yu), _ptr(out)) == 0
        return out

    def rho_min(self, rho, nthreads=0):
        nx, nz, ny = rho.shape[0] - 2, rho.shape[1] - 2, rho.shape[2] - 2
        return self.lib.orc_rho_min(nx, nz, ny, _ptr(np.asfortranarray(rho)), nthreads)

    def projection_vd(self, Uh, Vh, Wh, rho, P_now, P_old, div_now, dx, dz, dt, yu, band_mode="reference",
                      wall=(0.0,) * 6, nthreads=0):
        """Variable-density step (MCS:538-573, Poisson, MCS:1153-1197); returns
        (U, V, W, P, P_next, rho_min)."""
        nx, nz, ny = Uh.shape[0] - 2, Uh.shape[1] - 2, Uh.shape[2] - 2
        b6 = bands(yu, band_mode)
        idy, lo, hi = (np.ascontiguousarray(v) for v in metrics(yu))
        pad = self.vd_metric(yu)
        rmin = self.rho_min(rho, nthreads)
        F = [np.asfortranarray(a, dtype=np.float64) for a in (Uh, Vh, Wh, rho, P_now, P_old, div_now)]
        P = np.zeros((nx, nz, ny), order="F")
        rc = self.lib.orc_vd_rhs(nx, nz, ny, dx, dz, dt, _ptr(idy), _ptr(pad), _ptr(F[0]), _ptr(F[1]), _ptr(F[2]),
                                 wall[1], wall[4], _ptr(F[3]), _ptr(F[4]), _ptr(F[5]), _ptr(F[6]), rmin, _ptr(P),
                                 nthreads)
        if rc:
            raise RuntimeError(f"orc_vd_rhs failed: {rc}")
        P, _ = self.poisson(P, dx, dz, b6, nthreads)
        U, V, W, P_next = (np.zeros_like(F[0], order="F") for _ in range(4))
        w = np.ascontiguousarray(wall, dtype=np.float64)
        rc = self.lib.orc_vd_correction(nx, nz, ny, dx, dz, dt, _ptr(lo), _ptr(hi), _ptr(P), _ptr(F[0]), _ptr(F[1]),
                                        _ptr(F[2]), _ptr(w), _ptr(F[3]), _ptr(F[4]), _ptr(F[5]), rmin, _ptr(U),
                                        _ptr(V), _ptr(W), _ptr(P_next), nthreads)
        if rc:
            raise RuntimeError(f"orc_vd_correction failed: {rc}")
        return U, V, W, P, P_next, rmin

    def r2hc(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        hc = np.empty_like(x)
        assert self.lib.orc_r2hc(len(x), _ptr(x), _ptr(hc)) == 0
        return hc

    def hc2r(self, hc):
        hc = np.ascontiguousarray(hc, dtype=np.float64)
        x = np.empty_like(hc)
        assert self.lib.orc_hc2r(len(hc), _ptr(hc), _ptr(x)) == 0
        return x

    def bands_from_yu(self, yu, mode):
        yu = np.ascontiguousarray(yu, dtype=np.float64)
        ny = len(yu) - 1
        out = [np.zeros(ny) for _ in range(6)]
        m = {"reference": 0, "consistent": 1}[mode]
        assert self.lib.orc_bands_from_yu(ny, _ptr(yu), m, *[_ptr(v) for v in out]) == 0
        return tuple(out)

    def metrics_from_yu(self, yu):
        yu = np.ascontiguousarray(yu, dtype=np.float64)
        ny = len(yu) - 1
        out = [np.zeros(ny) for _ in range(3)]
        assert self.lib.orc_metrics_from_yu(ny, _ptr(yu), *[_ptr(v) for v in out]) == 0
        return tuple(out)


# --------------------------------------------------------------------- IBM forcing
def rough_force(Uh, Vh, Wh, inds, wall=(0.0,) * 6):
    """ibm_part_2 (src/ibm_setup/mod_cfd_ibm.f90:64-116) on halo'd [x+2, z+2, y+2] copies:
    column (i, j): k = 0..bot take the bottom wall value, k = top..ny-1 (v: ..ny) the top one.
    inds[name] is an (nx, nz) integer array.  Returns the forced (U, V, W)."""
    out = [np.array(a, order="F", copy=True) for a in (Uh, Vh, Wh)]
    ny = Uh.shape[2] - 2
    for F, c, lo, hi, kmax in ((out[0], "U", wall[0], wall[3], ny - 1), (out[1], "V", wall[1], wall[4], ny),
                               (out[2], "W", wall[2], wall[5], ny - 1)):
        bot, top = inds[f"{c}_bot"], inds[f"{c}_top"]
        nx, nz = bot.shape
        for i in range(nx):
            for j in range(nz):
                for k in range(0, bot[i, j] + 1):
                    F[i + 1, j + 1, k + 1] = lo
                for k in range(top[i, j], kmax + 1):
                    F[i + 1, j + 1, k + 1] = hi
    return tuple(out)


def ibm_interp(A, pos, src1, src2, c0, c1, c2, dst=(), src=()):
    """diezdecomp_ibm_exec on one rank (src/diezdecomp_api_ibm.f90:374-424) on the flat Fortran
    storage of A: sources gathered first, A[pos] = (c1 A[src1] + c2 A[src2]) + c0, then copies."""
    flat = np.array(A, order="F", copy=True).reshape(-1, order="F")
    g1, g2 = flat[np.asarray(src1)], flat[np.asarray(src2)]
    flat[np.asarray(pos)] = (np.asarray(c1) * g1 + np.asarray(c2) * g2) + np.asarray(c0)
    for d, s_ in zip(dst, src):
        flat[d] = flat[s_]
    return flat.reshape(A.shape, order="F")

"""Generate the golden fixtures of the pressure-Poisson parity tests.

Run ONCE, in a checkout that has the reference project next to it (it imports
the reference's own Python modules; nothing at test time does):

    python tests/golden/make_golden.py --reference /path/to/DNS-Supercritical-IBM

It writes three files next to this script:

trials_seed0.npz
    The ten seed-0 random trials of the reference's Poisson test generator
    (tests/test_poisson_solver_and_ibm_rand/mk_test_poisson_solver.py:109-151),
    reproduced draw for draw by calling that module's own helpers in the same
    order as its main loop (including the draws consumed by its IBM
    coefficients, mk_rand_ibm, so later trials see the same random state).
    For each trial: shape, (mpi_divs_z, mpi_divs_y), dx, dz, yu, the RHS
    ``A_input``, the reference output ``B_output`` (its rfftx2 solver, as the
    generator writes it) and the bands exactly as info.dat passes them to the
    Fortran driver (calc_bands.mk_P_abc, plain and pinned).

mms.npz
    The manufactured-solution convergence study of py_poi_solver.py:236-327:
    the sympy expressions of p and of its Laplacian (captured from the
    reference's own print), and for N = 4..64 the full-precision L-inf error of
    the reference solver against p (mean removed).  The stretched grid is the
    one of py_poi_solver.py:276-295, restated in ``mms_grid_y`` below; the
    check at the end pins that restatement against the reference's printed
    residuals.

channel_128x96x64.npz
    The channel Poisson case Nx=128, Ny=96, Nz=64 (tanh faces, beta=2,
    uniform[-1,1] RHS from default_rng(0) minus its dy-weighted mean) solved
    by the reference's Solver_Poisson_FFT_Thomas_3d: a strided subsample of
    the solution, its sum and sum of squares, and a checksum of the input.
"""
from __future__ import annotations

import argparse
import contextlib
import io
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "dns-supercritical-ibm_b200"))
import workloads  # noqa: E402


def mms_grid_y(L, n):
    """Stretched face grid of the manufactured-solution study (py_poi_solver.py:276-295)."""
    assert n % 2
    y, dy = [0.0], 1.0
    steps = iter(np.linspace(1, 10, n // 2).tolist())
    for _ in range(n // 2):
        y.append(y[-1] + dy)
        dy = next(steps)
    y = np.array(y) / max(y) * 0.5
    y[-1] = 0.5
    upper = np.cumsum(np.array(np.diff(y).tolist()[::-1]), 0)
    upper[-1] = 0.5
    y = y.tolist() + (0.5 + upper).tolist()
    y[-1] = 1
    y = np.array(y)
    y = y[:-1] + 0.5 * np.diff(y)
    return np.array([0.0] + y.tolist() + [1.0]) * L


def mms_fields(expr_p, expr_rhs, Lx, Ly, Lz, N):
    """rhs and p of the manufactured solution on the N x N x (N+1) grid ([x, z, y] order)."""
    env = dict(cos=np.cos, sin=np.sin, pi=np.pi)
    mk_p = lambda u: np.asarray(u)[:-1] + 0.5 * np.diff(u)
    yu = mms_grid_y(Ly, N + 1)
    xp = mk_p(np.linspace(0, Lx, N + 1)).reshape(-1, 1, 1)
    zp = mk_p(np.linspace(0, Lz, N + 1)).reshape(1, -1, 1)
    yp = mk_p(yu).reshape(1, 1, -1)
    dx = float(np.mean(np.diff(xp.reshape(-1))))
    dz = float(np.mean(np.diff(zp.reshape(-1))))
    shape = (N, N, yp.size)  # the stretched grid has N+1 cells in y
    rhs = eval(expr_rhs, env, dict(x=xp, y=yp, z=zp)) + np.zeros(shape)
    p = eval(expr_p, env, dict(x=xp, y=yp, z=zp)) + np.zeros(shape)
    return np.asfortranarray(rhs), np.asfortranarray(p), yu, dx, dz


def make_trials(ref_root):
    tdir = os.path.join(ref_root, "tests", "test_poisson_solver_and_ibm_rand")
    sys.path.insert(0, tdir)
    import mk_test_poisson_solver as G  # seeds random and np.random at import (SEED = 0)
    import random

    nproc_max, n_trials = 8, 10
    divs = [(i, j) for i in range(1, nproc_max + 1) for j in range(1, nproc_max + 1) if i * j <= nproc_max]
    out = {"n_trials": n_trials}
    for it in range(n_trials):
        mz, my = divs[random.randint(0, len(divs) - 1)]
        vmax = float("inf")
        while np.isnan(vmax) or vmax > 1e3:
            hi = max(10, 5 * max(my, mz))
            shape = [random.randint(max(my, mz), hi) for _ in range(2)] + [random.randint(2 * my, hi)]
            nx, nz, ny = shape
            dx, dz = [float(G.rand_val(0.1, 0.2)) for _ in range(2)]
            A = 5 * (np.random.rand(*shape) - 0.5)
            yu = np.array([0] + np.cumsum([G.rand_val(0.1, 0.2) for _ in range(ny)]).tolist()) + G.rand_val(-0.2, 0.2)
            B = G.Solver_Poisson_FFT_Thomas_3d_rfftx2(shape, dx + 0, dz + 0, yu.copy())(A.copy())
            vmax = np.fabs(B).max()
        check = np.fabs(B - G.Solver_Poisson_FFT_Thomas_3d(shape, dx + 0, dz + 0, yu.copy())(A.copy())).max()
        assert check < 1e-10
        yp = yu[:-1] + 0.5 * np.diff(yu)
        yp_ext = [float(v) for v in [yu[0]] + yp.tolist() + [yu[-1]]]
        abc = np.array(G.mk_P_abc(yp_ext, is_dirich_first=False))
        abc00 = np.array(G.mk_P_abc(yp_ext, is_dirich_first=True))
        n_ibm = random.randint(1, int(np.prod(shape)) // 5)
        [random.randint(0, 1) for _ in range(2)]  # nhalo, nskip
        G.mk_rand_ibm(shape, n_ibm, fname=None)  # consumes the IBM draws
        p = f"t{it}_"
        out[p + "shape"] = np.array(shape)
        out[p + "divs_zy"] = np.array([mz, my])
        out[p + "dxdz"] = np.array([dx, dz])
        out[p + "yu"] = yu
        out[p + "A_input"] = A
        out[p + "B_output"] = B
        out[p + "abc"] = abc
        out[p + "abc00"] = abc00
        print(f"trial {it}: shape={shape} divs_zy=({mz},{my}) dx={dx:.4f} dz={dz:.4f} max|B|={vmax:.3e}")
    sys.path.remove(tdir)
    return out


def make_mms(ref_root):
    tdir = os.path.join(ref_root, "tests", "test_poisson_solver_and_ibm_rand")
    sys.path.insert(0, tdir)
    import py_poi_solver as R

    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        R.test_poisson_solver()
    lines = buf.getvalue().splitlines()
    exprs = eval(lines[0].split("=", 1)[1])
    printed = {}
    for ln in lines[1:]:
        if ln.startswith("N:"):
            n = int(ln.split()[1])
            printed[n] = float(ln.split("residual:")[1].split(")")[0])
    Lx, Ly, Lz = 5.63, 2.0, 5.63 / 2
    Ns = [4, 8, 16, 32, 64]
    errs = []
    for N in Ns:
        rhs, p, yu, dx, dz = mms_fields(exprs["p"], exprs["rhs"], Lx, Ly, Lz, N)
        p = p - np.average(p)
        sol = R.Solver_Poisson_FFT_Thomas_3d(rhs.shape, dx, dz, yu)(np.array(rhs))
        sol = sol - np.average(sol)
        e = float(np.fabs(p - sol).max())
        errs.append(e)
        assert math.isclose(e, printed[N], rel_tol=2e-3), (N, e, printed[N])
        print(f"mms N={N}: err={e:.6e} (reference printed {printed[N]:.3e})")
    sys.path.remove(tdir)
    return dict(expr_p=np.array(exprs["p"]), expr_rhs=np.array(exprs["rhs"]), L=np.array([Lx, Ly, Lz]),
                N=np.array(Ns), err=np.array(errs))


def make_channel(ref_root):
    tdir = os.path.join(ref_root, "tests", "test_poisson_solver_and_ibm_rand")
    sys.path.insert(0, tdir)
    import py_poi_solver as R

    rhs, yu, dx, dz = workloads.poisson_rhs(128, 96, 64, beta=2.0, seed=0)
    P = R.Solver_Poisson_FFT_Thomas_3d(rhs.shape, dx, dz, yu)(np.array(rhs))
    sys.path.remove(tdir)
    return dict(shape=np.array(rhs.shape), dxdz=np.array([dx, dz]), yu=yu,
                rhs_sum=np.array(rhs.sum()), rhs_sumsq=np.array((rhs ** 2).sum()),
                P_sub=np.ascontiguousarray(P[::5, ::3, ::2]), P_sum=np.array(P.sum()),
                P_sumsq=np.array((P ** 2).sum()), stride=np.array([5, 3, 2]))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference project")
    args = ap.parse_args()
    np.savez_compressed(os.path.join(HERE, "trials_seed0.npz"), **make_trials(args.reference))
    np.savez_compressed(os.path.join(HERE, "mms.npz"), **make_mms(args.reference))
    np.savez_compressed(os.path.join(HERE, "channel_128x96x64.npz"), **make_channel(args.reference))


if __name__ == "__main__":
    main()

"""CPU tests of the variable-density projection's oracle (mod_cfd_subroutines.f90:538-573,
:1153-1221) and of the host-side metric builder of the C-ABI."""
import numpy as np

from conftest import rel_l2


def test_vd_metric_restatement(oracle):
    """inv_dy_p_pad = 1/diff(yp_pad), yp_pad = [2 yu_0 - yp_0, yp, 2 yu_ny - yp_{ny-1}]
    (calc_bands.py:273, :276), from the oracle and from the library's host builder."""
    import prj
    import workloads
    yu = workloads.tanh_faces(37, 1.7)
    yp = (yu[:-1] + yu[1:]) / 2
    yp_pad = np.concatenate([[2 * yu[0] - yp[0]], yp, [2 * yu[-1] - yp[-1]]])
    want = 1.0 / np.diff(yp_pad)
    np.testing.assert_array_equal(oracle.vd_metric(yu), want)
    np.testing.assert_array_equal(prj.vd_metric(yu), want)


def test_vd_constant_density_is_incompressible(oracle):
    """rho = 2 (a power of two) and div_now = 0: rho_+- = 1 - 2 (0.25 + 0.25) = 0 exactly, so the
    variable-density step is the incompressible one with P scaled by rho_min = 2, bit for bit."""
    import workloads
    nx, ny, nz = 24, 16, 12
    Uh, Vh, Wh, rho, Pn, Po, div, yu, dx, dz = workloads.vd_inputs(nx, ny, nz, rho_const=2.0)
    div[...] = 0.0
    wall = (0.1, 0.0, -0.2, 0.3, 0.0, 0.05)
    U, V, W, P, Pnext, rmin = oracle.projection_vd(Uh, Vh, Wh, rho, Pn, Po, div, dx, dz, 0.7, yu, "consistent", wall)
    assert rmin == 2.0
    Ui, Vi, Wi, Pi = oracle.projection(Uh, Vh, Wh, dx, dz, 0.7, yu, "consistent", wall)
    np.testing.assert_array_equal(P, 2.0 * Pi)
    for a, b in ((U, Ui), (V, Vi), (W, Wi)):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(Pnext, workloads.fill_halos(np.pad(P, 1)))


def test_vd_rhs_reduces_to_density_weighted_laplacian(oracle):
    """With u_hat = 0 and div_now = 0 the right-hand side is the density-weighted Laplacian of
    Ps = 2 P_now - P_old; checked against a NumPy restatement of MCS:543-564."""
    import prj
    import workloads
    nx, ny, nz = 10, 8, 6
    Uh, Vh, Wh, rho, Pn, Po, div, yu, dx, dz = workloads.vd_inputs(nx, ny, nz)
    for f in (Uh, Vh, Wh, div):
        f[...] = 0.0
    rmin = rho[1:-1, 1:-1, 1:-1].min()
    idy, _, _ = prj.metrics(yu)
    pad = oracle.vd_metric(yu)
    Ps = 2 * Pn - Po
    c = (slice(1, -1),) * 3

    def w(sl):
        return 1.0 - rmin * (0.5 / rho[sl] + 0.5 / rho[c])

    sh = lambda di, dj, dk: (slice(1 + di, nx + 1 + di), slice(1 + dj, nz + 1 + dj), slice(1 + dk, ny + 1 + dk))
    X = w(sh(1, 0, 0)) * (Ps[sh(1, 0, 0)] - Ps[c]) - w(sh(-1, 0, 0)) * (Ps[c] - Ps[sh(-1, 0, 0)])
    Z = w(sh(0, 1, 0)) * (Ps[sh(0, 1, 0)] - Ps[c]) - w(sh(0, -1, 0)) * (Ps[c] - Ps[sh(0, -1, 0)])
    Y = (w(sh(0, 0, 1)) * (Ps[sh(0, 0, 1)] - Ps[c]) * pad[None, None, 1:]
         - w(sh(0, 0, -1)) * (Ps[c] - Ps[sh(0, 0, -1)]) * pad[None, None, :-1])
    want = X / dx ** 2 + Z / dz ** 2 + Y * idy[None, None, :]
    import ctypes
    P = np.zeros((nx, nz, ny), order="F")
    F = [np.asfortranarray(a) for a in (Uh, Vh, Wh, rho, Pn, Po, div)]
    p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    rc = oracle.lib.orc_vd_rhs(nx, nz, ny, dx, dz, 1.0, p(np.ascontiguousarray(idy)), p(pad), p(F[0]), p(F[1]), p(F[2]),
                               0.0, 0.0, p(F[3]), p(F[4]), p(F[5]), p(F[6]), rmin, p(P), 1)
    assert rc == 0
    assert rel_l2(P, want) <= 1e-13

/*
 * prj_oracle.h -- CPU oracle for the pressure projection.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * FFTW (CPU) code path for the projection of one time step.  Only the tests,
 * the smoke check and the CPU-baseline leg of the benchmark may load it, and
 * only as the checker.  The product (the CUDA engine) never calls into it.
 *
 * What it restates (paths relative to the reference project root):
 *   - y-bands            src/pycode/calc_bands.py:181-201 (mk_P_abc)
 *   - 1-D metrics        src/pycode/calc_bands.py:274 (inv_dy_p), :336-343 (dPdy_ddy_lh)
 *   - solver set-up      src/poisson_solver_mgpu_dtdma/poisson_solver_multigpu.f90:83-104
 *                        (FFTW r2r R2HC/HC2R plans), :139-142 (halfcomplex wavenumber
 *                        map), :147-152 (a_x, a_z, poi_is_00), :164-179 (poi_C),
 *                        :181-197 (min_abs_div_bacp)
 *   - solve              poisson_solver_multigpu.f90:365 (x R2HC), :377 (x<->z
 *                        transpose), :383 (z R2HC), :395-422 (Thomas), :507 (z HC2R),
 *                        :520 (transpose back), :527 (x HC2R), :540-551 (1/(nx nz))
 *   - divergence         src/mod_cfd_subroutines.f90:504-537 (incompressible branch)
 *   - correction         src/mod_cfd_subroutines.f90:1086-1152 and :1223-1243
 *   - max|div u|         src/mod_get_bulk.f90:94-116
 * FFTW itself is absent from this machine, so the real-to-halfcomplex
 * transforms use a self-written mixed-radix complex FFT (textbook Cooley-Tukey)
 * and pack its output into FFTW's halfcomplex order
 * (r0, r1, ..., r_{n/2}, i_{(n+1)/2-1}, ..., i_1).
 *
 * Array layouts (Fortran column-major, x fastest, exactly as the reference):
 *   P        (0:nx-1, 0:nz-1, 0:ny-1)        idx = i + nx*(j + nz*k)
 *   halo'd   (-1:nx, -1:nz, -1:ny)           idx = (i+1) + (nx+2)*((j+1) + (nz+2)*(k+1))
 * Band arrays have ny entries (row k of the wall-normal tridiagonal).
 * All functions return 0 on success and a negative code on bad arguments.
 */
#ifndef PRJ_ORACLE_H
#define PRJ_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* y-bands of the Neumann pressure Laplacian, calc_bands.py:181-201.
 * yp_ext has ny+2 entries: [yu_0, yp_0 .. yp_{ny-1}, yu_ny]. */
int orc_mk_P_abc(int ny, const double* yp_ext, int is_dirich_first,
                 double* a, double* b, double* c);

/* Bands built from the face coordinates yu (ny+1 entries).
 * mode 0: the reference bands (mk_P_abc on yp_ext built as calc_bands.py:226-227).
 * mode 1: divergence-consistent bands a_k = inv_dy_p(k)/(yp_k-yp_{k-1}),
 *         c_k = inv_dy_p(k)/(yp_{k+1}-yp_k), b_k = -(a_k+c_k), a_0 = c_{ny-1} = 0;
 *         pinned variant b_0 -= 2*inv_dy_p(0)/(2*(yp_0-yu_0)) (same ghost as mode 0). */
int orc_bands_from_yu(int ny, const double* yu, int mode,
                      double* a, double* b, double* c,
                      double* a00, double* b00, double* c00);

/* inv_dy_p (ny), dPdy_lo (ny), dPdy_hi (ny) from yu, calc_bands.py:274, :336-343
 * (only rows 0..ny-1 of dPdy_ddy_lh are read by the solver, inc_set_alloc_arrays.f90:51-52). */
int orc_metrics_from_yu(int ny, const double* yu,
                        double* inv_dy_p, double* dPdy_lo, double* dPdy_hi);

/* The FFTW-path Poisson solve, in place on P (RHS in, solution out).
 * min_pivot (may be NULL) receives min_abs_div_bacp (poisson_solver_multigpu.f90:181-197).
 * nthreads <= 0 uses the OpenMP default. */
int orc_poisson(int nx, int nz, int ny, double dx, double dz,
                const double* a, const double* b, const double* c,
                const double* a00, const double* b00, const double* c00,
                double* P, double* min_pivot, int nthreads);

/* P = (1/dt) * div(u_hat), mod_cfd_subroutines.f90:504-537 (halos are
 * wrapped periodically in x and z; V_hat walls take vbot/vtop). */
int orc_divergence(int nx, int nz, int ny, double dx, double dz, double dt,
                   const double* inv_dy_p, const double* Uh, const double* Vh,
                   const double* Wh, double vbot, double vtop, double* P, int nthreads);

/* Velocity correction and the boundary fill of update_vars,
 * mod_cfd_subroutines.f90:1086-1152, :1223-1243.  wall[6] =
 * {U_bot, V_bot, W_bot, U_top, V_top, W_top}.  U, V, W are halo'd outputs. */
int orc_correction(int nx, int nz, int ny, double dx, double dz, double dt,
                   const double* dPdy_lo, const double* dPdy_hi, const double* P,
                   const double* Uh, const double* Vh, const double* Wh,
                   const double* wall, double* U, double* V, double* W, int nthreads);

/* max |div u| over the interior, mod_get_bulk.f90:94-116 (U, V, W halo'd,
 * halos already filled). */
double orc_div_maxabs(int nx, int nz, int ny, double dx, double dz,
                      const double* inv_dy_p, const double* U, const double* V,
                      const double* W, int nthreads);

/* divergence -> Poisson solve -> correction.  P (nx*nz*ny) receives the pressure. */
int orc_projection(int nx, int nz, int ny, double dx, double dz, double dt,
                   const double* a, const double* b, const double* c,
                   const double* a00, const double* b00, const double* c00,
                   const double* inv_dy_p, const double* dPdy_lo, const double* dPdy_hi,
                   const double* Uh, const double* Vh, const double* Wh, const double* wall,
                   double* U, double* V, double* W, double* P, int nthreads);

/* Halfcomplex real transforms (FFTW R2HC / HC2R semantics, unnormalised),
 * exposed so the tests can pin them against numpy's FFT. */
int orc_r2hc(int n, const double* x, double* hc);
int orc_hc2r(int n, const double* hc, double* x);

/* Variable-density pressure splitting (use_incompressible = .false.).
 *   orc_rho_min            min of rho over the interior, mod_cfd_subroutines.f90:476-486
 *   orc_vd_metric_from_yu  inv_dy_p_pad (ny+1 entries), calc_bands.py:273, :276
 *   orc_vd_rhs             RHS of the constant-coefficient Poisson equation, MCS:538-573:
 *                          rho_min/dt (div u_hat - div_now) + the density-weighted
 *                          Laplacian of Ps = 2 P_now - P_old (caller-filled halos of rho,
 *                          P_now, P_old are read as given)
 *   orc_vd_correction      u = u_hat - dt grad(P/rho_min + (1/rho - 1/rho_min) Ps),
 *                          MCS:1153-1197, with the boundary fill :1223-1243; P_next
 *                          receives P_per (MCS:1087-1118), the caller's next P_now
 *   orc_projection_vd      the three in sequence around orc_poisson
 * rho, P_now, P_old, div_now, P_next are halo'd. */
double orc_rho_min(int nx, int nz, int ny, const double* rho, int nthreads);
int orc_vd_metric_from_yu(int ny, const double* yu, double* inv_dy_p_pad);
int orc_vd_rhs(int nx, int nz, int ny, double dx, double dz, double dt,
               const double* inv_dy_p, const double* inv_dy_p_pad,
               const double* Uh, const double* Vh, const double* Wh, double vbot, double vtop,
               const double* rho, const double* P_now, const double* P_old, const double* div_now,
               double rho_min, double* P, int nthreads);
int orc_vd_correction(int nx, int nz, int ny, double dx, double dz, double dt,
                      const double* dPdy_lo, const double* dPdy_hi, const double* P,
                      const double* Uh, const double* Vh, const double* Wh, const double* wall,
                      const double* rho, const double* P_now, const double* P_old, double rho_min,
                      double* U, double* V, double* W, double* P_next, int nthreads);
int orc_projection_vd(int nx, int nz, int ny, double dx, double dz, double dt,
                      const double* a, const double* b, const double* c,
                      const double* a00, const double* b00, const double* c00,
                      const double* inv_dy_p, const double* dPdy_lo, const double* dPdy_hi,
                      const double* inv_dy_p_pad, const double* Uh, const double* Vh, const double* Wh,
                      const double* wall, const double* rho, const double* P_now, const double* P_old,
                      const double* div_now, double* U, double* V, double* W, double* P, double* P_next,
                      double* rho_min_out, int nthreads);

#ifdef __cplusplus
}
#endif
#endif

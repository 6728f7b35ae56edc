/*
 * projection.h -- C ABI of the B200 pressure-projection engine.
 *
 * The engine replaces, on one GPU, the pressure projection of the channel DNS
 * Rafael10Diez/DNS-Supercritical-IBM: the predictor divergence, the FFT-based
 * pressure Poisson solve (periodic x and z, Neumann walls in y, stretched y
 * grid, pinned kx = kz = 0 mode) and the velocity correction.
 *
 * Conventions (identical to the reference's Fortran arrays):
 *   - arrays are column-major with x fastest: P(i=x, j=z, k=y);
 *   - P has shape (nx, nz, ny)                        (alloc_poisson_solver_multigpu.f90:40);
 *   - halo'd velocity fields have shape (nx+2, nz+2, ny+2) and cover
 *     (-1:nx, -1:nz, -1:ny)                           (inc_set_alloc_arrays.f90:93-101);
 *   - band arrays and 1-D metrics have ny entries, row k of the wall-normal
 *     tridiagonal / metric of cell or face k          (inc_set_alloc_arrays.f90:51-61).
 * Device pointers are raw CUDA device addresses; streams are cudaStream_t
 * passed as void* (NULL = the legacy default stream).
 *
 * Every function returns PRJ_OK (0) or a negative status; none aborts the
 * process.  prj_last_error_string() describes the last failure of the calling
 * thread.
 */
#ifndef PRJ_PROJECTION_H
#define PRJ_PROJECTION_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum prj_status {
    PRJ_OK = 0,
    PRJ_ERR_ARG = -1,        /* bad size, pointer or flag */
    PRJ_ERR_UNSUPPORTED = -2,/* valid request the engine does not implement */
    PRJ_ERR_CUDA = -3,       /* a CUDA runtime call failed */
    PRJ_ERR_OOM = -4,        /* device allocation failed or budget exceeded */
    PRJ_ERR_NUMERIC = -5,    /* zero pivot, NaN or refinement that did not converge */
    PRJ_ERR_TIMEOUT = -6,    /* a bounded device-side wait gave up */
    PRJ_ERR_STATE = -7       /* call out of order (e.g. destroyed plan) */
};

/* plan flags */
#define PRJ_FLAG_NONE 0u

/* precision modes of prj_projection_step */
#define PRJ_MODE_FP64 0            /* plain FP64 path: the drop-in */
#define PRJ_MODE_FP32_REFINE 1     /* FP32 spectral work + FP64 iterative refinement */
/* or-ed into prj_batch_create's mode: the CUDA-graph form where the persistent kernel applies */
#define PRJ_BATCH_GRAPH 0x10

typedef struct prj_plan prj_plan;

/* Result record of one projection step. */
typedef struct prj_stats {
    double div_maxabs;      /* max |div u| after the correction (mod_get_bulk.f90:94-116); -1 if not computed */
    double p_maxabs;        /* max |P| */
    double min_pivot;       /* min |pivot| of the Thomas factorisation (min_abs_div_bacp, PSM:181-222) */
    int refine_iters;       /* refinement iterations used (0 for FP64) */
    int fp64_lines;         /* spectral lines solved in FP64 by the mixed path */
    double last_update_rel; /* rel-L2 of the last refinement update (mixed path) */
    double rho_min;         /* variable-density step: min rho over the interior (MCS:476-486); else 0 */
} prj_stats;

/* Scalars of one projection step (update_vars / build_vars arguments). */
typedef struct prj_step_params {
    double dt;              /* dtmax: P = (1/dt) div(u_hat); u = u_hat - dt grad P */
    double wall_U_bot, wall_V_bot, wall_W_bot;  /* wall_BC_*_bot */
    double wall_U_top, wall_V_top, wall_W_top;  /* wall_BC_*_top */
    int compute_stats;      /* nonzero: fill prj_stats.div_maxabs / p_maxabs */
} prj_step_params;

/*
 * Create a solver plan on `device` for an nx x nz x ny grid.
 * Replaces init_spec_poisson_multigpu (poisson_solver_multigpu.f90:33-326)
 * for mpi_divs_z = mpi_divs_y = 1: builds the FFT plans (:77-129), the
 * a_x / a_z / poi_is_00 tables (:133-155) and the Thomas pivot table that
 * takes the place of poi_C (:164-179), and records min_abs_div_bacp (:181-222).
 *   band_*     P_band_a/b/c      (ny)  bands of all non-(0,0) modes
 *   band_*00   P_band_a/b/c_00   (ny)  bands of the pinned (0,0) mode
 *   inv_dy_p   (ny)   1/(yu(k+1)-yu(k))          (divergence, MCS:534)
 *   dPdy_lo/hi (ny)   dPdy_ddy_lo/hi rows 0..ny-1 (correction, MCS:1148-1149);
 *              these three may be NULL for a Poisson-only plan.
 * Limits: 1 <= nx <= 8192, 1 <= nz <= 4094, 2 <= ny <= 65536; every prime
 * factor of nz and of nx (nx/2 for even nx) is at most 64.
 */
int prj_plan_create(int nx, int nz, int ny, double dx, double dz,
                    const double* band_a, const double* band_b, const double* band_c,
                    const double* band_a00, const double* band_b00, const double* band_c00,
                    const double* inv_dy_p, const double* dPdy_lo, const double* dPdy_hi,
                    unsigned flags, int device, prj_plan** out);

/* Release every device buffer of the plan.  Replaces
 * dealloc_poisson_solver_multigpu.f90:1-39.  NULL is accepted. */
int prj_plan_destroy(prj_plan* plan);

/*
 * FP64 Poisson solve in place on a device array P (nx, nz, ny): the RHS on
 * entry, the solution on exit.  Drop-in for run_spec_poisson_multigpu
 * (poisson_solver_multigpu.f90:328-554) with mpi_divs_y = 1: forward FFTs,
 * per-line Thomas with the pinned (0,0) mode, inverse FFTs, 1/(nx nz).
 * Asynchronous on `stream`.
 */
int prj_poisson_fp64(prj_plan* plan, double* d_P, void* stream);

/*
 * One pressure projection on device arrays: P = (1/dt) div(u_hat)
 * (mod_cfd_subroutines.f90:504-537), Poisson solve, and
 * u = u_hat - dt grad P with the boundary fill of update_vars
 * (mod_cfd_subroutines.f90:1086-1152, :1223-1243).  Uh, Vh, Wh (inputs) and
 * U, V, W (outputs) are halo'd; only interior input values are read (x and z
 * wrap periodically, V_hat at the walls is wall_V_bot / wall_V_top).  The
 * outputs are written everywhere, halos included.  P (nx, nz, ny) receives
 * the pressure.  `mode` is PRJ_MODE_FP64 or PRJ_MODE_FP32_REFINE.  `stats`
 * may be NULL; when non-NULL (or compute_stats is set) the call synchronises
 * `stream` to return the record.
 */
int prj_projection_step(prj_plan* plan, const double* d_Uh, const double* d_Vh, const double* d_Wh,
                        double* d_U, double* d_V, double* d_W, double* d_P,
                        const prj_step_params* params, int mode, prj_stats* stats, void* stream);

/* Host-buffer form of prj_poisson_fp64: copies P to the device, solves, and
 * copies the solution back (synchronous).  For callers that hold host arrays,
 * like the reference's FFTW build. */
int prj_poisson_fp64_host(prj_plan* plan, double* h_P);

/* Host-buffer form of prj_projection_step (synchronous, copies included). */
int prj_projection_step_host(prj_plan* plan, const double* h_Uh, const double* h_Vh, const double* h_Wh,
                             double* h_U, double* h_V, double* h_W, double* h_P,
                             const prj_step_params* params, int mode, prj_stats* stats);

/*
 * Pipelined form of prj_projection_step_host for a sequence of steps from host
 * memory: the call only enqueues (no statistics) and returns.  Two device staging
 * slots alternate, and the copy-in, the solve and the copy-out run on three
 * plan-owned streams ordered by events, so the device-to-host copy of one step
 * overlaps the host-to-device copy of the next on the two copy engines.  The host
 * buffers of a step must stay valid and untouched until prj_host_async_wait
 * returns (or, for the inputs, until two later steps were enqueued); use pinned
 * host memory, as pageable memory makes the copies synchronous.
 */
int prj_projection_step_host_async(prj_plan* plan, const double* h_Uh, const double* h_Vh, const double* h_Wh,
                                   double* h_U, double* h_V, double* h_W, double* h_P,
                                   const prj_step_params* params, int mode);
int prj_host_async_wait(prj_plan* plan);

/*
 * Poisson solve in place with FP32 spectral storage and FP64 iterative
 * refinement (the precision scheme of PRJ_MODE_FP32_REFINE): rows of
 * x-wavenumbers whose tridiagonals are badly conditioned stay FP64, the
 * residual b - A p of the pinned operator is formed in FP64.  One refinement
 * pass by default (the tuning's mixed_iters).  Needs in-place transform plans
 * (radices 2, 3, 4, 5, 6, 8 for nx/2 and nz).  Asynchronous.
 */
int prj_poisson_mixed(prj_plan* plan, double* d_P, void* stream);

/*
 * Variable-density projection (the reference's use_incompressible = .false.
 * branch).  The Poisson operator is the plan's constant-coefficient one; the
 * right-hand side is MCS:538-573 and the correction MCS:1153-1197 (MCS =
 * src/mod_cfd_subroutines.f90):
 *   rho_min = min rho over the interior,
 *   RHS     = rho_min/dt (div u_hat - div_now) + the density-weighted Laplacian
 *             of Ps = 2 P_now - P_old,
 *   u       = u_hat - dt grad(P/rho_min + (avg 1/rho - 1/rho_min) Ps).
 * rho, P_now, P_old and div_now are device arrays in the halo'd layout with
 * their halos filled by the caller (periodic x/z images, wall ghost planes),
 * read as given.  P_next (halo'd, device) receives the new pressure with
 * periodic halos and wall ghost planes P(-1) = P(0), P(ny) = P(ny-1) (P_per,
 * MCS:1087-1118): the caller's next P_now.  The reference copies P_now to
 * P_old and P_per to P_now after each step (MCS:1199-1221); callers of this
 * function rotate the three pointers instead.  No output may alias an input.
 * Needs inv_dy_p_pad (ny+1 entries, calc_bands.py:273-276; built by
 * prj_vd_metric_from_yu) set once per plan with prj_plan_set_vd_metric.
 */
typedef struct prj_vd_fields {
    const double* rho;
    const double* P_now;
    const double* P_old;
    const double* div_now;
    double* P_next;
} prj_vd_fields;
int prj_vd_metric_from_yu(int ny, const double* yu, double* inv_dy_p_pad);
int prj_plan_set_vd_metric(prj_plan* plan, const double* inv_dy_p_pad);
int prj_projection_step_vd(prj_plan* plan, const double* d_Uh, const double* d_Vh, const double* d_Wh,
                           double* d_U, double* d_V, double* d_W, double* d_P, const prj_step_params* params,
                           const prj_vd_fields* vd, int mode, prj_stats* stats, void* stream);

/*
 * Immersed-boundary forcing of the predictor before the projection (rough-wall
 * runs, src/mod_cfd_subroutines.f90:411-426), in place on the halo'd device
 * fields.
 *
 * prj_rough_force: ibm_part_2 (src/ibm_setup/mod_cfd_ibm.f90:47-131).  For each
 * column (i, j) (index c = i + nx j of the int32 device arrays): cells
 * k = 0..bot[c] take the bottom wall value, k = top[c]..ny-1 the top one (v:
 * k = top[c]..ny, up to the top wall face).  bot = -1 / top = ny force nothing.
 *
 * prj_ibm_interp: the interpolated forcing points of diezdecomp_ibm_exec on one
 * rank (src/diezdecomp_api_ibm.f90:374-424) for one field A of `len` elements:
 * A[pos_i] = c1_i A[src1_i] + c2_i A[src2_i] + c0_i for i < n, every source read
 * before any point is written, then A[dst_j] = A[src_j] for j < ncopy.  Offsets
 * are elements of the halo'd array.  d_scratch holds 2 n + 1 doubles.  An offset
 * outside [0, len) is skipped and reported as PRJ_ERR_ARG; the call synchronises
 * `stream`.
 */
typedef struct prj_rough_inds {
    const int* U_bot;
    const int* U_top;
    const int* V_bot;
    const int* V_top;
    const int* W_bot;
    const int* W_top;
} prj_rough_inds;
int prj_rough_force(int nx, int nz, int ny, double* d_Uh, double* d_Vh, double* d_Wh, const prj_rough_inds* inds,
                    const prj_step_params* walls, void* stream);
int prj_ibm_interp(double* d_A, long long len, int n, const long long* d_pos, const long long* d_src1,
                   const long long* d_src2, const double* d_c0, const double* d_c1, const double* d_c2, int ncopy,
                   const long long* d_dst, const long long* d_src, double* d_scratch, void* stream);

/*
 * Field files of the reference (src/mod_io.f90:7-149, cfd_read_arr /
 * cfd_write_arr: array_ini_*.dat, end/array_end_*.dat): stream-unformatted,
 * three 4-byte integers nx, nz, ny, then the nx*nz*ny interior values as
 * float64, x fastest, then z, then y.  `halo` = 0: the array is (nx, nz, ny);
 * halo = 1: it is halo'd (nx+2, nz+2, ny+2) and only its interior is read or
 * written (halos untouched).  Reads fail with PRJ_ERR_ARG when the file's grid
 * differs from (nx, nz, ny) (the reference stops there, mod_io.f90:27-33).
 * The device forms stage y-plane chunks through pinned host memory and overlap
 * the file transfer with the copies; they first wait for the device's pending
 * work and return when the transfer is complete.
 */
int prj_field_read_header(const char* path, int* nx, int* nz, int* ny);
int prj_field_read(const char* path, int nx, int nz, int ny, double* h_dst, int halo);
int prj_field_write(const char* path, int nx, int nz, int ny, const double* h_src, int halo);
int prj_field_read_device(const char* path, int nx, int nz, int ny, double* d_dst, int halo, int device);
int prj_field_write_device(const char* path, int nx, int nz, int ny, const double* d_src, int halo, int device);

/*
 * Geometry folder of a reference case (the geom_data files that
 * src/pycode/calc_bands.py writes, calc_bands.py:358-364: first line the row
 * count, then one row of space-separated values per line).  Host only.
 *
 * prj_geom_read_column: read_column_r8 (src/mod_utils.f90:14-35): rows
 *   n_prev .. n_prev+n-1 of column icol (0..3) into out[0..n-1]; PRJ_ERR_ARG when
 *   that range runs past the row count (the reference stops there).
 * prj_geom_read_bands: P_band_a/b/c from P_band_abc.dat and the pinned-mode bands
 *   from P_band_abc_00.dat, rows 0..ny-1 (src/inc_set_alloc_arrays.f90:54-59),
 *   the band_* arguments of prj_plan_create.
 * prj_geom_read_metrics: inv_dy_p (inv_dy_p.dat) and dPdy_ddy_lo/hi (columns 0
 *   and 1 of dPdy_ddy_lh.dat), rows 0..ny-1 (inc_set_alloc_arrays.f90:51-53, :61).
 * prj_geom_read_base_params: the records of base_params.txt this path needs
 *   (src/inc_set_read_params.f90:14-40): the grid, nstep, dtmax, dx, dz, the
 *   rough-surface flag, the wall values of U, V, W and use_incompressible.
 */
typedef struct prj_case_params {
    int nx, nz, ny;
    int use_rough_surf;
    long long nstep;
    double dtmax;
    double dx, dz;
    double wall_U_bot, wall_V_bot, wall_W_bot;
    double wall_U_top, wall_V_top, wall_W_top;
    int use_incompressible;
} prj_case_params;
int prj_geom_read_column(const char* path, int icol, int n, int n_prev, double* out);
int prj_geom_read_bands(const char* geom_dir, int ny, double* band_a, double* band_b, double* band_c,
                        double* band_a00, double* band_b00, double* band_c00);
int prj_geom_read_metrics(const char* geom_dir, int ny, double* inv_dy_p, double* dPdy_lo, double* dPdy_hi);
int prj_geom_read_base_params(const char* path, prj_case_params* out);

/*
 * Batched solves: case i solves plans[i] in place on the device array d_P[i].
 * The plans must be distinct (a plan's scratch serves one solve at a time) and
 * outlive the batch; the arrays are bound at creation; the plans' tuning must not
 * change while the batch exists.  No counterpart in the reference, which solves
 * one grid per run (and plans it once, poisson_solver_multigpu.f90:77-129).
 *   FP64, every case with even nx, nx/2 and nz among the pass-plan lengths up to
 *   256 (16, 24, 32, 48, 64, 96, 128, 192, 256) and a 16-byte aligned array: one
 *   persistent kernel runs all
 *   cases from a work queue of (case, stage, tile) items in stage-major order
 *   (forward x transform, the fused z solve of each x wavenumber, inverse x
 *   transform), with bounded waits on per-case stage counters; prj_batch_launch
 *   issues a counter reset and that one kernel (both capturable in a CUDA graph).
 *   Otherwise (FP32 + refinement, other lengths, or mode | PRJ_BATCH_GRAPH): one
 *   CUDA graph holding every case's kernels on parallel branches, replayed by one
 *   graph launch.
 * Each case's P equals its own prj_poisson_fp64 / prj_poisson_mixed bit for bit.
 * prj_batch_info: whether the batch is persistent, its kernel launches per
 * prj_batch_launch, and its work items.  prj_batch_check_error waits for
 * `stream`, returns PRJ_ERR_TIMEOUT if a bounded wait of the persistent kernel
 * gave up since the last check (that launch's results are not valid), and clears
 * the word.
 */
typedef struct prj_batch prj_batch;
int prj_batch_create(prj_plan* const* plans, double* const* d_P, int ncases, int mode, prj_batch** out);
int prj_batch_launch(prj_batch* batch, void* stream);
int prj_batch_info(const prj_batch* batch, int* persistent, int* kernels_per_launch, long long* work_items);
int prj_batch_check_error(prj_batch* batch, void* stream);
int prj_batch_destroy(prj_batch* batch);

/*
 * Tuning of a plan: launch shapes and kernel choices (read by the autotuner,
 * which times candidates and caches the winner per grid size), and the
 * parameters of the mixed path.  Every knob is a plan field: the launchers read
 * nothing else.
 *   x_rows      x-rows per CTA of the x-transform kernels (power of two, 1..16);
 *   z_rows      spectral rows per CTA of the split z-transform kernels (0 = default,
 *               else a power of two, 1..16);
 *   z_mode      0 = z FFT / Thomas / inverse z FFT as three kernels, 1 = one fused
 *               pipelined kernel per x wavenumber (runtime radices; the kernel of z
 *               lengths with a prime factor above 5), 2 = its unpipelined form,
 *               3 = one kernel per x wavenumber on the compile-time pass plans (the
 *               three kernels where nz has no pass plan).  The default is 3 when
 *               nx/2+1 >= 2 x the SM count, else 0;
 *   z_planes    planes per chunk of the per-wavenumber z kernels (0 = default);
 *   z_stages    stages of their copy rings (0 = default, else 2..4; 2..8 for mode 1);
 *   thomas_ring shared-memory ring of the split Thomas kernel: -1 = default (the
 *               mixed storage only), 0 = none, 1..4 = shapes 4x4, 8x2, 2x8, 8x3
 *               (planes x stages) for both storages;
 *   mixed_iters refinement passes of PRJ_MODE_FP32_REFINE (default 1, 0..8);
 *   mixed_tau   x-wavenumber rows with |a_x| < mixed_tau max|b| keep FP64 storage in
 *               the mixed path (default 1e-3; must lie in (0, 1));
 *   x_order,    radix order of the in-place x (length nx/2) and z (length nz)
 *   z_order     transforms: 0 = the default pass plan, k >= 1 = the k-th other compiled
 *               order of that length (64: 4x4x4; 96: 8x6x2; 128: 8x8x2; 192: 6x4x8;
 *               256: 4x8x8, 8x8x4; 384: 8x6x8, 8x8x6).  Orders round differently (each
 *               within the parity bounds); a given order gives the same bits in every
 *               kernel family.  Changing an order rebuilds the transform's tables.
 * prj_plan_set_tuning rejects values out of range and shapes that do not fit
 * shared memory; it may free and later reallocate the mixed path's FP32 spectrum
 * (after a change of mixed_tau), so call it outside stream capture.  The library
 * reads no environment variable.
 */
typedef struct prj_tuning {
    int x_rows;
    int z_rows;
    int z_mode;
    int z_planes;
    int z_stages;
    int thomas_ring;
    int mixed_iters;
    double mixed_tau;
    int x_order;
    int z_order;
} prj_tuning;
int prj_plan_get_tuning(const prj_plan* plan, prj_tuning* out);
int prj_plan_set_tuning(prj_plan* plan, const prj_tuning* tuning);

/* Diagnostic of the bounded device-side waits of the pipelined kernels: one
 * kernel waits, for at most budget_cycles SM clock cycles, on an mbarrier that
 * nothing arrives on, gives up, and reports it.  Returns PRJ_ERR_TIMEOUT when the
 * wait gave up as designed (the context stays usable), PRJ_OK if it unexpectedly
 * completed.  No fault, trap or unbounded wait is involved. */
int prj_selftest_wait_timeout(int device, long long budget_cycles);

/* Diagnostic of the division the Thomas forward sweeps use: n pseudo-random pairs
 * (u, D) from `seed` -- half with u within 2^+-200 and D within 2^+-40 of 1, a quarter
 * with u anywhere in the double range (zeros, subnormals, infinities and NaNs
 * included), a quarter with quotients near the bounds of the fast path's exponent
 * window; D always within the pivot range [2^-40, 2^1000] that plan creation enforces;
 * random and edge mantissas -- each divided both by __ddiv_rn and by the
 * reciprocal-and-correction form of div_rn.cuh; *mismatches counts the pairs whose two results differ in any bit
 * (the first such pair in first_u, first_d when not NULL).  No counterpart in the
 * reference. */
int prj_selftest_division(int device, long long n, unsigned long long seed, long long* mismatches,
                          double* first_u, double* first_d);

/* Kernel launches one prj_projection_step of `mode` issues with the plan's current
 * configuration (statistics excluded). */
int prj_plan_schedule(const prj_plan* plan, int mode, int* launches);

/* band modes of prj_bands_from_yu */
#define PRJ_BANDS_REFERENCE 0   /* the reference's mk_P_abc bands */
#define PRJ_BANDS_CONSISTENT 1  /* bands of div(grad p) with the divergence/correction metrics */

/*
 * Wall-normal bands from the face coordinates yu (ny+1 values, increasing).
 * PRJ_BANDS_REFERENCE restates mk_P_abc (src/pycode/calc_bands.py:181-201) on
 * yp_ext = [yu_0, yp_0 .. yp_{ny-1}, yu_ny] (calc_bands.py:226-227); the _00
 * arrays are its is_dirich_first variant (the pinned (0,0) mode).
 * PRJ_BANDS_CONSISTENT gives a_k = inv_dy_p(k)/(yp_k - yp_{k-1}),
 * c_k = inv_dy_p(k)/(yp_{k+1} - yp_k), b_k = -(a_k + c_k), a_0 = c_{ny-1} = 0,
 * so that the discrete Laplacian equals div(grad p) of the divergence and
 * correction stencils; its pinned variant subtracts the same mirrored-ghost
 * term from b_0.  Host-only (no GPU needed).
 */
int prj_bands_from_yu(int ny, const double* yu, int mode, double* a, double* b, double* c,
                      double* a00, double* b00, double* c00);

/* 1-D metrics from yu: inv_dy_p (calc_bands.py:274) and rows 0..ny-1 of
 * dPdy_ddy_lh (calc_bands.py:336-343).  Host-only. */
int prj_metrics_from_yu(int ny, const double* yu, double* inv_dy_p, double* dPdy_lo, double* dPdy_hi);

/* min_abs_div_bacp of the plan (poisson_solver_multigpu.f90:181-222). */
int prj_plan_min_pivot(const prj_plan* plan, double* out);

/* Device bytes the plan holds (for HBM-budget admission). */
int prj_plan_device_bytes(const prj_plan* plan, size_t* out);

/*
 * Per-kernel device timing (diagnostics; no counterpart in the reference,
 * which only prints wall time per iteration, mod_get_bulk.f90:174-175).
 * While enabled, every call records CUDA events around each kernel on the
 * caller's stream.  prj_plan_stage_times synchronises those events, writes
 * the summed milliseconds and launch counts per stage (index = stage id, up
 * to max_stages entries), sets *n_stages and clears the record.
 */
int prj_plan_enable_stage_timing(prj_plan* plan, int enable);
int prj_plan_stage_times(prj_plan* plan, double* ms, int* launches, int max_stages, int* n_stages);
/* Kernel name of a stage id ("" if unknown). */
const char* prj_stage_name(int stage);

/*
 * FP64 Poisson solve for callers that cannot allocate device memory.
 * No counterpart in the reference (there, Fortran allocates every array up
 * front, alloc_poisson_solver_multigpu.f90:39-64); it serves host programs
 * whose device memory is owned elsewhere (an OpenACC/Fortran runtime, a time
 * loop under a memory cap, code that must not call cudaMalloc, which may
 * synchronise the device).  Same arguments and result as prj_plan_create
 * followed by prj_poisson_fp64 (bands are host arrays of ny values, d_P is the
 * device array (nx, nz, ny), solved in place), but it allocates nothing: all
 * scratch (tables, pivots, spectrum) lives in one static device array of
 * PRJ_NOALLOC_SCRATCH_BYTES that every GPU using the library holds until the
 * process exits.  Grids whose scratch exceeds that size are rejected with
 * PRJ_ERR_ARG (roughly 10 bytes per grid point: about 6.5e6 points at most;
 * 256 x 128 x 128 fits).
 * The first call on a device resolves the array's address on that device
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * The function is synchronous: before it returns it waits for `stream` and
 * reads back the minimum pivot and the error word of the z solve's bounded
 * device waits (PRJ_ERR_TIMEOUT when one gave up; P is then not solved).
 * Calls share the array and each finds what the previous one left, so every
 * region it reads, the error word included, is re-initialised first; calls are
 * serialised with a process lock, and work that overlapped on the GPU with
 * another user of the array would race.
 */
#define PRJ_NOALLOC_SCRATCH_BYTES ((size_t)64 << 20)
int prj_poisson_fp64_noalloc(int nx, int nz, int ny, double dx, double dz,
                             const double* band_a, const double* band_b, const double* band_c,
                             const double* band_a00, const double* band_b00, const double* band_c00,
                             double* d_P, void* stream);

/* One FP64 Poisson solve spread over several GPUs (one rank per GPU, each with a
 * plan of the whole grid on its own device).  Replaces the multi-rank form of
 * run_spec_poisson_multigpu (poisson_solver_multigpu.f90:328-554 with
 * mpi_divs_z x mpi_divs_y > 1, whose diezDecomp transposes tr_poi_xy / tr_poi_yx
 * move the spectrum between ownerships).  Rank r owns the y planes [y0, y1) of P
 * for the transforms and the x wavenumbers [kx_bounds[r], kx_bounds[r+1]) for the
 * Thomas lines; the caller moves the spectrum between the two with an all-to-all
 * (dns-supercritical-ibm_b200/prj_dist.py does it over torch.distributed / NCCL).
 * The y ranges ascend with the rank and tile [0, ny); kx_bounds[0] = 0 and
 * kx_bounds[nranks] = nx/2+1.  Needs a z length with a compile-time pass plan and
 * an x length of radices 2, 3, 4, 5, 6, 8.
 * All calls are asynchronous on `stream`.  Spectrum values are complex FP64
 * (two doubles).
 *   prj_dist_forward  forward x and z transforms of the planes [y0, y1); d_P_local
 *                     holds those planes, (y1-y0) x nz x nx values, x fastest.
 *   prj_dist_pack     the planes' spectrum as blocks for the destinations q,
 *                     q-major: [q][y - y0][kx - kx_bounds[q]][z].
 *   prj_dist_thomas   Thomas sweeps of the lines kx0 .. kx1-1 held in d_lines as
 *                     [y][kx - kx0][z] over all ny planes (the blocks received
 *                     from all ranks, in rank order).
 *   prj_dist_unpack   the blocks received back (layout of prj_dist_pack) into the
 *                     planes' spectrum.
 *   prj_dist_inverse  inverse z and x transforms of the planes into d_P_local.
 * The assembled P equals prj_poisson_fp64's on one GPU bit for bit. */
int prj_dist_forward(prj_plan* plan, const double* d_P_local, int y0, int y1, void* stream);
int prj_dist_pack(prj_plan* plan, int y0, int y1, const int* kx_bounds, int nranks, double* d_send, void* stream);
int prj_dist_thomas(prj_plan* plan, double* d_lines, int kx0, int kx1, void* stream);
int prj_dist_unpack(prj_plan* plan, int y0, int y1, const int* kx_bounds, int nranks, const double* d_recv,
                    void* stream);
int prj_dist_inverse(prj_plan* plan, double* d_P_local, int y0, int y1, void* stream);
/* The projection step over ranks (the plan made with metrics, as for
 * prj_projection_step): prj_dist_divergence takes the place of prj_dist_forward
 * (the divergence of the predictor, then the forward x and z transforms of the
 * planes [y0, y1)), and prj_dist_correct follows prj_dist_inverse.  The halo'd local
 * arrays hold the halo'd planes y0 .. y1+1 (global planes y0-1 .. y1, ghost planes
 * filled by the caller's halo exchange), (nx+2) x (nz+2) x (y1-y0+2) values, x
 * fastest.  d_P_ext holds the P planes y0-1 .. y1-1: plane y0-1 from the rank below
 * (not read on the first rank), then the rank's own planes as prj_dist_inverse left
 * them.  prj_dist_correct writes the rank's planes of U, V, W with their periodic
 * x/z halos, and the wall planes on the first and last ranks. */
int prj_dist_divergence(prj_plan* plan, const double* d_Uh_loc, const double* d_Vh_loc, const double* d_Wh_loc,
                        int y0, int y1, const prj_step_params* params, void* stream);
int prj_dist_correct(prj_plan* plan, const double* d_P_ext, const double* d_Uh_loc, const double* d_Vh_loc,
                     const double* d_Wh_loc, double* d_U_loc, double* d_V_loc, double* d_W_loc, int y0, int y1,
                     const prj_step_params* params, void* stream);

/* Device error word of the plan's bounded device-side waits (the pipelined z
 * kernel used for z lengths with a prime factor above 5, and the diagnostics).
 * The asynchronous solves cannot report a wait that gave up when they return;
 * this call waits for `stream`, reads the word, clears it, and returns
 * PRJ_ERR_TIMEOUT if any wait gave up since the last check (the results of
 * that work are then not valid), else PRJ_OK.  prj_projection_step with
 * statistics performs the same check. */
int prj_plan_check_error(prj_plan* plan, void* stream);

/* Synthetic channel predictor on the device, for benchmarks, tests and served
 * requests that name their field by a seed (no counterpart in the reference, whose
 * predictor comes from its momentum step): on the interior of the halo'd arrays
 * u_hat = 1.5 (1 - (yp_k - 1)^2) + sigma n, v_hat = sigma n, w_hat = sigma n, and
 * v_hat = 0 on the bottom wall face k = 0, with yp (ny values, device) the cell
 * centres and n standard normals that are a fixed function of (seed, field, point)
 * (a counter hash and one single-precision Box-Muller step, stored as doubles).
 * Halos are not written.  Asynchronous on `stream`. */
int prj_synth_channel_predictor(int nx, int nz, int ny, const double* d_yp, unsigned long long seed, double sigma,
                                double* d_Uh, double* d_Vh, double* d_Wh, void* stream);

/* Message of the calling thread's last failure ("" if none). */
const char* prj_last_error_string(void);

/* Engine version string. */
const char* prj_version(void);

#ifdef __cplusplus
}
#endif
#endif /* PRJ_PROJECTION_H */

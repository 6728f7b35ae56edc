/*
 * prj_oracle.c -- CPU oracle for the pressure projection (TEST INFRASTRUCTURE).
 *
 * A plain-C restatement of the reference's FFTW code path; see prj_oracle.h for
 * the list of reference lines each function follows.  It is used by the tests
 * as the checker and by the benchmark as the timed CPU baseline ("port").  The
 * CUDA engine never calls it.
 */
#include "prj_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define HIDX(i, j, k) ((size_t)((i) + 1) + (size_t)(nx + 2) * ((size_t)((j) + 1) + (size_t)(nz + 2) * (size_t)((k) + 1)))
#define PIDX(i, j, k) ((size_t)(i) + (size_t)nx * ((size_t)(j) + (size_t)nz * (size_t)(k)))

static void set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

/* ------------------------------------------------------------------------- */
/* Mixed-radix complex FFT (textbook recursive Cooley-Tukey, decimation in    */
/* time).  X_k = sum_j x_j exp(sign * 2 pi i j k / n), unnormalised.          */
/* ------------------------------------------------------------------------- */

typedef struct {
    int n;
    int nfac;
    int fac[64];
    double* twr; /* cos(2 pi k / n) */
    double* twi; /* sin(2 pi k / n) */
} cfft_plan;

static int cfft_init(cfft_plan* p, int n) {
    p->n = n;
    p->nfac = 0;
    int m = n;
    while (m % 4 == 0) { p->fac[p->nfac++] = 4; m /= 4; }
    while (m % 2 == 0) { p->fac[p->nfac++] = 2; m /= 2; }
    for (int f = 3; m > 1; f += 2) {
        while (m % f == 0) { p->fac[p->nfac++] = f; m /= f; }
        if ((long)f * f > m && m > 1) { p->fac[p->nfac++] = m; m = 1; }
    }
    p->twr = (double*)malloc(sizeof(double) * (size_t)n);
    p->twi = (double*)malloc(sizeof(double) * (size_t)n);
    if (!p->twr || !p->twi) return -1;
    for (int k = 0; k < n; k++) {
        long double ang = 2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)n;
        p->twr[k] = (double)cosl(ang);
        p->twi[k] = (double)sinl(ang);
    }
    return 0;
}

static void cfft_free(cfft_plan* p) {
    free(p->twr);
    free(p->twi);
}

/* out[0..n-1] = DFT_n of in[0], in[s], ..., in[(n-1)s] */
static void cfft_rec(const cfft_plan* P, const double* xr, const double* xi, size_t s,
                     double* yr, double* yi, int n, const int* fac, int sign, double* tmp) {
    if (n == 1) { yr[0] = xr[0]; yi[0] = xi[0]; return; }
    const int p = fac[0];
    const int m = n / p;
    for (int r = 0; r < p; r++)
        cfft_rec(P, xr + (size_t)r * s, xi + (size_t)r * s, s * (size_t)p, yr + (size_t)r * m, yi + (size_t)r * m, m, fac + 1, sign, tmp);
    const int N = P->n;
    const int tstep = N / n;
    double* tr = tmp;
    double* ti = tmp + p;
    for (int k = 0; k < m; k++) {
        for (int r = 0; r < p; r++) {
            double ar = yr[(size_t)r * m + k], ai = yi[(size_t)r * m + k];
            long e = ((long)r * k * tstep) % N;
            double wr = P->twr[e], wi = sign * P->twi[e];
            tr[r] = ar * wr - ai * wi;
            ti[r] = ar * wi + ai * wr;
        }
        for (int q = 0; q < p; q++) {
            double accr = 0.0, acci = 0.0;
            for (int r = 0; r < p; r++) {
                long e = ((long)((r * q) % p)) * (N / p);
                double wr = P->twr[e], wi = sign * P->twi[e];
                accr += tr[r] * wr - ti[r] * wi;
                acci += tr[r] * wi + ti[r] * wr;
            }
            yr[(size_t)k + (size_t)q * m] = accr;
            yi[(size_t)k + (size_t)q * m] = acci;
        }
    }
}

/* per-thread work space for one line transform */
typedef struct {
    double* xr; double* xi; double* yr; double* yi; double* tmp;
} cfft_work;

static int work_init(cfft_work* w, int n) {
    w->xr = (double*)malloc(sizeof(double) * (size_t)(6 * n + 2)); /* 4 lines + 2*radix */
    if (!w->xr) return -1;
    w->xi = w->xr + n; w->yr = w->xi + n; w->yi = w->yr + n; w->tmp = w->yi + n;
    return 0;
}
static void work_free(cfft_work* w) { free(w->xr); }

/* FFTW R2HC: x (stride sx) -> hc (stride sh) */
static void r2hc_line(const cfft_plan* P, cfft_work* w, const double* x, size_t sx, double* hc, size_t sh) {
    const int n = P->n;
    for (int j = 0; j < n; j++) { w->xr[j] = x[(size_t)j * sx]; w->xi[j] = 0.0; }
    cfft_rec(P, w->xr, w->xi, 1, w->yr, w->yi, n, P->fac, -1, w->tmp);
    for (int k = 0; k <= n / 2; k++) hc[(size_t)k * sh] = w->yr[k];
    for (int k = 1; k < (n + 1) / 2; k++) hc[(size_t)(n - k) * sh] = w->yi[k];
}

/* FFTW HC2R (unnormalised inverse) */
static void hc2r_line(const cfft_plan* P, cfft_work* w, const double* hc, size_t sh, double* x, size_t sx) {
    const int n = P->n;
    w->xr[0] = hc[0]; w->xi[0] = 0.0;
    for (int k = 1; k < (n + 1) / 2; k++) {
        double re = hc[(size_t)k * sh], im = hc[(size_t)(n - k) * sh];
        w->xr[k] = re; w->xi[k] = im;
        w->xr[n - k] = re; w->xi[n - k] = -im;
    }
    if (n % 2 == 0) { w->xr[n / 2] = hc[(size_t)(n / 2) * sh]; w->xi[n / 2] = 0.0; }
    cfft_rec(P, w->xr, w->xi, 1, w->yr, w->yi, n, P->fac, +1, w->tmp);
    for (int j = 0; j < n; j++) x[(size_t)j * sx] = w->yr[j];
}

int orc_r2hc(int n, const double* x, double* hc) {
    if (n < 1 || !x || !hc) return -1;
    cfft_plan P; cfft_work w;
    if (cfft_init(&P, n) || work_init(&w, n)) return -2;
    r2hc_line(&P, &w, x, 1, hc, 1);
    work_free(&w); cfft_free(&P);
    return 0;
}

int orc_hc2r(int n, const double* hc, double* x) {
    if (n < 1 || !x || !hc) return -1;
    cfft_plan P; cfft_work w;
    if (cfft_init(&P, n) || work_init(&w, n)) return -2;
    hc2r_line(&P, &w, hc, 1, x, 1);
    work_free(&w); cfft_free(&P);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Bands and 1-D metrics                                                      */
/* ------------------------------------------------------------------------- */

int orc_mk_P_abc(int ny, const double* yp_ext, int is_dirich_first, double* a, double* b, double* c) {
    if (ny < 2 || !yp_ext || !a || !b || !c) return -1;
    double* yp_pad = (double*)malloc(sizeof(double) * (size_t)(ny + 2));
    if (!yp_pad) return -2;
    memcpy(yp_pad, yp_ext, sizeof(double) * (size_t)(ny + 2));
    yp_pad[0] = 2 * yp_ext[0] - yp_ext[1];
    yp_pad[ny + 1] = 2 * yp_ext[ny + 1] - yp_ext[ny];
    for (int i = 0; i < ny; i++) {
        double x0 = yp_pad[i], x1 = yp_pad[i + 1], x2 = yp_pad[i + 2];
        double dy = 0.5 * (x2 - x0);
        a[i] = 1.0 / ((x1 - x0) * dy);
        c[i] = 1.0 / ((x2 - x1) * dy);
        b[i] = -(a[i] + c[i]);
    }
    if (is_dirich_first) b[0] -= a[0];
    else b[0] += a[0];
    b[ny - 1] += c[ny - 1];
    a[0] = 0.0;
    c[ny - 1] = 0.0;
    free(yp_pad);
    return 0;
}

static void yp_ext_from_yu(int ny, const double* yu, double* yp_ext) {
    yp_ext[0] = yu[0];
    for (int i = 0; i < ny; i++) yp_ext[i + 1] = (yu[i] + yu[i + 1]) / 2;
    yp_ext[ny + 1] = yu[ny];
}

int orc_bands_from_yu(int ny, const double* yu, int mode, double* a, double* b, double* c,
                      double* a00, double* b00, double* c00) {
    if (ny < 2 || !yu || !a || !b || !c || !a00 || !b00 || !c00) return -1;
    double* yp_ext = (double*)malloc(sizeof(double) * (size_t)(ny + 2));
    if (!yp_ext) return -2;
    yp_ext_from_yu(ny, yu, yp_ext);
    int rc = 0;
    if (mode == 0) {
        rc = orc_mk_P_abc(ny, yp_ext, 0, a, b, c);
        if (!rc) rc = orc_mk_P_abc(ny, yp_ext, 1, a00, b00, c00);
    } else if (mode == 1) {
        const double* yp = yp_ext + 1;
        for (int k = 0; k < ny; k++) {
            double idy = 1.0 / (yu[k + 1] - yu[k]);
            a[k] = (k > 0) ? idy / (yp[k] - yp[k - 1]) : 0.0;
            c[k] = (k < ny - 1) ? idy / (yp[k + 1] - yp[k]) : 0.0;
            b[k] = -(a[k] + c[k]);
            a00[k] = a[k]; b00[k] = b[k]; c00[k] = c[k];
        }
        /* Dirichlet ghost mirrored about the wall, as mk_P_abc's yp_pad[0] */
        double ghost = 2 * yu[0] - yp[0];
        b00[0] -= 2.0 * (1.0 / (yu[1] - yu[0])) / (yp[0] - ghost);
    } else {
        rc = -1;
    }
    free(yp_ext);
    return rc;
}

int orc_metrics_from_yu(int ny, const double* yu, double* inv_dy_p, double* dPdy_lo, double* dPdy_hi) {
    if (ny < 2 || !yu || !inv_dy_p || !dPdy_lo || !dPdy_hi) return -1;
    for (int i = 0; i < ny; i++) inv_dy_p[i] = 1. / (yu[i + 1] - yu[i]);
    dPdy_lo[0] = 0.0; dPdy_hi[0] = 0.0;
    for (int i = 1; i < ny; i++) {
        double ypi = (yu[i] + yu[i + 1]) / 2, ypm = (yu[i - 1] + yu[i]) / 2;
        double dy = ypi - ypm;
        dPdy_lo[i] = -1 / dy;
        dPdy_hi[i] = 1 / dy;
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Poisson solve, FFTW path of run_spec_poisson_multigpu (single rank)        */
/* ------------------------------------------------------------------------- */

/* halfcomplex index -> wavenumber, poisson_solver_multigpu.f90:141-142 */
static int hc_wavenumber(int i, int n) {
    if (i <= n / 2) return i;
    int v = (n + 1) / 2 - 1 - (i - (n / 2 + 1));
    return v < 1 ? 1 : v;
}

int orc_poisson(int nx, int nz, int ny, double dx, double dz,
                const double* a, const double* b, const double* c,
                const double* a00, const double* b00, const double* c00,
                double* P, double* min_pivot, int nthreads) {
    if (nx < 1 || nz < 1 || ny < 2 || !P || !a || !b || !c || !a00 || !b00 || !c00) return -1;
    set_threads(nthreads);
    const double const_pi = 4.0 * atan(1.0);
    const double inv_dx = 1.0 / dx, inv_dz = 1.0 / dz;
    /* P_z(j=z, i=x halfcomplex, k) holds the x-transformed data, z fastest */
    double* Pz = (double*)malloc(sizeof(double) * (size_t)nx * nz * ny);
    double* ax = (double*)malloc(sizeof(double) * (size_t)nx);
    double* az = (double*)malloc(sizeof(double) * (size_t)nz);
    int* isx = (int*)malloc(sizeof(int) * (size_t)nx);
    int* isz = (int*)malloc(sizeof(int) * (size_t)nz);
    if (!Pz || !ax || !az || !isx || !isz) { free(Pz); free(ax); free(az); free(isx); free(isz); return -2; }
    for (int i = 0; i < nx; i++) {
        int ii = hc_wavenumber(i, nx);
        double s = sin(ii * const_pi / nx);
        ax[i] = -4 * (inv_dx * inv_dx) * (s * s);
        isx[i] = (ii == 0);
    }
    for (int j = 0; j < nz; j++) {
        int jj = hc_wavenumber(j, nz);
        double s = sin(jj * const_pi / nz);
        az[j] = -4 * (inv_dz * inv_dz) * (s * s);
        isz[j] = (jj == 0);
    }
    cfft_plan Px, Pzp;
    if (cfft_init(&Px, nx) || cfft_init(&Pzp, nz)) { free(Pz); free(ax); free(az); free(isx); free(isz); return -2; }
    int err = 0;
    double minpiv = 1e20;

    /* forward x (R2HC) and transpose into P_z, :365, :377 */
#pragma omp parallel reduction(| : err)
    {
        cfft_work w;
        double* line = (double*)malloc(sizeof(double) * (size_t)nx);
        if (work_init(&w, nx) || !line) err |= 1;
        else {
#pragma omp for schedule(static)
            for (long jk = 0; jk < (long)nz * ny; jk++) {
                int j = (int)(jk % nz), k = (int)(jk / nz);
                r2hc_line(&Px, &w, P + PIDX(0, j, k), 1, line, 1);
                for (int i = 0; i < nx; i++) Pz[(size_t)j + (size_t)nz * ((size_t)i + (size_t)nx * k)] = line[i];
            }
            work_free(&w);
        }
        free(line);
    }
    /* forward z (R2HC) in place, Thomas per (j,i), inverse z, :383, :395-422, :507 */
#pragma omp parallel reduction(| : err) reduction(min : minpiv)
    {
        cfft_work w;
        double* line = (double*)malloc(sizeof(double) * (size_t)nz);
        double* cp = (double*)malloc(sizeof(double) * (size_t)ny);
        double* spec = (double*)malloc(sizeof(double) * (size_t)nz * ny);
        if (work_init(&w, nz) || !line || !cp || !spec) err |= 1;
        else {
#pragma omp for schedule(static)
            for (int i = 0; i < nx; i++) {
                for (int k = 0; k < ny; k++)
                    r2hc_line(&Pzp, &w, Pz + (size_t)nz * ((size_t)i + (size_t)nx * k), 1, spec + (size_t)nz * k, 1);
                for (int j = 0; j < nz; j++) {
                    const int is00 = isx[i] * isz[j];
                    const double* A = is00 ? a00 : a;
                    const double* B = is00 ? b00 : b;
                    const double* C = is00 ? c00 : c;
                    const double axz = (ax[i] + az[j]);
                    /* poi_C, :167-176 ; min pivot, :187-193 */
                    cp[0] = C[0] / (B[0] + axz);
                    double pv = fabs(B[0] + axz);
                    if (pv < minpiv) minpiv = pv;
                    for (int k = 1; k < ny; k++) {
                        cp[k] = C[k] / (B[k] + axz - A[k] * cp[k - 1]);
                        pv = fabs(B[k] + axz - A[k] * cp[k - 1]);
                        if (pv < minpiv) minpiv = pv;
                    }
                    /* Thomas, :401-419 */
                    double* s = spec + j;
                    s[0] = s[0] / (B[0] + axz);
                    for (int k = 1; k < ny; k++)
                        s[(size_t)nz * k] = (s[(size_t)nz * k] - A[k] * s[(size_t)nz * (k - 1)]) / (B[k] + axz - A[k] * cp[k - 1]);
                    for (int k = ny - 2; k >= 0; k--)
                        s[(size_t)nz * k] = s[(size_t)nz * k] - s[(size_t)nz * (k + 1)] * cp[k];
                }
                for (int k = 0; k < ny; k++)
                    hc2r_line(&Pzp, &w, spec + (size_t)nz * k, 1, Pz + (size_t)nz * ((size_t)i + (size_t)nx * k), 1);
            }
            work_free(&w);
        }
        free(line); free(cp); free(spec);
    }
    /* transpose back, inverse x (HC2R) and scale, :520, :527, :540-551 */
    const double inv_nxnz = 1.0 / ((double)nx * (double)nz + 0.0);
#pragma omp parallel reduction(| : err)
    {
        cfft_work w;
        double* line = (double*)malloc(sizeof(double) * (size_t)nx);
        if (work_init(&w, nx) || !line) err |= 1;
        else {
#pragma omp for schedule(static)
            for (long jk = 0; jk < (long)nz * ny; jk++) {
                int j = (int)(jk % nz), k = (int)(jk / nz);
                for (int i = 0; i < nx; i++) line[i] = Pz[(size_t)j + (size_t)nz * ((size_t)i + (size_t)nx * k)];
                double* out = P + PIDX(0, j, k);
                hc2r_line(&Px, &w, line, 1, out, 1);
                for (int i = 0; i < nx; i++) out[i] = out[i] * inv_nxnz;
            }
            work_free(&w);
        }
        free(line);
    }
    cfft_free(&Px); cfft_free(&Pzp);
    free(Pz); free(ax); free(az); free(isx); free(isz);
    if (min_pivot) *min_pivot = minpiv;
    return err ? -2 : 0;
}

/* ------------------------------------------------------------------------- */
/* Divergence, correction, max|div|                                           */
/* ------------------------------------------------------------------------- */

static inline double vh_face(int nx, int nz, const double* Vh, int i, int j, int k, int ny, double vbot, double vtop) {
    if (k == 0) return vbot;
    if (k == ny) return vtop;
    return Vh[HIDX(i, j, k)];
}

int orc_divergence(int nx, int nz, int ny, double dx, double dz, double dt,
                   const double* inv_dy_p, const double* Uh, const double* Vh,
                   const double* Wh, double vbot, double vtop, double* P, int nthreads) {
    if (nx < 1 || nz < 1 || ny < 2 || !inv_dy_p || !Uh || !Vh || !Wh || !P) return -1;
    set_threads(nthreads);
    const double inv_dx = 1.0 / dx, inv_dz = 1.0 / dz, inv_dtmax = 1.0 / dt;
#pragma omp parallel for schedule(static)
    for (long jk = 0; jk < (long)nz * ny; jk++) {
        int j = (int)(jk % nz), k = (int)(jk / nz);
        int jp = (j + 1 == nz) ? 0 : j + 1; /* periodic halo, :505 */
        for (int i = 0; i < nx; i++) {
            int ip = (i + 1 == nx) ? 0 : i + 1; /* periodic halo, :504 */
            double vp = vh_face(nx, nz, Vh, i, j, k + 1, ny, vbot, vtop);
            double v0 = vh_face(nx, nz, Vh, i, j, k, ny, vbot, vtop);
            P[PIDX(i, j, k)] = inv_dtmax * ((Uh[HIDX(ip, j, k)] - Uh[HIDX(i, j, k)]) * inv_dx +
                                            (Wh[HIDX(i, jp, k)] - Wh[HIDX(i, j, k)]) * inv_dz +
                                            (vp - v0) * inv_dy_p[k]);
        }
    }
    return 0;
}

/* periodic x/z halos on every y-slice, then the wall slices (set_val_slice
 * covers the full x/z extent including halos, mod_utils.f90:38-61) */
static void fill_halos(int nx, int nz, int ny, double* F, int kfirst_bot, double bot, double top) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < ny; k++) {
        for (int j = 0; j < nz; j++) {
            F[HIDX(-1, j, k)] = F[HIDX(nx - 1, j, k)];
            F[HIDX(nx, j, k)] = F[HIDX(0, j, k)];
        }
        for (int i = -1; i <= nx; i++) {
            F[HIDX(i, -1, k)] = F[HIDX(i, nz - 1, k)];
            F[HIDX(i, nz, k)] = F[HIDX(i, 0, k)];
        }
    }
#pragma omp parallel for schedule(static)
    for (int j = -1; j <= nz; j++)
        for (int i = -1; i <= nx; i++) {
            for (int k = -1; k <= kfirst_bot; k++) F[HIDX(i, j, k)] = bot;
            F[HIDX(i, j, ny)] = top;
        }
}

int orc_correction(int nx, int nz, int ny, double dx, double dz, double dt,
                   const double* dPdy_lo, const double* dPdy_hi, const double* P,
                   const double* Uh, const double* Vh, const double* Wh,
                   const double* wall, double* U, double* V, double* W, int nthreads) {
    if (nx < 1 || nz < 1 || ny < 2 || !dPdy_lo || !dPdy_hi || !P || !Uh || !Vh || !Wh || !wall || !U || !V || !W) return -1;
    set_threads(nthreads);
    const double inv_dx = 1.0 / dx, inv_dz = 1.0 / dz, dtmax = dt;
    const int kmin_Vhat = 1; /* single rank in y: main.f90:86-87 */
#pragma omp parallel for schedule(static)
    for (long jk = 0; jk < (long)nz * ny; jk++) {
        int j = (int)(jk % nz), k = (int)(jk / nz);
        int jm = (j == 0) ? nz - 1 : j - 1;
        for (int i = 0; i < nx; i++) {
            int im = (i == 0) ? nx - 1 : i - 1;
            double p0 = P[PIDX(i, j, k)];
            U[HIDX(i, j, k)] = Uh[HIDX(i, j, k)] - dtmax * (p0 - P[PIDX(im, j, k)]) * inv_dx;
            W[HIDX(i, j, k)] = Wh[HIDX(i, j, k)] - dtmax * (p0 - P[PIDX(i, jm, k)]) * inv_dz;
            if (k >= kmin_Vhat)
                V[HIDX(i, j, k)] = Vh[HIDX(i, j, k)] - dtmax * (dPdy_hi[k] * p0 + dPdy_lo[k] * P[PIDX(i, j, k - 1)]);
        }
    }
    fill_halos(nx, nz, ny, U, -1, wall[0], wall[3]);
    fill_halos(nx, nz, ny, V, 0, wall[1], wall[4]);
    fill_halos(nx, nz, ny, W, -1, wall[2], wall[5]);
    return 0;
}

double orc_div_maxabs(int nx, int nz, int ny, double dx, double dz,
                      const double* inv_dy_p, const double* U, const double* V,
                      const double* W, int nthreads) {
    set_threads(nthreads);
    const double inv_dx = 1.0 / dx, inv_dz = 1.0 / dz;
    double m = -1e20;
#pragma omp parallel for schedule(static) reduction(max : m)
    for (long jk = 0; jk < (long)nz * ny; jk++) {
        int j = (int)(jk % nz), k = (int)(jk / nz);
        for (int i = 0; i < nx; i++) {
            double d = fabs((U[HIDX(i + 1, j, k)] - U[HIDX(i, j, k)]) * inv_dx +
                            (W[HIDX(i, j + 1, k)] - W[HIDX(i, j, k)]) * inv_dz +
                            (V[HIDX(i, j, k + 1)] - V[HIDX(i, j, k)]) * inv_dy_p[k]);
            if (d > m) m = d;
        }
    }
    return m;
}

int orc_projection(int nx, int nz, int ny, double dx, double dz, double dt,
                   const double* a, const double* b, const double* c,
                   const double* a00, const double* b00, const double* c00,
                   const double* inv_dy_p, const double* dPdy_lo, const double* dPdy_hi,
                   const double* Uh, const double* Vh, const double* Wh, const double* wall,
                   double* U, double* V, double* W, double* P, int nthreads) {
    if (!wall) return -1;
    int rc = orc_divergence(nx, nz, ny, dx, dz, dt, inv_dy_p, Uh, Vh, Wh, wall[1], wall[4], P, nthreads);
    if (rc) return rc;
    rc = orc_poisson(nx, nz, ny, dx, dz, a, b, c, a00, b00, c00, P, NULL, nthreads);
    if (rc) return rc;
    return orc_correction(nx, nz, ny, dx, dz, dt, dPdy_lo, dPdy_hi, P, Uh, Vh, Wh, wall, U, V, W, nthreads);
}

/* ------------------------------------------------------------------------- */
/* Variable-density projection (use_incompressible = .false.)                */
/* ------------------------------------------------------------------------- */

double orc_rho_min(int nx, int nz, int ny, const double* rho, int nthreads) {
    set_threads(nthreads);
    double m = 1e20; /* mod_cfd_subroutines.f90:476 */
#pragma omp parallel for schedule(static) reduction(min : m)
    for (long jk = 0; jk < (long)nz * ny; jk++) {
        int j = (int)(jk % nz), k = (int)(jk / nz);
        for (int i = 0; i < nx; i++) {
            double r = rho[HIDX(i, j, k)];
            if (r < m) m = r;
        }
    }
    return m;
}

int orc_vd_metric_from_yu(int ny, const double* yu, double* inv_dy_p_pad) {
    if (ny < 2 || !yu || !inv_dy_p_pad) return -1;
    /* yp_pad = [2 yu_0 - yp_0, yp_0 .. yp_{ny-1}, 2 yu_ny - yp_{ny-1}], calc_bands.py:273, :276 */
    double* yp_pad = (double*)malloc((size_t)(ny + 2) * sizeof(double));
    if (!yp_pad) return -3;
    for (int k = 0; k < ny; k++) yp_pad[k + 1] = (yu[k] + yu[k + 1]) / 2;
    yp_pad[0] = 2 * yu[0] - yp_pad[1];
    yp_pad[ny + 1] = 2 * yu[ny] - yp_pad[ny];
    for (int i = 0; i <= ny; i++) inv_dy_p_pad[i] = 1. / (yp_pad[i + 1] - yp_pad[i]);
    free(yp_pad);
    return 0;
}

/* 2 P_now - P_old at a halo'd index */
static inline double ps_at(const double* Pn, const double* Po, size_t h) { return 2 * Pn[h] - Po[h]; }

/* 1 - rho_min (0.5/rho_a + 0.5/rho_b) */
static inline double rho_w(double rho_min, double ra, double rb) { return 1.0 - rho_min * (0.5 / ra + 0.5 / rb); }

int orc_vd_rhs(int nx, int nz, int ny, double dx, double dz, double dt,
               const double* inv_dy_p, const double* inv_dy_p_pad,
               const double* Uh, const double* Vh, const double* Wh, double vbot, double vtop,
               const double* rho, const double* P_now, const double* P_old, const double* div_now,
               double rho_min, double* P, int nthreads) {
    if (nx < 1 || nz < 1 || ny < 2 || !inv_dy_p || !inv_dy_p_pad || !Uh || !Vh || !Wh || !rho || !P_now ||
        !P_old || !div_now || !P)
        return -1;
    set_threads(nthreads);
    const double inv_dx = 1.0 / dx, inv_dz = 1.0 / dz, inv_dtmax = 1.0 / dt;
    const double inv_dx2 = inv_dx * inv_dx, inv_dz2 = inv_dz * inv_dz;
#pragma omp parallel for schedule(static)
    for (long jk = 0; jk < (long)nz * ny; jk++) {
        int j = (int)(jk % nz), k = (int)(jk / nz);
        int jp = (j + 1 == nz) ? 0 : j + 1;
        for (int i = 0; i < nx; i++) {
            int ip = (i + 1 == nx) ? 0 : i + 1;
            const size_t h = HIDX(i, j, k);
            double vp = vh_face(nx, nz, Vh, i, j, k + 1, ny, vbot, vtop);
            double v0 = vh_face(nx, nz, Vh, i, j, k, ny, vbot, vtop);
            /* the stencil of P_now, P_old and rho reads the caller's halos, MCS:543-556 */
            double Ps_00 = ps_at(P_now, P_old, h);
            double Ps_xp = ps_at(P_now, P_old, HIDX(i + 1, j, k)), Ps_xm = ps_at(P_now, P_old, HIDX(i - 1, j, k));
            double Ps_zp = ps_at(P_now, P_old, HIDX(i, j + 1, k)), Ps_zm = ps_at(P_now, P_old, HIDX(i, j - 1, k));
            double Ps_yp = ps_at(P_now, P_old, HIDX(i, j, k + 1)), Ps_ym = ps_at(P_now, P_old, HIDX(i, j, k - 1));
            double r0 = rho[h];
            double rho_xp = rho_w(rho_min, rho[HIDX(i + 1, j, k)], r0), rho_xm = rho_w(rho_min, rho[HIDX(i - 1, j, k)], r0);
            double rho_zp = rho_w(rho_min, rho[HIDX(i, j + 1, k)], r0), rho_zm = rho_w(rho_min, rho[HIDX(i, j - 1, k)], r0);
            double rho_yp = rho_w(rho_min, rho[HIDX(i, j, k + 1)], r0), rho_ym = rho_w(rho_min, rho[HIDX(i, j, k - 1)], r0);
            /* MCS:558-564 */
            double dv = ((Uh[HIDX(ip, j, k)] - Uh[h]) * inv_dx + (Wh[HIDX(i, jp, k)] - Wh[h]) * inv_dz +
                         (vp - v0) * inv_dy_p[k]);
            P[PIDX(i, j, k)] = inv_dtmax * dv * rho_min - inv_dtmax * rho_min * div_now[h] +
                               ((rho_xp * (Ps_xp - Ps_00) - rho_xm * (Ps_00 - Ps_xm)) * inv_dx2 +
                                (rho_zp * (Ps_zp - Ps_00) - rho_zm * (Ps_00 - Ps_zm)) * inv_dz2 +
                                (rho_yp * (Ps_yp - Ps_00) * inv_dy_p_pad[k + 1] -
                                 rho_ym * (Ps_00 - Ps_ym) * inv_dy_p_pad[k]) * inv_dy_p[k]);
        }
    }
    return 0;
}

int orc_vd_correction(int nx, int nz, int ny, double dx, double dz, double dt,
                      const double* dPdy_lo, const double* dPdy_hi, const double* P,
                      const double* Uh, const double* Vh, const double* Wh, const double* wall,
                      const double* rho, const double* P_now, const double* P_old, double rho_min,
                      double* U, double* V, double* W, double* P_next, int nthreads) {
    if (nx < 1 || nz < 1 || ny < 2 || !dPdy_lo || !dPdy_hi || !P || !Uh || !Vh || !Wh || !wall || !rho ||
        !P_now || !P_old || !U || !V || !W || !P_next)
        return -1;
    set_threads(nthreads);
    const double inv_dx = 1.0 / dx, inv_dz = 1.0 / dz, dtmax = dt;
    const double inv_rho_min = 1.0 / rho_min;
    const int kmin_Vhat = 1;
    /* P_per: P with periodic x/z halos and the wall ghost planes P(-1) = P(0),
     * P(ny) = P(ny-1), MCS:1087-1118; it becomes P_next (the caller's next P_now) */
#pragma omp parallel for schedule(static)
    for (long jk = 0; jk < (long)(nz + 2) * (ny + 2); jk++) {
        int j = (int)(jk % (nz + 2)) - 1, k = (int)(jk / (nz + 2)) - 1;
        int js = (j < 0) ? nz - 1 : (j == nz ? 0 : j);
        int ks = (k < 0) ? 0 : (k == ny ? ny - 1 : k);
        for (int i = -1; i <= nx; i++) {
            int is = (i < 0) ? nx - 1 : (i == nx ? 0 : i);
            P_next[HIDX(i, j, k)] = P[PIDX(is, js, ks)];
        }
    }
    /* MCS:1153-1197 */
#pragma omp parallel for schedule(static)
    for (long jk = 0; jk < (long)nz * ny; jk++) {
        int j = (int)(jk % nz), k = (int)(jk / nz);
        for (int i = 0; i < nx; i++) {
            const size_t h = HIDX(i, j, k);
            double inv_rho_now, P_fwd, P_bwd;
            size_t hm = HIDX(i - 1, j, k);
            inv_rho_now = 0.5 / rho[h] + 0.5 / rho[hm];
            P_fwd = P_next[h] * inv_rho_min + (inv_rho_now - inv_rho_min) * (2 * P_now[h] - P_old[h]);
            P_bwd = P_next[hm] * inv_rho_min + (inv_rho_now - inv_rho_min) * (2 * P_now[hm] - P_old[hm]);
            U[h] = Uh[h] - dtmax * (P_fwd - P_bwd) * inv_dx;
            hm = HIDX(i, j - 1, k);
            inv_rho_now = 0.5 / rho[h] + 0.5 / rho[hm];
            P_fwd = P_next[h] * inv_rho_min + (inv_rho_now - inv_rho_min) * (2 * P_now[h] - P_old[h]);
            P_bwd = P_next[hm] * inv_rho_min + (inv_rho_now - inv_rho_min) * (2 * P_now[hm] - P_old[hm]);
            W[h] = Wh[h] - dtmax * (P_fwd - P_bwd) * inv_dz;
            if (k >= kmin_Vhat) {
                hm = HIDX(i, j, k - 1);
                inv_rho_now = 0.5 / rho[h] + 0.5 / rho[hm];
                P_fwd = P_next[h] * inv_rho_min + (inv_rho_now - inv_rho_min) * (2 * P_now[h] - P_old[h]);
                P_bwd = P_next[hm] * inv_rho_min + (inv_rho_now - inv_rho_min) * (2 * P_now[hm] - P_old[hm]);
                V[h] = Vh[h] - dtmax * (dPdy_hi[k] * P_fwd + dPdy_lo[k] * P_bwd);
            }
        }
    }
    fill_halos(nx, nz, ny, U, -1, wall[0], wall[3]);
    fill_halos(nx, nz, ny, V, 0, wall[1], wall[4]);
    fill_halos(nx, nz, ny, W, -1, wall[2], wall[5]);
    return 0;
}

int orc_projection_vd(int nx, int nz, int ny, double dx, double dz, double dt,
                      const double* a, const double* b, const double* c,
                      const double* a00, const double* b00, const double* c00,
                      const double* inv_dy_p, const double* dPdy_lo, const double* dPdy_hi,
                      const double* inv_dy_p_pad, const double* Uh, const double* Vh, const double* Wh,
                      const double* wall, const double* rho, const double* P_now, const double* P_old,
                      const double* div_now, double* U, double* V, double* W, double* P, double* P_next,
                      double* rho_min_out, int nthreads) {
    if (!wall || !rho) return -1;
    const double rho_min = orc_rho_min(nx, nz, ny, rho, nthreads);
    if (rho_min_out) *rho_min_out = rho_min;
    int rc = orc_vd_rhs(nx, nz, ny, dx, dz, dt, inv_dy_p, inv_dy_p_pad, Uh, Vh, Wh, wall[1], wall[4], rho, P_now,
                        P_old, div_now, rho_min, P, nthreads);
    if (rc) return rc;
    rc = orc_poisson(nx, nz, ny, dx, dz, a, b, c, a00, b00, c00, P, NULL, nthreads);
    if (rc) return rc;
    return orc_vd_correction(nx, nz, ny, dx, dz, dt, dPdy_lo, dPdy_hi, P, Uh, Vh, Wh, wall, rho, P_now, P_old,
                             rho_min, U, V, W, P_next, nthreads);
}

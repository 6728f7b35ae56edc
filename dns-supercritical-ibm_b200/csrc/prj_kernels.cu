// prj_kernels.cu -- CUDA kernels of the FP64 pressure projection (sm_100a).
//
// Data flow of one projection (one CTA grid per arrow):
//
//   u_hat --(k_fwd_x: divergence + real FFT along x)--> X[y][kx][z]
//         --(k_zsolve: per kx, stream over y: FFT along z, Thomas forward
//            sweep, then backward sweep + inverse FFT along z)--> X
//         --(k_bwd_x: inverse real FFT along x, 1/(nx nz))--> P
//         --(k_correct: u = u_hat - dt grad P, halos, walls)--> u
//
// The x and z transforms are the reference's cuFFT D2Z/Z2D pair and
// diezDecomp transpose (poisson_solver_multigpu.f90:360-392, :501-537) fused
// into two kernels that read/write x-rows and z-major spectral tiles.  The
// Thomas recurrence keeps the reference's operation order
// (poisson_solver_multigpu.f90:395-422, with poi_C(k) = c_k / pivot_k) and
// uses round-to-nearest intrinsics so the compiler cannot contract it into
// FMAs; only the pivots (not poi_C) are tabulated.
#include <cstdio>

#include "prj_internal.h"

namespace prj {

namespace {

__device__ __forceinline__ size_t hidx(int nx, int nz, int i, int j, int k) {
    return (size_t)(i + 1) + (size_t)(nx + 2) * ((size_t)(j + 1) + (size_t)(nz + 2) * (size_t)(k + 1));
}

struct FwdArgs {
    int nx, nz, ny, nh, m, tz, rs;
    int even;
    FftDev f;
    const double2* tw;
    const double2* post;
    const double* P;
    const double* Uh;
    const double* Vh;
    const double* Wh;
    const double* inv_dy_p;
    double inv_dx, inv_dz, inv_dt, vbot, vtop;
    double2* X;
};

// divergence of the predictor at cell (i, j, k): mod_cfd_subroutines.f90:532-534
__device__ __forceinline__ double divergence_at(const FwdArgs& a, int i, int j, int k) {
    const int nx = a.nx, nz = a.nz;
    const int ip = (i + 1 == nx) ? 0 : i + 1;
    const int jp = (j + 1 == nz) ? 0 : j + 1;
    const double u1 = a.Uh[hidx(nx, nz, ip, j, k)], u0 = a.Uh[hidx(nx, nz, i, j, k)];
    const double w1 = a.Wh[hidx(nx, nz, i, jp, k)], w0 = a.Wh[hidx(nx, nz, i, j, k)];
    const double v1 = (k + 1 == a.ny) ? a.vtop : a.Vh[hidx(nx, nz, i, j, k + 1)];
    const double v0 = (k == 0) ? a.vbot : a.Vh[hidx(nx, nz, i, j, k)];
    double s = __dmul_rn(__dsub_rn(u1, u0), a.inv_dx);
    s = __dadd_rn(s, __dmul_rn(__dsub_rn(w1, w0), a.inv_dz));
    s = __dadd_rn(s, __dmul_rn(__dsub_rn(v1, v0), a.inv_dy_p[k]));
    return __dmul_rn(a.inv_dt, s);
}

template <int SRC>
__global__ void __launch_bounds__(256) k_fwd_x(const FwdArgs a) {
    extern __shared__ double2 sm[];
    double2* A = sm;
    double2* B = sm + a.tz * a.rs;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int y = blockIdx.y;
    const int z0 = blockIdx.x * a.tz;
    const int m = a.m;

    // load tz x-rows (packed even/odd samples for even nx)
    for (int idx = tid; idx < a.tz * m; idx += nthr) {
        const int r = idx / m, n = idx - r * m;
        const int z = z0 + r;
        double2 v = make_double2(0.0, 0.0);
        if (z < a.nz) {
            if (SRC == 0) {
                const double* row = a.P + ((size_t)y * a.nz + z) * a.nx;
                if (a.even) v = reinterpret_cast<const double2*>(row)[n];
                else v.x = row[n];
            } else {
                if (a.even) { v.x = divergence_at(a, 2 * n, z, y); v.y = divergence_at(a, 2 * n + 1, z, y); }
                else v.x = divergence_at(a, n, z, y);
            }
        }
        A[r * a.rs + n] = v;
    }
    __syncthreads();
    double2* F = fft_rows<-1>(A, B, a.tz, a.rs, a.f, a.tw);
    double2* G = F;
    if (a.even) {
        // split the packed transform into the spectrum of the real row:
        // X_k = E_k + exp(-2 pi i k/n) O_k, E/O = transforms of even/odd samples
        G = (F == A) ? B : A;
        for (int idx = tid; idx < a.tz * (m + 1); idx += nthr) {
            const int r = idx / (m + 1), k = idx - r * (m + 1);
            const double2* Z = F + r * a.rs;
            const double2 zk = Z[k == m ? 0 : k];
            const double2 zm = cconj(Z[k == 0 ? 0 : m - k]);
            const double2 e = cscale(cadd(zk, zm), 0.5);
            const double2 d = csub(zk, zm);
            const double2 o = make_double2(0.5 * d.y, -0.5 * d.x);
            G[r * a.rs + k] = cadd(e, cmul(a.post[k], o));
        }
        __syncthreads();
    }
    // transposed store: X[y][kx][z0 .. z0+tz)
    for (int idx = tid; idx < a.nh * a.tz; idx += nthr) {
        const int kx = idx / a.tz, r = idx - kx * a.tz;
        const int z = z0 + r;
        if (z < a.nz) a.X[((size_t)y * a.nh + kx) * a.nz + z] = G[r * a.rs + kx];
    }
}

struct BwdArgs {
    int nx, nz, ny, nh, m, tz, rs;
    int even;
    FftDev f;
    const double2* tw;
    const double2* post;
    const double2* X;
    double* P;
    double scale;
};

__global__ void __launch_bounds__(256) k_bwd_x(const BwdArgs a) {
    extern __shared__ double2 sm[];
    double2* A = sm;
    double2* B = sm + a.tz * a.rs;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int y = blockIdx.y;
    const int z0 = blockIdx.x * a.tz;
    const int m = a.m;
    for (int idx = tid; idx < a.nh * a.tz; idx += nthr) {
        const int kx = idx / a.tz, r = idx - kx * a.tz;
        const int z = z0 + r;
        double2 v = make_double2(0.0, 0.0);
        if (z < a.nz) v = a.X[((size_t)y * a.nh + kx) * a.nz + z];
        A[r * a.rs + kx] = v;
    }
    __syncthreads();
    if (a.even) {
        // inverse of the split: Z_k = (X_k + conj X_{m-k}) + i (X_k - conj X_{m-k}) exp(+2 pi i k/n);
        // the imaginary parts of the k = 0 and k = m modes are ignored (c2r semantics)
        for (int idx = tid; idx < a.tz * m; idx += nthr) {
            const int r = idx / m, k = idx - r * m;
            const double2* Xr = A + r * a.rs;
            double2 xk = Xr[k];
            double2 xm = Xr[m - k];
            if (k == 0) { xk.y = 0.0; xm.y = 0.0; }
            xm = cconj(xm);
            const double2 e = cadd(xk, xm);
            const double2 o = cmulc(csub(xk, xm), a.post[k]);
            B[r * a.rs + k] = cscale(make_double2(e.x - o.y, e.y + o.x), a.scale);
        }
    } else {
        for (int idx = tid; idx < a.tz * m; idx += nthr) {
            const int r = idx / m, k = idx - r * m;
            const double2* Xr = A + r * a.rs;
            double2 v;
            if (k < a.nh) { v = Xr[k]; if (k == 0) v.y = 0.0; }
            else v = cconj(Xr[m - k]);
            B[r * a.rs + k] = cscale(v, a.scale);
        }
    }
    __syncthreads();
    double2* F = fft_rows<+1>(B, A, a.tz, a.rs, a.f, a.tw);
    for (int idx = tid; idx < a.tz * m; idx += nthr) {
        const int r = idx / m, n = idx - r * m;
        const int z = z0 + r;
        if (z >= a.nz) continue;
        double* row = a.P + ((size_t)y * a.nz + z) * a.nx;
        const double2 v = F[r * a.rs + n];
        if (a.even) reinterpret_cast<double2*>(row)[n] = v;
        else row[n] = v.x;
    }
}

struct ZArgs {
    int nz, ny, nh, nzh, mzp;
    FftDev f;
    const double2* tw;
    const double* bands;  // a, b, c, a00, b00, c00
    const double* piv;    // D[y][kx][kzs]
    double2* X;
};

constexpr int kPairsPerThread = 4;

// One CTA per kx.  Forward pass over y: FFT along z, then one Thomas forward
// step for every kz line (the pair kz, nz-kz shares its pivots).  Backward pass
// over y: back substitution, inverse FFT along z.  X is overwritten in place:
// forward-sweep values d' on the way up, the final spectrum on the way down.
__global__ void __launch_bounds__(512) k_zsolve(const ZArgs a) {
    extern __shared__ double2 sm[];
    double2* A = sm;
    double2* B = sm + a.nz;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int kx = blockIdx.x;
    const int nz = a.nz, ny = a.ny;
    const double* ba = a.bands;
    const double* bc = a.bands + 2 * ny;
    const double* ba0 = a.bands + 3 * ny;
    const double* bc0 = a.bands + 5 * ny;
    double2 p0[kPairsPerThread], p1[kPairsPerThread];
#pragma unroll
    for (int s = 0; s < kPairsPerThread; s++) { p0[s] = make_double2(0, 0); p1[s] = make_double2(0, 0); }

    for (int y = 0; y < ny; y++) {
        double2* row = a.X + ((size_t)y * a.nh + kx) * nz;
        for (int i = tid; i < nz; i += nthr) A[i] = row[i];
        __syncthreads();
        const double2* F = fft_rows<-1>(A, B, 1, nz, a.f, a.tw);
        const double* drow = a.piv + ((size_t)y * a.nh + kx) * a.mzp;
#pragma unroll
        for (int s = 0; s < kPairsPerThread; s++) {
            const int t = tid + s * nthr;
            if (t < a.nzh) {
                const bool is00 = (kx == 0 && t == 0);
                const bool two = (t > 0) && (2 * t != nz);
                const double D = drow[t];
                double2 v0 = F[t];
                double2 v1 = two ? F[nz - t] : make_double2(0, 0);
                if (y == 0) {
                    v0.x = __ddiv_rn(v0.x, D); v0.y = __ddiv_rn(v0.y, D);
                    v1.x = __ddiv_rn(v1.x, D); v1.y = __ddiv_rn(v1.y, D);
                } else {
                    const double av = is00 ? ba0[y] : ba[y];
                    v0.x = __ddiv_rn(__dsub_rn(v0.x, __dmul_rn(av, p0[s].x)), D);
                    v0.y = __ddiv_rn(__dsub_rn(v0.y, __dmul_rn(av, p0[s].y)), D);
                    v1.x = __ddiv_rn(__dsub_rn(v1.x, __dmul_rn(av, p1[s].x)), D);
                    v1.y = __ddiv_rn(__dsub_rn(v1.y, __dmul_rn(av, p1[s].y)), D);
                }
                p0[s] = v0; p1[s] = v1;
                if (y < ny - 1) {
                    row[t] = v0;
                    if (two) row[nz - t] = v1;
                }
            }
        }
        __syncthreads();
    }
    for (int y = ny - 1; y >= 0; y--) {
        double2* row = a.X + ((size_t)y * a.nh + kx) * nz;
        const double* drow = a.piv + ((size_t)y * a.nh + kx) * a.mzp;
#pragma unroll
        for (int s = 0; s < kPairsPerThread; s++) {
            const int t = tid + s * nthr;
            if (t < a.nzh) {
                const bool is00 = (kx == 0 && t == 0);
                const bool two = (t > 0) && (2 * t != nz);
                if (y < ny - 1) {
                    const double C = __ddiv_rn(is00 ? bc0[y] : bc[y], drow[t]);
                    const double2 d0 = row[t];
                    p0[s].x = __dsub_rn(d0.x, __dmul_rn(p0[s].x, C));
                    p0[s].y = __dsub_rn(d0.y, __dmul_rn(p0[s].y, C));
                    if (two) {
                        const double2 d1 = row[nz - t];
                        p1[s].x = __dsub_rn(d1.x, __dmul_rn(p1[s].x, C));
                        p1[s].y = __dsub_rn(d1.y, __dmul_rn(p1[s].y, C));
                    }
                }
                A[t] = p0[s];
                if (two) A[nz - t] = p1[s];
            }
        }
        __syncthreads();
        const double2* G = fft_rows<+1>(A, B, 1, nz, a.f, a.tw);
        for (int i = tid; i < nz; i += nthr) row[i] = G[i];
        __syncthreads();
    }
}

// Thomas pivots of every (kx, kzs) line, poisson_solver_multigpu.f90:164-179:
// D_0 = b_0 + lambda, D_k = (b_k + lambda) - a_k c'_{k-1}, c'_k = c_k / D_k.
// Also reduces min |D| (min_abs_div_bacp, :181-197) into *minpiv (as bits).
// minpiv[0] / minpiv[1] receive the smallest / largest |pivot| (as the bits of a
// non-negative double).  pivc (may be null): the back-substitution factors c'_y = c_y / D_y of every line, the
// quotients the backward sweep would otherwise form
__global__ void k_build_pivots(int nh, int nzh, int mzp, int ny, const double* __restrict__ bands,
                               const double* __restrict__ ax, const double* __restrict__ az, double* piv,
                               double* pivc, unsigned long long* minpiv) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int kx = gid / mzp, t = gid - kx * mzp;
    if (kx >= nh) return;
    if (t >= nzh) {  // padding slots
        for (int y = 0; y < ny; y++) {
            piv[((size_t)y * nh + kx) * mzp + t] = 1.0;
            if (pivc) pivc[((size_t)y * nh + kx) * mzp + t] = 0.0;
        }
        return;
    }
    const bool is00 = (kx == 0 && t == 0);
    const double* A = bands + (is00 ? 3 : 0) * ny;
    const double* Bb = bands + (is00 ? 4 : 1) * ny;
    const double* C = bands + (is00 ? 5 : 2) * ny;
    const double lam = __dadd_rn(ax[kx], az[t]);
    double D = __dadd_rn(Bb[0], lam);
    double cp = __ddiv_rn(C[0], D);
    double mn = fabs(D), mx = fabs(D);
    piv[((size_t)0 * nh + kx) * mzp + t] = D;
    if (pivc) pivc[((size_t)0 * nh + kx) * mzp + t] = cp;
    for (int y = 1; y < ny; y++) {
        D = __dsub_rn(__dadd_rn(Bb[y], lam), __dmul_rn(A[y], cp));
        cp = __ddiv_rn(C[y], D);
        mn = fmin(mn, fabs(D));
        mx = fmax(mx, fabs(D));
        piv[((size_t)y * nh + kx) * mzp + t] = D;
        if (pivc) pivc[((size_t)y * nh + kx) * mzp + t] = cp;
    }
    if (mn == mn) atomicMin(minpiv, (unsigned long long)__double_as_longlong(mn));
    else atomicMin(minpiv, 0ull);  // NaN pivot: report 0
    // the largest |pivot| (slot 1): the division of the forward sweeps needs every pivot
    // within [2^-40, 2^1000] (div_rn.cuh); an infinite or NaN pivot reports +inf
    atomicMax(minpiv + 1, (unsigned long long)__double_as_longlong(mx == mx ? mx : __longlong_as_double(0x7ff0000000000000ll)));
}

struct CorrArgs {
    int nx, nz, ny;
    const double* P;
    const double* Uh;
    const double* Vh;
    const double* Wh;
    const double* lo;
    const double* hi;
    double* U;
    double* V;
    double* W;
    double dt, inv_dx, inv_dz;
    double wall[6];
    int kh0;  // first halo'd plane of this launch (grid.x planes from kh0)
};

// u = u_hat - dt grad P on the whole halo'd box (mod_cfd_subroutines.f90:1124-1152);
// x/z halos take the periodic image (the halo exchange of :1225-1231), the
// y slices -1 and ny (and V at k = 0) take the wall values (:1234-1244).
__global__ void __launch_bounds__(128) k_correct(const CorrArgs a) {
    // one block per halo'd x-row (jh, kh): no index division, coalesced along x
    const int nx = a.nx, nz = a.nz, ny = a.ny;
    const int jh = blockIdx.y;
    const int k = (int)blockIdx.x + a.kh0 - 1;
    const size_t rowh = (size_t)(nx + 2) * ((size_t)jh + (size_t)(nz + 2) * (size_t)(k + 1));
    if (k < 0 || k == ny) {
        const double u = k < 0 ? a.wall[0] : a.wall[3];
        const double v = k < 0 ? a.wall[1] : a.wall[4];
        const double w = k < 0 ? a.wall[2] : a.wall[5];
        for (int ih = threadIdx.x; ih < nx + 2; ih += blockDim.x) {
            a.U[rowh + ih] = u;
            a.V[rowh + ih] = v;
            a.W[rowh + ih] = w;
        }
        return;
    }
    const int j = jh - 1;
    const int jw = j < 0 ? nz - 1 : (j == nz ? 0 : j);
    const int jm = jw == 0 ? nz - 1 : jw - 1;
    const double* P0 = a.P + ((size_t)k * nz + jw) * nx;
    const double* Pjm = a.P + ((size_t)k * nz + jm) * nx;
    const double* Pkm = a.P + ((size_t)(k > 0 ? k - 1 : 0) * nz + jw) * nx;
    const size_t roww = (size_t)(nx + 2) * ((size_t)(jw + 1) + (size_t)(nz + 2) * (size_t)(k + 1));
    const double hi = a.hi[k], lo = a.lo[k];
    for (int ih = threadIdx.x; ih < nx + 2; ih += blockDim.x) {
        const int i = ih - 1;
        const int iw = i < 0 ? nx - 1 : (i == nx ? 0 : i);
        const int im = iw == 0 ? nx - 1 : iw - 1;
        const double p0 = P0[iw];
        const size_t hw = roww + (size_t)(iw + 1);
        const double u = __dsub_rn(a.Uh[hw], __dmul_rn(__dmul_rn(a.dt, __dsub_rn(p0, P0[im])), a.inv_dx));
        const double w = __dsub_rn(a.Wh[hw], __dmul_rn(__dmul_rn(a.dt, __dsub_rn(p0, Pjm[iw])), a.inv_dz));
        double v = a.wall[1];
        if (k > 0) v = __dsub_rn(a.Vh[hw], __dmul_rn(a.dt, __dadd_rn(__dmul_rn(hi, p0), __dmul_rn(lo, Pkm[iw]))));
        a.U[rowh + ih] = u;
        a.V[rowh + ih] = v;
        a.W[rowh + ih] = w;
    }
}

// max |div u| over the interior (mod_get_bulk.f90:94-96) and max |P|
__global__ void k_stats(int nx, int nz, int ny, double inv_dx, double inv_dz, const double* __restrict__ inv_dy_p,
                        const double* __restrict__ U, const double* __restrict__ V, const double* __restrict__ W,
                        const double* __restrict__ P, unsigned long long* out) {
    double dmax = 0.0, pmax = 0.0;
    const size_t tot = (size_t)nx * nz * ny;
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < tot; idx += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % nx);
        const size_t r = idx / nx;
        const int j = (int)(r % nz);
        const int k = (int)(r / nz);
        const double d = (U[hidx(nx, nz, i + 1, j, k)] - U[hidx(nx, nz, i, j, k)]) * inv_dx +
                         (W[hidx(nx, nz, i, j + 1, k)] - W[hidx(nx, nz, i, j, k)]) * inv_dz +
                         (V[hidx(nx, nz, i, j, k + 1)] - V[hidx(nx, nz, i, j, k)]) * inv_dy_p[k];
        dmax = fmax(dmax, fabs(d));
        pmax = fmax(pmax, fabs(P[idx]));
    }
    for (int o = 16; o > 0; o >>= 1) {
        dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
        pmax = fmax(pmax, __shfl_xor_sync(0xffffffffu, pmax, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out + 0, (unsigned long long)__double_as_longlong(dmax));
        atomicMax(out + 1, (unsigned long long)__double_as_longlong(pmax));
    }
}

template <typename K>
cudaError_t set_smem(K kernel, size_t bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

}  // namespace

cudaError_t launch_fwd_x(const prj_plan* pl, FwdSource src, const double* P, const double* Uh, const double* Vh,
                         const double* Wh, const StepScalars* sc, cudaStream_t st) {
    if (pl->xd.ok) return launch_fwd_xd(pl, src, P, Uh, Vh, Wh, sc, st);
    const Geometry& g = pl->g;
    FwdArgs a{};
    a.nx = g.nx; a.nz = g.nz; a.ny = g.ny; a.nh = g.nxh;
    a.m = pl->fx64.m; a.tz = pl->tz_fwd; a.rs = pl->fx64.m + 1; a.even = pl->fx64.even;
    a.f = pl->fx64.f; a.tw = pl->fx64.tw; a.post = pl->fx64.post;
    a.P = P; a.Uh = Uh; a.Vh = Vh; a.Wh = Wh; a.inv_dy_p = pl->t.inv_dy_p;
    a.inv_dx = 1.0 / g.dx; a.inv_dz = 1.0 / g.dz;
    if (sc) { a.inv_dt = sc->inv_dt; a.vbot = sc->wall[1]; a.vtop = sc->wall[4]; }
    a.X = pl->spec;
    const size_t smem = (size_t)2 * a.tz * a.rs * sizeof(double2);
    dim3 grid((g.nz + a.tz - 1) / a.tz, g.ny);
    cudaError_t e;
    if (src == FwdSource::Pressure) {
        if ((e = set_smem(k_fwd_x<0>, smem)) != cudaSuccess) return e;
        k_fwd_x<0><<<grid, 256, smem, st>>>(a);
    } else {
        if ((e = set_smem(k_fwd_x<1>, smem)) != cudaSuccess) return e;
        k_fwd_x<1><<<grid, 256, smem, st>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t launch_bwd_x(const prj_plan* pl, double* P, cudaStream_t st) {
    if (pl->xd.ok) return launch_bwd_xd(pl, P, st);
    const Geometry& g = pl->g;
    BwdArgs a{};
    a.nx = g.nx; a.nz = g.nz; a.ny = g.ny; a.nh = g.nxh;
    a.m = pl->fx64.m; a.tz = pl->tz_fwd; a.rs = pl->fx64.m + 1; a.even = pl->fx64.even;
    a.f = pl->fx64.f; a.tw = pl->fx64.tw; a.post = pl->fx64.post;
    a.X = pl->spec; a.P = P;
    a.scale = 1.0 / ((double)g.nx * (double)g.nz + 0.0);
    const size_t smem = (size_t)2 * a.tz * a.rs * sizeof(double2);
    cudaError_t e = set_smem(k_bwd_x, smem);
    if (e != cudaSuccess) return e;
    dim3 grid((g.nz + a.tz - 1) / a.tz, g.ny);
    k_bwd_x<<<grid, 256, smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_zsolve(const prj_plan* pl, cudaStream_t st) {
    if (pl->zmode != 2) {
        cudaError_t ep = launch_zsolve_pipelined(pl, reinterpret_cast<int*>(pl->stat_buf + kStatErrSlot), st);
        if (ep != cudaErrorNotSupported) return ep;
    }
    const Geometry& g = pl->g;
    ZArgs a{};
    a.nz = g.nz; a.ny = g.ny; a.nh = g.nxh; a.nzh = g.nzh; a.mzp = g.mzp;
    a.f = pl->fz64.f; a.tw = pl->fz64.tw; a.bands = pl->t.bands; a.piv = pl->t.piv; a.X = pl->spec;
    int nthr = (g.nz + 3) / 4;
    nthr = ((nthr + 31) / 32) * 32;
    if (nthr < 64) nthr = 64;
    if (nthr > 512) nthr = 512;
    if (g.nzh > kPairsPerThread * nthr) return cudaErrorInvalidValue;
    const size_t smem = (size_t)2 * g.nz * sizeof(double2);
    cudaError_t e = set_smem(k_zsolve, smem);
    if (e != cudaSuccess) return e;
    k_zsolve<<<g.nxh, nthr, smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_build_pivots(const prj_plan* pl, cudaStream_t st) {
    const Geometry& g = pl->g;
    const int tot = g.nxh * g.mzp;
    unsigned long long* mp = reinterpret_cast<unsigned long long*>(pl->stat_buf);
    const double init[2] = {1e300, 0.0};  // running min and max of |pivot|
    cudaError_t e = cudaMemcpyAsync(mp, init, sizeof(init), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    k_build_pivots<<<(tot + 127) / 128, 128, 0, st>>>(g.nxh, g.nzh, g.mzp, g.ny, pl->t.bands, pl->t.ax, pl->t.az,
                                                      pl->t.piv, pl->t.pivc, mp);
    return cudaGetLastError();
}

cudaError_t launch_correction(const prj_plan* pl, const double* P, const double* Uh, const double* Vh,
                              const double* Wh, double* U, double* V, double* W, const StepScalars& sc,
                              cudaStream_t st, YRange kh) {
    const Geometry& g = pl->g;
    kh = kh.resolved(g.ny + 2);
    CorrArgs a{};
    a.kh0 = kh.y0;
    a.nx = g.nx; a.nz = g.nz; a.ny = g.ny;
    a.P = P; a.Uh = Uh; a.Vh = Vh; a.Wh = Wh; a.lo = pl->t.dpdy_lo; a.hi = pl->t.dpdy_hi;
    a.U = U; a.V = V; a.W = W;
    a.dt = sc.dt; a.inv_dx = 1.0 / g.dx; a.inv_dz = 1.0 / g.dz;
    for (int i = 0; i < 6; i++) a.wall[i] = sc.wall[i];
    if (kh.y1 <= kh.y0) return cudaSuccess;
    const dim3 grid((unsigned)(kh.y1 - kh.y0), (unsigned)(g.nz + 2));
    k_correct<<<grid, 128, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_stats(const prj_plan* pl, const double* U, const double* V, const double* W, const double* P,
                         double* out2, cudaStream_t st) {
    const Geometry& g = pl->g;
    cudaError_t e = cudaMemsetAsync(out2, 0, 2 * sizeof(double), st);
    if (e != cudaSuccess) return e;
    const size_t tot = (size_t)g.nx * g.nz * g.ny;
    size_t blocks = (tot + 255) / 256;
    const size_t cap = (size_t)sm_count() * 8;
    if (blocks > cap) blocks = cap;
    k_stats<<<(unsigned)blocks, 256, 0, st>>>(g.nx, g.nz, g.ny, 1.0 / g.dx, 1.0 / g.dz, pl->t.inv_dy_p, U, V, W, P,
                                             reinterpret_cast<unsigned long long*>(out2));
    return cudaGetLastError();
}

}  // namespace prj

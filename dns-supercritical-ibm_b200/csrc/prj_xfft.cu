// prj_xfft.cu -- x-direction real transforms with in-place DIF FFTs.
//
// k_fwd_xd: divergence of the predictor (or P itself) -> real FFT along x of
//           `tz` x-rows at one y -> transposed store X[y][kx][z0 .. z0+tz).
// k_bwd_xd: transposed load of X -> inverse real FFT along x, 1/(nx nz) ->
//           P rows.
// The real transform of even length n is a complex transform of length m = n/2
// on the packed samples x_2j + i x_2j+1 plus a split pass; odd n uses a
// complex transform of length n.  The in-place DIF transform (fft_dif.cuh)
// needs one row buffer per x-row, half of an out-of-place transform, so more
// CTAs fit on an SM.  Loads and stores of P and u_hat are one element per
// thread along x (fully coalesced).
#include "fft_dif.cuh"
#include "fft_pass.cuh"
#include "prj_internal.h"
#include "xfft_tiles.cuh"

// minimum resident CTAs per SM requested for the shared-memory FFT kernels
#ifndef PRJ_FFT_MINB
#define PRJ_FFT_MINB 4
#endif

namespace prj {

namespace {

// divergence at cell (i, j, k), mod_cfd_subroutines.f90:532-534 (periodic wrap in x and z,
// V_hat walls from the step parameters); reference operation order, no contraction
__device__ __forceinline__ double div_at(const XArgs& a, int i, int j, int k) {
    const int nx = a.nx, nz = a.nz;
    const int ip = (i + 1 == nx) ? 0 : i + 1;
    const int jp = (j + 1 == nz) ? 0 : j + 1;
    const double u1 = a.Uh[hidx_d(nx, nz, ip, j, k)], u0 = a.Uh[hidx_d(nx, nz, i, j, k)];
    const double w1 = a.Wh[hidx_d(nx, nz, i, jp, k)], w0 = a.Wh[hidx_d(nx, nz, i, j, k)];
    const double v1 = (k + 1 == a.ny) ? a.vtop : a.Vh[hidx_d(nx, nz, i, j, k + 1)];
    const double v0 = (k == 0) ? a.vbot : a.Vh[hidx_d(nx, nz, i, j, k)];
    double s = __dmul_rn(__dsub_rn(u1, u0), a.inv_dx);
    s = __dadd_rn(s, __dmul_rn(__dsub_rn(w1, w0), a.inv_dz));
    s = __dadd_rn(s, __dmul_rn(__dsub_rn(v1, v0), a.inv_dy_p[k]));
    return __dmul_rn(a.inv_dt, s);
}

// element g of the tz x rs row buffer lives at slot S(g) = g + g/8 (bank-conflict padding)
#define S(g) sidx<true>(g)

template <int SRC>
__global__ void __launch_bounds__(256, PRJ_FFT_MINB) k_fwd_xd(const XArgs a) {
    extern __shared__ __align__(16) unsigned char sm[];
    double2* A = reinterpret_cast<double2*>(sm);
    int* pos = reinterpret_cast<int*>(sm + (size_t)padded_len(a.tz * a.rs, true) * sizeof(double2));
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int y = a.y0 + (int)blockIdx.y, z0 = blockIdx.x * a.tz;
    const int m = a.m, nx = a.nx;
    for (int i = tid; i < m; i += nthr) pos[i] = a.pos[i];
    // kUnroll elements per thread per batch: their loads are independent and in flight together
    const int total = a.tz * nx;
    for (int base = tid; base < total; base += kUnroll * nthr) {
        double v[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
            const int idx = base + u * nthr;
            v[u] = 0.0;
            if (idx < total) {
                const int r = idx / nx, i = idx - r * nx;
                const int z = z0 + r;
                if (z < a.nz) {
                    v[u] = (SRC == 0) ? a.P[((size_t)y * a.nz + z) * nx + i] : div_at(a, i, z, y);
                    if (a.Bout) a.Bout[((size_t)y * a.nz + z) * nx + i] = v[u];
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
            const int idx = base + u * nthr;
            if (idx < total) {
                const int r = idx / nx, i = idx - r * nx;
                if (a.even) reinterpret_cast<double*>(A)[2 * S(r * a.rs + (i >> 1)) + (i & 1)] = v[u];
                else A[S(r * a.rs + i)] = make_double2(v[u], 0.0);
            }
        }
    }
    __syncthreads();
    inplace_rows<-1, false, true>(A, a.tz, a.rs, a.f, a.tw);
    if (a.even) {
        // split: X_k = E_k + W^k O_k and X_{m-k} = conj(E_k) + W^{m-k} conj(O_k), in place
        const int half = m / 2;
        // row index fastest: the rows are rs (odd) slots apart, so a warp's
        // digit-reversed gathers land in distinct bank groups
        for (int idx = tid; idx < a.tz * (half + 1); idx += nthr) {
            const int k = idx / a.tz, r = idx - k * a.tz;
            const int base = r * a.rs;
            if (k == 0) {
                const double2 z = A[S(base + pos[0])];
                A[S(base + pos[0])] = make_double2(z.x + z.y, 0.0);
                A[S(base + m)] = make_double2(z.x - z.y, 0.0);
            } else {
                const int kk = m - k;
                const double2 zk = A[S(base + pos[k])];
                const double2 zm = cconj(A[S(base + pos[kk])]);
                const double2 e = cscale(cadd(zk, zm), 0.5);
                const double2 d = csub(zk, zm);
                const double2 o = make_double2(0.5 * d.y, -0.5 * d.x);
                A[S(base + pos[k])] = cadd(e, cmul(a.post[k], o));
                if (kk != k) A[S(base + pos[kk])] = cadd(cconj(e), cmul(a.post[kk], cconj(o)));
            }
        }
        __syncthreads();
    }
    for (int idx = tid; idx < a.nh * a.tz; idx += nthr) {
        const int kx = idx / a.tz, r = idx - kx * a.tz;
        const int z = z0 + r;
        if (z >= a.nz) continue;
        const int slot = (a.even && kx == m) ? m : pos[kx];
        spec_store(a, y, kx, z, A[S(r * a.rs + slot)]);
    }
}

__global__ void __launch_bounds__(256, PRJ_FFT_MINB) k_bwd_xd(const XArgs a) {
    extern __shared__ __align__(16) unsigned char sm[];
    double2* A = reinterpret_cast<double2*>(sm);
    int* pos = reinterpret_cast<int*>(sm + (size_t)padded_len(a.tz * a.rs, true) * sizeof(double2));
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int y = a.y0 + (int)blockIdx.y, z0 = blockIdx.x * a.tz;
    const int m = a.m, nx = a.nx;
    for (int i = tid; i < m; i += nthr) pos[i] = a.pos[i];
    const int total = a.nh * a.tz;
    for (int base = tid; base < total; base += kUnroll * nthr) {
        double2 v[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
            const int idx = base + u * nthr;
            v[u] = make_double2(0.0, 0.0);
            if (idx < total) {
                const int kx = idx / a.tz, r = idx - kx * a.tz;
                const int z = z0 + r;
                if (z < a.nz) v[u] = spec_load(a, y, kx, z);
            }
        }
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
            const int idx = base + u * nthr;
            if (idx < total) {
                const int kx = idx / a.tz, r = idx - kx * a.tz;
                A[S(r * a.rs + kx)] = v[u];
            }
        }
    }
    __syncthreads();
    const double s = a.scale;
    if (a.even) {
        // inverse split, in place on pairs (k, m-k); imaginary parts of X_0 and X_m ignored
        const int half = m / 2;
        for (int idx = tid; idx < a.tz * (half + 1); idx += nthr) {
            const int r = idx / (half + 1), k = idx - r * (half + 1);
            const int base = r * a.rs;
            if (k == 0) {
                const double x0 = A[S(base)].x, xm = A[S(base + m)].x;
                A[S(base)] = make_double2((x0 + xm) * s, (x0 - xm) * s);
            } else {
                const int kk = m - k;
                const double2 xk = A[S(base + k)], xkk = A[S(base + kk)];
                const double2 e1 = cadd(xk, cconj(xkk));
                const double2 o1 = cmulc(csub(xk, cconj(xkk)), a.post[k]);
                A[S(base + k)] = cscale(make_double2(e1.x - o1.y, e1.y + o1.x), s);
                if (kk != k) {
                    const double2 e2 = cadd(xkk, cconj(xk));
                    const double2 o2 = cmulc(csub(xkk, cconj(xk)), a.post[kk]);
                    A[S(base + kk)] = cscale(make_double2(e2.x - o2.y, e2.y + o2.x), s);
                }
            }
        }
    } else {
        // Hermitian completion of the odd-length row, scaled
        for (int idx = tid; idx < a.tz * a.nh; idx += nthr) {
            const int r = idx / a.nh, k = idx - r * a.nh;
            const int base = r * a.rs;
            double2 v = A[S(base + k)];
            if (k == 0) v.y = 0.0;
            v = cscale(v, s);
            A[S(base + k)] = v;
            if (k > 0) A[S(base + m - k)] = cconj(v);
        }
    }
    __syncthreads();
    inplace_rows<+1, false, true>(A, a.tz, a.rs, a.f, a.tw);
    // x fastest: fully coalesced row stores (measured faster here than conflict-free
    // row-fastest gathers with sector-sized stores)
    double sq0 = 0.0, sq1 = 0.0;
    for (int idx = tid; idx < a.tz * nx; idx += nthr) {
        const int r = idx / nx, i = idx - r * nx;
        const int z = z0 + r;
        if (z >= a.nz) continue;
        double v;
        if (a.even) {
            const double2 c = A[S(r * a.rs + pos[i >> 1])];
            v = (i & 1) ? c.y : c.x;
        } else {
            v = A[S(r * a.rs + pos[i])].x;
        }
        double* out = a.Pout + ((size_t)y * a.nz + z) * nx + i;
        if (a.accum) {
            const double nv = *out + v;
            sq0 += v * v;
            sq1 += nv * nv;
            *out = nv;
        } else {
            *out = v;
        }
    }
    if (a.sq) {
        for (int o = 16; o > 0; o >>= 1) {
            sq0 += __shfl_xor_sync(0xffffffffu, sq0, o);
            sq1 += __shfl_xor_sync(0xffffffffu, sq1, o);
        }
        if ((tid & 31) == 0) {
            atomicAdd(a.sq, sq0);
            atomicAdd(a.sq + 1, sq1);
        }
    }
}

// ---------------------------------------------------------------------------
// Pass-plan x kernels (fft_pass.cuh), m = nx/2 with a compile-time plan PL.
// Rows at stride pass_row_stride(m) in shared memory.  nr = rows present in this
// CTA (the last CTA may hold fewer).

// k_fwd_xp / k_bwd_xp: one CTA per tile of the pass-plan x transforms (xfft_tiles.cuh)
template <int SRC, class PL>
__global__ void __launch_bounds__(kPassThreads, PRJ_PASS_MINB) k_fwd_xp(const XArgs a) {
    extern __shared__ __align__(16) unsigned char sm[];
    fwd_xp_tile<SRC, PL>(a, sm, blockIdx.x, blockIdx.y);
}

template <class PL>
__global__ void __launch_bounds__(kPassThreads, PRJ_PASS_MINB) k_bwd_xp(const XArgs a) {
    extern __shared__ __align__(16) unsigned char sm[];
    bwd_xp_tile<PL>(a, sm, blockIdx.x, blockIdx.y, gridDim.x);
}

XArgs make_args(const prj_plan* pl) {
    const Geometry& g = pl->g;
    XArgs a{};
    a.nx = g.nx; a.nz = g.nz; a.ny = g.ny; a.nh = g.nxh;
    a.m = pl->fx64.m; a.even = pl->fx64.even;
    a.tz = pl->tz_xd;
    a.rs = a.even ? a.m + 1 : a.m;
    a.f = pl->xd.f; a.tw = pl->xd.tw; a.pos = pl->xd.pos; a.post = pl->fx64.post;
    a.inv_dx = 1.0 / g.dx; a.inv_dz = 1.0 / g.dz;
    a.X = pl->spec;
    a.X32 = pl->spec32;
    a.kxs = pl->kxs;
    return a;
}

}  // namespace

XArgs batch_x_args(const prj_plan* pl, double* P) {
    XArgs a = make_args(pl);
    a.tz = pl->tz_xp;
    a.y0 = 0;
    a.P = P;
    a.Pout = P;
    a.scale = 1.0 / ((double)pl->g.nx * (double)pl->g.nz + 0.0);
    return a;
}

namespace {

size_t smem_bytes(const XArgs& a) {
    return (size_t)padded_len(a.tz * a.rs, true) * sizeof(double2) + (size_t)a.m * sizeof(int);
}

template <typename K>
cudaError_t allow_smem(K kernel, size_t bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace

// CTAs per y plane of the pass-plan inverse x kernel (the width of its partial sums)
int bwd_tiles_per_plane(const prj_plan* pl) { return (pl->g.nz + pl->tz_xp - 1) / pl->tz_xp; }

// rows per CTA of the pass-plan x kernels: a power of two up to 16 whose padded rows
// (stride pass_row_stride(m)) fit 32 KB, so that 6 CTAs share an SM
int choose_tz_xp(int m) {
    int tz = 16;
    while (tz > 1 && (size_t)padded_len(tz * pass_row_stride(m), true) * sizeof(double2) > 32 * 1024) tz /= 2;
    return tz;
}

size_t pass_x_smem(int m, int tz) { return (size_t)padded_len(tz * pass_row_stride(m), true) * sizeof(double2); }

// rows per CTA of the in-place x kernels: a power of two up to 16 within ~56 KB
int choose_tz_xd(int m, bool even) {
    const int rs = even ? m + 1 : m;
    int tz = 16;
    while (tz > 1 && (size_t)padded_len(tz * rs, true) * sizeof(double2) + (size_t)m * sizeof(int) > 56 * 1024) tz /= 2;
    return tz;
}

namespace {

inline bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

size_t pass_smem_bytes(const XArgs& a) {
    return (size_t)padded_len(a.tz * pass_row_stride(a.m), true) * sizeof(double2);
}

template <class PL>
cudaError_t launch_fwd_xp_pl(const XArgs& a, FwdSource src, const dim3& grid, cudaStream_t st) {
    const size_t smem = pass_smem_bytes(a);
    cudaError_t e;
    if (src == FwdSource::Pressure) {
        if ((e = allow_smem(k_fwd_xp<0, PL>, smem)) != cudaSuccess) return e;
        k_fwd_xp<0, PL><<<grid, kPassThreads, smem, st>>>(a);
    } else if (src == FwdSource::Residual) {
        if ((e = allow_smem(k_fwd_xp<3, PL>, smem)) != cudaSuccess) return e;
        k_fwd_xp<3, PL><<<grid, kPassThreads, smem, st>>>(a);
    } else {
        if ((e = allow_smem(k_fwd_xp<1, PL>, smem)) != cudaSuccess) return e;
        k_fwd_xp<1, PL><<<grid, kPassThreads, smem, st>>>(a);
    }
    return cudaGetLastError();
}

template <class PL>
cudaError_t launch_bwd_xp_pl(const XArgs& a, const dim3& grid, cudaStream_t st) {
    const size_t smem = pass_smem_bytes(a);
    cudaError_t e = allow_smem(k_bwd_xp<PL>, smem);
    if (e != cudaSuccess) return e;
    k_bwd_xp<PL><<<grid, kPassThreads, smem, st>>>(a);
    return cudaGetLastError();
}

// pass-plan x kernels for even nx whose half length has a pass plan built with the
// same radices; cudaErrorNotSupported otherwise (the caller uses the runtime-radix kernels)
cudaError_t launch_xpass(const prj_plan* pl, bool fwd, FwdSource src, XArgs a, int ny_launch, cudaStream_t st) {
    if (!pl->use_pass || !a.even) return cudaErrorNotSupported;
    a.tz = pl->tz_xp;
    const dim3 grid((pl->g.nz + a.tz - 1) / a.tz, ny_launch);
#define PRJ_X_CASE(N, ...)                                                                          \
    if (a.m == N && same_radices<PassList<__VA_ARGS__>>(pl->xd.f)) {                                \
        using PL = PassList<__VA_ARGS__>;                                                           \
        return fwd ? launch_fwd_xp_pl<PL>(a, src, grid, st) : launch_bwd_xp_pl<PL>(a, grid, st);    \
    }
    PRJ_PASS_ALL(PRJ_X_CASE)
#undef PRJ_X_CASE
    return cudaErrorNotSupported;
}

}  // namespace

cudaError_t launch_fwd_xd(const prj_plan* pl, FwdSource src, const double* P, const double* Uh, const double* Vh,
                          const double* Wh, const StepScalars* sc, cudaStream_t st, double* bout, YRange yr) {
    XArgs a = make_args(pl);
    yr = yr.resolved(pl->g.ny);
    a.y0 = yr.y0;
    a.Bout = bout;
    a.P = P; a.Uh = Uh; a.Vh = Vh; a.Wh = Wh; a.inv_dy_p = pl->t.inv_dy_p;
    if (sc) { a.inv_dt = sc->inv_dt; a.vbot = sc->wall[1]; a.vtop = sc->wall[4]; }
    if (src == FwdSource::Divergence || (aligned16(P) && aligned16(bout))) {
        const cudaError_t e = launch_xpass(pl, true, src, a, yr.y1 - yr.y0, st);
        if (e != cudaErrorNotSupported) return e;
    }
    const size_t smem = smem_bytes(a);
    const dim3 grid((pl->g.nz + a.tz - 1) / a.tz, yr.y1 - yr.y0);
    cudaError_t e;
    if (src == FwdSource::Pressure) {
        if ((e = allow_smem(k_fwd_xd<0>, smem)) != cudaSuccess) return e;
        k_fwd_xd<0><<<grid, 256, smem, st>>>(a);
    } else {
        if ((e = allow_smem(k_fwd_xd<1>, smem)) != cudaSuccess) return e;
        k_fwd_xd<1><<<grid, 256, smem, st>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t launch_fwd_residual(const prj_plan* pl, const double* B, const double* P, const double* pbar,
                                cudaStream_t st) {
    if (!aligned16(B) || !aligned16(P)) return cudaErrorNotSupported;
    XArgs a = make_args(pl);
    a.y0 = 0;
    a.P = P;
    a.B = B;
    a.pm = pbar;
    a.bands = pl->t.bands;
    a.idx2 = 1.0 / (pl->g.dx * pl->g.dx);
    a.idz2 = 1.0 / (pl->g.dz * pl->g.dz);
    return launch_xpass(pl, true, FwdSource::Residual, a, pl->g.ny, st);
}

cudaError_t launch_bwd_xd(const prj_plan* pl, double* P, cudaStream_t st, int accum, double* sq, YRange yr,
                          double* psum) {
    XArgs a = make_args(pl);
    a.psum = psum;
    yr = yr.resolved(pl->g.ny);
    a.y0 = yr.y0;
    a.Pout = P;
    a.accum = accum;
    a.sq = sq;
    a.scale = 1.0 / ((double)pl->g.nx * (double)pl->g.nz + 0.0);
    if (aligned16(P)) {
        const cudaError_t e2 = launch_xpass(pl, false, FwdSource::Pressure, a, yr.y1 - yr.y0, st);
        if (e2 != cudaErrorNotSupported) return e2;
    }
    if (psum) return cudaErrorNotSupported;  // partial sums come from the pass-plan kernel only
    const size_t smem = smem_bytes(a);
    cudaError_t e = allow_smem(k_bwd_xd, smem);
    if (e != cudaSuccess) return e;
    const dim3 grid((pl->g.nz + a.tz - 1) / a.tz, yr.y1 - yr.y0);
    k_bwd_xd<<<grid, 256, smem, st>>>(a);
    return cudaGetLastError();
}

#undef S

}  // namespace prj

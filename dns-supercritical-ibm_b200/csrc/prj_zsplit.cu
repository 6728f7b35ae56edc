// prj_zsplit.cu -- the z direction as three throughput kernels.
//
//   k_zfft_fwd : every spectral row X[y][kx][:] (natural z order) -> in-place
//                DIF FFT -> stored back in the transform's slot order
//                (wavenumber kz at slot pos[kz]);
//   k_thomas   : one thread per (kx, slot) line, streaming over y: forward
//                sweep d'_y = (d_y - a_y d'_{y-1}) / D_y, backward sweep
//                x_y = d'_y - c'_y x_{y+1} with c'_y = c_y / D_y tabulated with the
//                pivots, in place, rows prefetched into registers kBlock planes at
//                a time;
//   k_zfft_inv : slot-order rows -> in-place DIT inverse FFT -> natural z.
//
// Compared with one fused per-kx kernel this moves the spectrum through HBM
// four more times, but every kernel has thousands of CTAs, so the FP64 FFT
// work and the sequential Thomas chains are spread over the whole GPU instead
// of nx/2+1 CTAs.  The Thomas arithmetic keeps the reference's operation order
// and rounding (poisson_solver_multigpu.f90:401-419) with pivots D from the
// plan's table (the pair kz, nz-kz shares one pivot row entry).
#include <cstdlib>

#include "div_rn.cuh"
#include "fft_pass.cuh"
#include "prj_internal.h"
#include "zsplit_tiles.cuh"

// minimum resident CTAs per SM requested for the shared-memory FFT kernels
#ifndef PRJ_FFT_MINB
#define PRJ_FFT_MINB 4
#endif

namespace prj {

namespace {

template <typename K>
cudaError_t allow_smem(K kernel, size_t bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}


// T: storage type of the spectrum rows (arithmetic is FP64 in shared memory)
template <int DIR, typename T>
__global__ void __launch_bounds__(256, PRJ_FFT_MINB) k_zfft(const ZfftArgs a) {
    extern __shared__ __align__(16) double2 zs[];
    const int tid = threadIdx.x, nthr = blockDim.x;
    const size_t row0 = (size_t)blockIdx.x * a.rb;
    const int nr = (int)min((size_t)a.rb, (size_t)a.nrow_total - row0);
    const int tot = nr * a.nz;
    const T* src = static_cast<const T*>(a.X) + row0 * a.nz;
    constexpr int U = 4;
    for (int base = tid; base < tot; base += U * nthr) {
        double2 v[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int i = base + u * nthr;
            if (i < tot) v[u] = to_d2(src[i]);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int i = base + u * nthr;
            if (i < tot) zs[sidx<true>(i)] = v[u];
        }
    }
    __syncthreads();
    if (DIR < 0) inplace_rows<-1, false, true>(zs, nr, a.nz, a.f, a.tw);
    else inplace_rows<+1, true, true>(zs, nr, a.nz, a.f, a.tw);
    T* dst = static_cast<T*>(a.X) + row0 * a.nz;
    for (int i = tid; i < tot; i += nthr) from_d2(dst[i], zs[sidx<true>(i)]);
}

// k_zfft_pass: one CTA per group of rb rows (zsplit_tiles.cuh)
template <int DIR, typename T, class PL, bool STAGE_INV = false>
__global__ void __launch_bounds__(kPassThreads, PRJ_ZPASS_MINB) k_zfft_pass(const ZfftArgs a) {
    extern __shared__ __align__(16) double2 zp[];
    zfft_pass_tile<DIR, T, PL, STAGE_INV>(a, zp, blockIdx.x);
}


template <typename T>
__global__ void __launch_bounds__(kThomasTile) k_thomas(const ThomasArgs a) {
    thomas_line<T>(a, blockIdx.x);
}

template <typename T, int B, int NS>
__global__ void __launch_bounds__(kThomasTile) k_thomas_async(const ThomasArgs a) {
    extern __shared__ __align__(16) unsigned char tsm[];
    thomas_line_async<T, B, NS>(a, blockIdx.x, tsm);
}

template <int B, int NS>
__global__ void __launch_bounds__(kThomasTile) k_thomas_mixed_async(const ThomasArgs a64, const ThomasArgs a32,
                                                                    int nblk64) {
    extern __shared__ __align__(16) unsigned char tsm[];
    if ((int)blockIdx.x < nblk64) thomas_line_async<double2, B, NS>(a64, blockIdx.x, tsm);
    else thomas_line_async<float2, B, NS>(a32, blockIdx.x - nblk64, tsm);
}

template <typename T, int B, int NS>
cudaError_t launch_thomas_async(const ThomasArgs& t, unsigned grid, cudaStream_t st) {
    constexpr size_t smem = thomas_async_smem<T, B, NS>();
    const cudaError_t e = allow_smem(k_thomas_async<T, B, NS>, smem);
    if (e != cudaSuccess) return e;
    k_thomas_async<T, B, NS><<<grid, kThomasTile, smem, st>>>(t);
    return cudaGetLastError();
}

template <int B, int NS>
cudaError_t launch_thomas_mixed_async(const ThomasArgs& a64, const ThomasArgs& a32, int nblk64, unsigned grid,
                                      cudaStream_t st) {
    constexpr size_t smem = thomas_async_smem<double2, B, NS>();
    const cudaError_t e = allow_smem(k_thomas_mixed_async<B, NS>, smem);
    if (e != cudaSuccess) return e;
    k_thomas_mixed_async<B, NS><<<grid, kThomasTile, smem, st>>>(a64, a32, nblk64);
    return cudaGetLastError();
}

// mixed storage in one launch: blocks [0, nblk64) solve the FP64 rows (a64), the
// rest the FP32 rows (a32), so the few FP64 rows overlap the FP32 ones
__global__ void __launch_bounds__(kThomasTile) k_thomas_mixed(const ThomasArgs a64, const ThomasArgs a32,
                                                              int nblk64) {
    if ((int)blockIdx.x < nblk64) thomas_line<double2>(a64, blockIdx.x);
    else thomas_line<float2>(a32, blockIdx.x - nblk64);
}

}  // namespace

// rows per CTA of the pass-plan kernels: the requested count, else the largest
// power of two up to 32 whose padded rows fit 28 KB (7-8 CTAs per SM)
inline int pass_rows(int n, int requested, size_t limit_req = (size_t)200 * 1024) {
    int rb = requested > 0 ? requested : 32;
    const size_t limit = requested > 0 ? limit_req : (size_t)28 * 1024;
    while (rb > 1 && (size_t)padded_len(rb * n, true) * sizeof(double2) > limit) rb /= 2;
    return rb;
}

template <int DIR, typename T, class PL>
cudaError_t launch_zfft_pass_pl(ZfftArgs a, int rows_req, cudaStream_t st) {
    a.rb = pass_rows(PL::n, rows_req);
    const size_t smem = (size_t)padded_len(a.rb * PL::n, true) * sizeof(double2);
    const unsigned grid = (unsigned)((a.nrow_total + a.rb - 1) / a.rb);
    if (grid == 0) return cudaSuccess;
    // the inverse stages its slot-order rows through shared memory (coalesced copy-in;
    // measured at 768x384x384: 0.33 ms staged against 0.37 ms reading them in the first
    // pass; 0.093 / 0.113 ms at 512x256x256)
    if (DIR > 0) {
        cudaError_t e = allow_smem(k_zfft_pass<DIR, T, PL, true>, smem);
        if (e != cudaSuccess) return e;
        k_zfft_pass<DIR, T, PL, true><<<grid, kPassThreads, smem, st>>>(a);
        return cudaGetLastError();
    }
    cudaError_t e = allow_smem(k_zfft_pass<DIR, T, PL>, smem);
    if (e != cudaSuccess) return e;
    k_zfft_pass<DIR, T, PL><<<grid, kPassThreads, smem, st>>>(a);
    return cudaGetLastError();
}

// pass-plan z transform of one buffer; cudaErrorNotSupported when nz has no pass
// plan (or the plan was built with other radices)
template <typename T>
cudaError_t launch_zfft_pass(const prj_plan* pl, int dir, void* X, int rows_per_plane, cudaStream_t st, int nplanes = -1) {
    if (!pl->use_pass) return cudaErrorNotSupported;
    const Geometry& g = pl->g;
    ZfftArgs a{};
    a.nrow_total = (nplanes < 0 ? g.ny : nplanes) * rows_per_plane;
    a.nz = g.nz;
    a.f = pl->zd.f;
    a.tw = pl->zd.tw;
    a.X = X;
#define PRJ_Z_CASE(N, ...)                                                                    \
    if (g.nz == N && same_radices<PassList<__VA_ARGS__>>(pl->zd.f)) {                         \
        using PL = PassList<__VA_ARGS__>;                                                     \
        return dir < 0 ? launch_zfft_pass_pl<-1, T, PL>(a, pl->zfft_rows, st)                 \
                       : launch_zfft_pass_pl<+1, T, PL>(a, pl->zfft_rows, st);                \
    }
    PRJ_PASS_ALL(PRJ_Z_CASE)
#undef PRJ_Z_CASE
    return cudaErrorNotSupported;
}

// in-place z FFT of every spectral row of one buffer: dir < 0 forward (natural ->
// slot order), dir > 0 inverse (slot order -> natural); needs pl->zd.ok.
// `rows_per_plane` rows of T storage per y plane.
template <typename T>
cudaError_t launch_zfft_t(const prj_plan* pl, int dir, void* X, int rows_per_plane, cudaStream_t st) {
    {
        const cudaError_t e = launch_zfft_pass<T>(pl, dir, X, rows_per_plane, st);
        if (e != cudaErrorNotSupported) return e;
    }
    const Geometry& g = pl->g;
    ZfftArgs a{};
    a.nrow_total = g.ny * rows_per_plane;
    a.nz = g.nz;
    a.f = pl->zd.f;
    a.tw = pl->zd.tw;
    a.X = X;
    int rb = pl->zfft_rows > 0 ? pl->zfft_rows : 16;
    const size_t limit = pl->zfft_rows > 0 ? (size_t)200 * 1024 : (size_t)48 * 1024;
    while (rb > 1 && (size_t)padded_len(rb * g.nz, true) * sizeof(double2) > limit) rb /= 2;
    a.rb = rb;
    const size_t smem = (size_t)padded_len(rb * g.nz, true) * sizeof(double2);
    const unsigned grid = (unsigned)((a.nrow_total + rb - 1) / rb);
    if (grid == 0) return cudaSuccess;
    cudaError_t e;
    if (dir < 0) {
        if ((e = allow_smem(k_zfft<-1, T>, smem)) != cudaSuccess) return e;
        k_zfft<-1, T><<<grid, 256, smem, st>>>(a);
    } else {
        if ((e = allow_smem(k_zfft<+1, T>, smem)) != cudaSuccess) return e;
        k_zfft<+1, T><<<grid, 256, smem, st>>>(a);
    }
    return cudaGetLastError();
}

int batch_z_default_rows(int nz) { return pass_rows(nz, 0); }

ZfftArgs batch_z_args(const prj_plan* pl) {
    const Geometry& g = pl->g;
    ZfftArgs a{};
    a.nrow_total = g.ny * g.nxh;
    a.nz = g.nz;
    a.f = pl->zd.f;
    a.tw = pl->zd.tw;
    a.X = pl->spec;
    a.rb = pass_rows(g.nz, pl->zfft_rows);
    return a;
}

ThomasArgs thomas_args(const prj_plan* pl, void* X, int kx0, int rows_per_plane) {
    const Geometry& g = pl->g;
    ThomasArgs t{};
    t.nz = g.nz; t.ny = g.ny; t.nh = g.nxh; t.mzp = g.mzp;
    t.tiles = (g.nz + kThomasTile - 1) / kThomasTile;
    t.nhb = rows_per_plane; t.kx0 = kx0;
    t.bands = pl->t.bands; t.piv = pl->t.piv; t.pivc = pl->t.pivc; t.kz_of_slot = pl->kz_of_slot; t.X = X;
    return t;
}

template <typename T>
cudaError_t launch_thomas_t(const prj_plan* pl, void* X, int kx0, int rows_per_plane, cudaStream_t st) {
    if (rows_per_plane <= 0) return cudaSuccess;
    if (!pl->t.piv || !pl->t.pivc) return cudaErrorInvalidValue;
    const ThomasArgs t = thomas_args(pl, X, kx0, rows_per_plane);
    const unsigned grid = (unsigned)(rows_per_plane * t.tiles);
    switch (pl->thomas_async > 0 ? pl->thomas_async : 0) {
    case 1: return launch_thomas_async<T, 4, 4>(t, grid, st);
    case 2: return launch_thomas_async<T, 8, 2>(t, grid, st);
    case 3: return launch_thomas_async<T, 2, 8>(t, grid, st);
    case 4: return launch_thomas_async<T, 8, 3>(t, grid, st);
    default: break;
    }
    k_thomas<T><<<grid, kThomasTile, 0, st>>>(t);
    return cudaGetLastError();
}

cudaError_t launch_zfft(const prj_plan* pl, int dir, cudaStream_t st, YRange yr) {
    yr = yr.resolved(pl->g.ny);
    if (yr.y0 == 0 && yr.y1 == pl->g.ny) return launch_zfft_t<double2>(pl, dir, pl->spec, pl->g.nxh, st);
    // a y range (one rank's planes of the distributed solve): the pass-plan kernel only
    double2* X = pl->spec + (size_t)yr.y0 * pl->g.nxh * pl->g.nz;
    return launch_zfft_pass<double2>(pl, dir, X, pl->g.nxh, st, yr.y1 - yr.y0);
}

cudaError_t launch_thomas(const prj_plan* pl, cudaStream_t st) {
    return launch_thomas_t<double2>(pl, pl->spec, 0, pl->g.nxh, st);
}

cudaError_t launch_thomas_rows(const prj_plan* pl, double2* X, int kx0, int rows, cudaStream_t st) {
    return launch_thomas_t<double2>(pl, X, kx0, rows, st);
}

// mixed storage: FP64 rows kx < kxs in pl->spec (kxs rows per plane), FP32 rows in pl->spec32
cudaError_t launch_zfft_mixed(const prj_plan* pl, int dir, cudaStream_t st) {
    cudaError_t e = launch_zfft_t<double2>(pl, dir, pl->spec, pl->kxs, st);
    if (e != cudaSuccess) return e;
    return launch_zfft_t<float2>(pl, dir, pl->spec32, pl->g.nxh - pl->kxs, st);
}

cudaError_t launch_thomas_mixed(const prj_plan* pl, cudaStream_t st) {
    if (!pl->t.piv || !pl->t.pivc) return cudaErrorInvalidValue;
    const int rows32 = pl->g.nxh - pl->kxs;
    if (rows32 <= 0) return launch_thomas_t<double2>(pl, pl->spec, 0, pl->kxs, st);
    const ThomasArgs a64 = thomas_args(pl, pl->spec, 0, pl->kxs);
    const ThomasArgs a32 = thomas_args(pl, pl->spec32, pl->kxs, rows32);
    const int nblk64 = pl->kxs * a64.tiles;
    const unsigned grid = (unsigned)(nblk64 + rows32 * a32.tiles);
    // the mixed storage streams by default (measured 0.69 ms against 1.10 ms per solve at
    // 768x384x384); thomas_ring 0 keeps the register-prefetch kernel
    switch (pl->thomas_async) {
    case 0: break;
    case 2: return launch_thomas_mixed_async<8, 2>(a64, a32, nblk64, grid, st);
    case 3: return launch_thomas_mixed_async<2, 8>(a64, a32, nblk64, grid, st);
    case 4: return launch_thomas_mixed_async<8, 3>(a64, a32, nblk64, grid, st);
    default: return launch_thomas_mixed_async<4, 4>(a64, a32, nblk64, grid, st);
    }
    k_thomas_mixed<<<grid, kThomasTile, 0, st>>>(a64, a32, nblk64);
    return cudaGetLastError();
}

}  // namespace prj

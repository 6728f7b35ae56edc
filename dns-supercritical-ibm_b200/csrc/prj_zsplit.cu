// prj_zsplit.cu -- the z direction as three throughput kernels.
//
//   k_zfft_fwd : every spectral row X[y][kx][:] (natural z order) -> in-place
//                DIF FFT -> stored back in the transform's slot order
//                (wavenumber kz at slot pos[kz]);
//   k_thomas   : one thread per (kx, slot) line, streaming over y: forward
//                sweep d'_y = (d_y - a_y d'_{y-1}) / D_y, backward sweep
//                x_y = d'_y - (c_y / D_y) x_{y+1}, in place, rows prefetched
//                into registers kBlock planes at a time;
//   k_zfft_inv : slot-order rows -> in-place DIT inverse FFT -> natural z.
//
// Compared with one fused per-kx kernel this moves the spectrum through HBM
// four more times, but every kernel has thousands of CTAs, so the FP64 FFT
// work and the sequential Thomas chains are spread over the whole GPU instead
// of nx/2+1 CTAs.  The Thomas arithmetic keeps the reference's operation order
// and rounding (poisson_solver_multigpu.f90:401-419) with pivots D from the
// plan's table (the pair kz, nz-kz shares one pivot row entry).
#include "prj_internal.h"

// minimum resident CTAs per SM requested for the shared-memory FFT kernels
#ifndef PRJ_FFT_MINB
#define PRJ_FFT_MINB 4
#endif

namespace prj {

namespace {

struct ZfftArgs {
    int nrow_total;  // ny * nxh rows of length nz
    int nz, rb;      // rows per CTA
    DifDev f;
    const double2* tw;
    double2* X;
};

template <int DIR>
__global__ void __launch_bounds__(256, PRJ_FFT_MINB) k_zfft(const ZfftArgs a) {
    extern __shared__ __align__(16) double2 zs[];
    const int tid = threadIdx.x, nthr = blockDim.x;
    const size_t row0 = (size_t)blockIdx.x * a.rb;
    const int nr = (int)min((size_t)a.rb, (size_t)a.nrow_total - row0);
    const int tot = nr * a.nz;
    const double2* src = a.X + row0 * a.nz;
    constexpr int U = 4;
    for (int base = tid; base < tot; base += U * nthr) {
        double2 v[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int i = base + u * nthr;
            if (i < tot) v[u] = src[i];
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
    double2* dst = a.X + row0 * a.nz;
    for (int i = tid; i < tot; i += nthr) dst[i] = zs[sidx<true>(i)];
}

struct ThomasArgs {
    int nz, ny, nh, mzp, tiles;  // tiles of kThomasTile slots per kx
    const double* bands;         // a, b, c, a00, b00, c00
    const double* piv;           // D[y][kx][kzs]
    const int* kz_of_slot;       // wavenumber held by each slot
    double2* X;
};

constexpr int kThomasTile = 128;
constexpr int kBlock = 8;  // planes loaded together (independent loads in flight)

__global__ void __launch_bounds__(kThomasTile) k_thomas(const ThomasArgs a) {
    const int kx = blockIdx.x / a.tiles;
    const int slot = (blockIdx.x - kx * a.tiles) * kThomasTile + threadIdx.x;
    if (slot >= a.nz) return;
    const int nz = a.nz, ny = a.ny, nh = a.nh, mzp = a.mzp;
    const int kz = a.kz_of_slot[slot];
    const int kzs = kz <= nz - kz ? kz : nz - kz;
    const bool is00 = (kx == 0 && kz == 0);
    const double* A = a.bands + (is00 ? 3 : 0) * ny;
    const double* C = a.bands + (is00 ? 5 : 2) * ny;
    const size_t rstride = (size_t)nh * nz;  // X: next y plane
    const size_t pstride = (size_t)nh * mzp;  // D: next y plane
    double2* x = a.X + (size_t)kx * nz + slot;
    const double* d = a.piv + (size_t)kx * mzp + kzs;

    // forward sweep, y ascending
    double2 prev = make_double2(0.0, 0.0);
    for (int y0 = 0; y0 < ny; y0 += kBlock) {
        double2 v[kBlock];
        double D[kBlock], av[kBlock];
#pragma unroll
        for (int u = 0; u < kBlock; u++) {
            const int y = y0 + u;
            if (y < ny) {
                v[u] = x[(size_t)y * rstride];
                D[u] = d[(size_t)y * pstride];
                av[u] = A[y];
            }
        }
#pragma unroll
        for (int u = 0; u < kBlock; u++) {
            const int y = y0 + u;
            if (y < ny) {
                double2 r = v[u];
                if (y == 0) {
                    r.x = __ddiv_rn(r.x, D[u]);
                    r.y = __ddiv_rn(r.y, D[u]);
                } else {
                    r.x = __ddiv_rn(__dsub_rn(r.x, __dmul_rn(av[u], prev.x)), D[u]);
                    r.y = __ddiv_rn(__dsub_rn(r.y, __dmul_rn(av[u], prev.y)), D[u]);
                }
                prev = r;
                if (y < ny - 1) x[(size_t)y * rstride] = r;
            }
        }
    }
    // backward sweep, y descending; prev holds d'_{ny-1} = x_{ny-1}
    x[(size_t)(ny - 1) * rstride] = prev;
    for (int y1 = ny - 2; y1 >= 0; y1 -= kBlock) {
        double2 v[kBlock];
        double D[kBlock], cv[kBlock];
#pragma unroll
        for (int u = 0; u < kBlock; u++) {
            const int y = y1 - u;
            if (y >= 0) {
                v[u] = x[(size_t)y * rstride];
                D[u] = d[(size_t)y * pstride];
                cv[u] = C[y];
            }
        }
#pragma unroll
        for (int u = 0; u < kBlock; u++) {
            const int y = y1 - u;
            if (y >= 0) {
                const double c = __ddiv_rn(cv[u], D[u]);
                double2 r;
                r.x = __dsub_rn(v[u].x, __dmul_rn(prev.x, c));
                r.y = __dsub_rn(v[u].y, __dmul_rn(prev.y, c));
                prev = r;
                x[(size_t)y * rstride] = r;
            }
        }
    }
}

template <typename K>
cudaError_t allow_smem(K kernel, size_t bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace

// in-place z FFT of every spectral row: dir < 0 forward (natural -> slot order),
// dir > 0 inverse (slot order -> natural); needs pl->zd.ok
cudaError_t launch_zfft(const prj_plan* pl, int dir, cudaStream_t st) {
    const Geometry& g = pl->g;
    ZfftArgs a{};
    a.nrow_total = g.ny * g.nxh;
    a.nz = g.nz;
    a.f = pl->zd.f;
    a.tw = pl->zd.tw;
    a.X = pl->spec;
    const size_t row = (size_t)g.nz * sizeof(double2);
    int rb = 16;
    while (rb > 1 && (size_t)padded_len(rb * g.nz, true) * sizeof(double2) > 48 * 1024) rb /= 2;
    a.rb = rb;
    const size_t smem = (size_t)padded_len(rb * g.nz, true) * sizeof(double2);
    (void)row;
    const unsigned grid = (unsigned)((a.nrow_total + rb - 1) / rb);
    cudaError_t e;
    if (dir < 0) {
        if ((e = allow_smem(k_zfft<-1>, smem)) != cudaSuccess) return e;
        k_zfft<-1><<<grid, 256, smem, st>>>(a);
    } else {
        if ((e = allow_smem(k_zfft<+1>, smem)) != cudaSuccess) return e;
        k_zfft<+1><<<grid, 256, smem, st>>>(a);
    }
    return cudaGetLastError();
}


// Thomas sweeps over y for every (kx, slot) line, in place on the slot-ordered spectrum
cudaError_t launch_thomas(const prj_plan* pl, cudaStream_t st) {
    const Geometry& g = pl->g;
    ThomasArgs t{};
    t.nz = g.nz; t.ny = g.ny; t.nh = g.nxh; t.mzp = g.mzp;
    t.tiles = (g.nz + kThomasTile - 1) / kThomasTile;
    t.bands = pl->t.bands; t.piv = pl->t.piv; t.kz_of_slot = pl->kz_of_slot; t.X = pl->spec;
    k_thomas<<<(unsigned)(g.nxh * t.tiles), kThomasTile, 0, st>>>(t);
    return cudaGetLastError();
}

}  // namespace prj

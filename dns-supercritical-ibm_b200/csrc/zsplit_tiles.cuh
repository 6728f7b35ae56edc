// zsplit_tiles.cuh -- the split z direction as per-tile device functions.
//
// zfft_pass_tile: rb spectral z-rows of one buffer, in-place pass-plan FFT (forward:
// natural z order -> slot order; inverse: slot order -> natural).  thomas_line: the
// Thomas sweeps of one line (kx, slot) per thread, 128 lines per tile; thomas_line_async:
// the same sweeps with the planes streamed through a cp.async shared-memory ring.  The kernels of
// prj_zsplit.cu run one tile per CTA; the persistent batch kernel (prj_batchk.cu) runs
// tiles of many cases from a work queue with the same code, so both give the same bits.
#pragma once
#include "cp_async.cuh"
#include "div_rn.cuh"
#include "fft_pass.cuh"

struct prj_plan;

namespace prj {

struct ZfftArgs {
    int nrow_total;  // rows of length nz in this buffer (ny * rows per plane)
    int nz, rb;      // rows per CTA
    DifDev f;
    const double2* tw;
    void* X;         // double2 (FP64 storage) or float2 (FP32 storage) rows
};

__device__ __forceinline__ double2 to_d2(double2 v) { return v; }
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2(v.x, v.y); }
__device__ __forceinline__ void from_d2(double2& o, double2 v) { o = v; }
__device__ __forceinline__ void from_d2(float2& o, double2 v) { o = make_float2((float)v.x, (float)v.y); }


// Pass-plan z transform (fft_pass.cuh): the first pass reads the rows from global
// memory, the last writes them back; rb rows per CTA, kPassThreads threads.
// resident CTAs per SM asked of the pass-plan z kernels (measured at 768x384x384: 5 gives
// the forward z 0.300 ms against 0.345 ms at 6, the x kernels' setting)
#ifndef PRJ_ZPASS_MINB
#define PRJ_ZPASS_MINB 5
#endif

// staged input of a z tile (the persistent batch kernel, which copies the next tile's
// input by cp.async while the current one computes): its nr FP64 rows, contiguous in X,
// as S[r n + e]
template <class PL>
__device__ __forceinline__ void zfft_stage(const ZfftArgs& a, double2* S, int bx) {
    constexpr int n = PL::n;
    const size_t row0 = (size_t)bx * a.rb;
    const int nr = (int)min((size_t)a.rb, (size_t)a.nrow_total - row0);
    const double2* X = static_cast<const double2*>(a.X) + row0 * n;
    for (int i = threadIdx.x; i < nr * n; i += blockDim.x) cp_async(S + i, X + i, 16);
    cp_async_commit();
}

// STAGED: the rows come from S, where zfft_stage put them, and after_load() is called
// once S is no longer read
template <int DIR, typename T, class PL, bool STAGE_INV = false, bool STAGED = false, class Hook = NoHook>
__device__ __forceinline__ void zfft_pass_tile(const ZfftArgs& a, double2* zp, int bx, const double2* S = nullptr,
                                               Hook after_load = Hook{}) {
    static_assert(!STAGED || (STAGE_INV || DIR < 0), "a staged inverse copies its rows in whole");
    constexpr int n = PL::n;
    const size_t row0 = (size_t)bx * a.rb;
    const int nr = (int)min((size_t)a.rb, (size_t)a.nrow_total - row0);
    T* X = static_cast<T*>(a.X) + row0 * n;
    const double2* tw = a.tw;
    // the forward transform's slot-order rows leave shared memory in whole coalesced
    // rows (its last pass would store R contiguous elements per thread: half-sector
    // writes per instruction); the inverse copies them in whole rows the same way
    // (STAGE_INV) or reads them in its first pass
    const int tot = nr * n;
    if (DIR < 0) {
        if constexpr (STAGED) {
            dif_first_pass<-1, PL>(zp, nr, n, tw, [&](int r, int e) { return S[(size_t)r * n + e]; });
        } else {
            dif_first_pass<-1, PL>(zp, nr, n, tw, [&](int r, int e) { return to_d2(X[(size_t)r * n + e]); });
        }
        __syncthreads();
        after_load();
        dif_passes_shared<-1, PL, 1, PL::P>(zp, nr, n, tw);
        for (int i = threadIdx.x; i < tot; i += blockDim.x) from_d2(X[i], zp[sidx<true>(i)]);
    } else {
        if (STAGE_INV) {
            // slot-order rows copied in whole (coalesced), every pass in shared memory
            if constexpr (STAGED) {
                for (int i = threadIdx.x; i < tot; i += blockDim.x) zp[sidx<true>(i)] = S[i];
            } else {
#pragma unroll 4
                for (int i = threadIdx.x; i < tot; i += blockDim.x) zp[sidx<true>(i)] = to_d2(X[i]);
            }
            __syncthreads();
            after_load();
            dit_passes_shared<+1, PL, PL::P - 1, 0>(zp, nr, n, tw);
        } else {
            dit_first_pass<+1, PL>(zp, nr, n, [&](int r, int q) { return to_d2(X[(size_t)r * n + q]); });
            __syncthreads();
            dit_passes_shared<+1, PL, PL::P - 2, 0>(zp, nr, n, tw);
        }
        dit_last_pass<+1, PL>(zp, nr, n, tw, [&](int r, int e, double2 v) { from_d2(X[(size_t)r * n + e], v); });
    }
}

struct ThomasArgs {
    int nz, ny, nh, mzp, tiles;  // tiles of kThomasTile slots per kx
    int nhb, kx0;                // rows per plane in this buffer; its first kx
    const double* bands;         // a, b, c, a00, b00, c00
    const double* piv;           // D[y][kx][kzs], kx over all nh rows
    const double* pivc;          // c'[y][kx][kzs] = c_y / D_y, same layout
    const int* kz_of_slot;       // wavenumber held by each slot
    void* X;                     // T rows [y][kx - kx0][slot]
};

constexpr int kThomasTile = 128;
#ifndef PRJ_THOMAS_BLOCK
#define PRJ_THOMAS_BLOCK 8
#endif
constexpr int kBlock = PRJ_THOMAS_BLOCK;  // planes loaded together (independent loads in flight)

// One line: the CTA's block index `blk` within the buffer a.X (T storage).
// B planes of a line are loaded together (independent loads in flight); the result does
// not depend on B
template <typename T, int B = kBlock>
__device__ __forceinline__ void thomas_line(const ThomasArgs& a, int blk) {
    constexpr int kBlock = B;
    const int kb = blk / a.tiles;  // row within this buffer
    const int kx = a.kx0 + kb;
    const int slot = (blk - kb * a.tiles) * kThomasTile + threadIdx.x;
    if (slot >= a.nz) return;
    const int nz = a.nz, ny = a.ny, nh = a.nh, mzp = a.mzp;
    const int kz = a.kz_of_slot[slot];
    const int kzs = kz <= nz - kz ? kz : nz - kz;
    const bool is00 = (kx == 0 && kz == 0);
    const double* A = a.bands + (is00 ? 3 : 0) * ny;
    const size_t rstride = (size_t)a.nhb * nz;  // X: next y plane
    const size_t pstride = (size_t)nh * mzp;     // D: next y plane
    T* x = static_cast<T*>(a.X) + (size_t)kb * nz + slot;
    const double* d = a.piv + (size_t)kx * mzp + kzs;
    const double* dc = a.pivc + (size_t)kx * mzp + kzs;

    // forward sweep, y ascending
    double2 prev = make_double2(0.0, 0.0);
    for (int y0 = 0; y0 < ny; y0 += kBlock) {
        double2 v[kBlock];
        double D[kBlock], av[kBlock];
#pragma unroll
        for (int u = 0; u < kBlock; u++) {
            const int y = y0 + u;
            if (y < ny) {
                v[u] = to_d2(x[(size_t)y * rstride]);
                D[u] = d[(size_t)y * pstride];
                av[u] = A[y];
            }
        }
#pragma unroll
        for (int u = 0; u < kBlock; u++) {
            const int y = y0 + u;
            if (y < ny) {
                double2 r = v[u];
                const double rD = __drcp_rn(D[u]);  // off the recurrence's chain
                if (y == 0) {
                    r.x = div_by_recip(r.x, D[u], rD);
                    r.y = div_by_recip(r.y, D[u], rD);
                } else {
                    r.x = div_by_recip(__dsub_rn(r.x, __dmul_rn(av[u], prev.x)), D[u], rD);
                    r.y = div_by_recip(__dsub_rn(r.y, __dmul_rn(av[u], prev.y)), D[u], rD);
                }
                prev = r;
                if (y < ny - 1) from_d2(x[(size_t)y * rstride], r);
            }
        }
    }
    // backward sweep, y descending; prev holds d'_{ny-1} = x_{ny-1}
    from_d2(x[(size_t)(ny - 1) * rstride], prev);
    for (int y1 = ny - 2; y1 >= 0; y1 -= kBlock) {
        double2 v[kBlock];
        double cp[kBlock];
#pragma unroll
        for (int u = 0; u < kBlock; u++) {
            const int y = y1 - u;
            if (y >= 0) {
                v[u] = to_d2(x[(size_t)y * rstride]);
                cp[u] = dc[(size_t)y * pstride];  // c_y / D_y, tabulated with the pivots
            }
        }
#pragma unroll
        for (int u = 0; u < kBlock; u++) {
            const int y = y1 - u;
            if (y >= 0) {
                const double c = cp[u];
                double2 r;
                r.x = __dsub_rn(v[u].x, __dmul_rn(prev.x, c));
                r.y = __dsub_rn(v[u].y, __dmul_rn(prev.y, c));
                prev = r;
                from_d2(x[(size_t)y * rstride], r);
            }
        }
    }
}

// The same line solve with the planes streamed through a ring of NS shared-memory
// stages of B planes by cp.async (global -> shared, no register staging): while a
// thread computes block b it already has blocks b+1 .. b+NS-1 in flight, so the
// sequential recurrence no longer waits on one memory round trip per block.  Each
// thread copies exactly the elements it consumes (its own line), so a thread only
// waits for its own copy groups and no CTA barrier is needed.  Arithmetic and
// order are those of thomas_line, so the results are bit-identical.
template <typename T, int B, int NS>
__device__ __forceinline__ void thomas_line_async(const ThomasArgs& a, int blk, unsigned char* sm) {
    const int kb = blk / a.tiles;
    const int kx = a.kx0 + kb;
    const int slot = (blk - kb * a.tiles) * kThomasTile + threadIdx.x;
    if (slot >= a.nz) return;  // a thread leaves only its own copy groups behind: none issued
    const int nz = a.nz, ny = a.ny, nh = a.nh, mzp = a.mzp, tid = threadIdx.x;
    const int kz = a.kz_of_slot[slot];
    const int kzs = kz <= nz - kz ? kz : nz - kz;
    const bool is00 = (kx == 0 && kz == 0);
    const double* A = a.bands + (is00 ? 3 : 0) * ny;
    const size_t rstride = (size_t)a.nhb * nz;
    const size_t pstride = (size_t)nh * mzp;
    T* x = static_cast<T*>(a.X) + (size_t)kb * nz + slot;
    const double* d = a.piv + (size_t)kx * mzp + kzs;
    const double* dc = a.pivc + (size_t)kx * mzp + kzs;
    T* Xs = reinterpret_cast<T*>(sm);                                        // [NS][B][tile]
    double* Ds = reinterpret_cast<double*>(sm + (size_t)NS * B * kThomasTile * sizeof(T));  // [NS][B][tile]
    auto xs = [&](int st, int u) -> T& { return Xs[((size_t)st * B + u) * kThomasTile + tid]; };
    auto ds = [&](int st, int u) -> double& { return Ds[((size_t)st * B + u) * kThomasTile + tid]; };
    const int nb = (ny + B - 1) / B;

    // forward sweep, y ascending: block b = planes b B .. b B + B - 1
    auto issue_f = [&](int b) {
        if (b < nb) {
            const int st = b % NS;
            for (int u = 0; u < B; u++) {
                const int y = b * B + u;
                if (y < ny) {
                    cp_async(&xs(st, u), x + (size_t)y * rstride, (int)sizeof(T));
                    cp_async(&ds(st, u), d + (size_t)y * pstride, 8);
                }
            }
        }
        cp_async_commit();
    };
#pragma unroll
    for (int b = 0; b < NS - 1; b++) issue_f(b);
    double2 prev = make_double2(0.0, 0.0);
    for (int b = 0; b < nb; b++) {
        issue_f(b + NS - 1);
        cp_async_wait<NS - 1>();
        const int st = b % NS;
#pragma unroll
        for (int u = 0; u < B; u++) {
            const int y = b * B + u;
            if (y < ny) {
                double2 r = to_d2(xs(st, u));
                const double D = ds(st, u);
                const double rD = __drcp_rn(D);  // off the recurrence's chain
                if (y == 0) {
                    r.x = div_by_recip(r.x, D, rD);
                    r.y = div_by_recip(r.y, D, rD);
                } else {
                    const double av = A[y];
                    r.x = div_by_recip(__dsub_rn(r.x, __dmul_rn(av, prev.x)), D, rD);
                    r.y = div_by_recip(__dsub_rn(r.y, __dmul_rn(av, prev.y)), D, rD);
                }
                prev = r;
                if (y < ny - 1) from_d2(x[(size_t)y * rstride], r);
            }
        }
    }
    cp_async_wait<0>();
    // the backward sweep reads what this thread just stored: complete those stores first
    __threadfence();
    from_d2(x[(size_t)(ny - 1) * rstride], prev);
    // backward sweep, y descending from ny-2: block b = planes ny-2 - b B - u
    const int nbb = (ny - 1 + B - 1) / B;
    auto issue_b = [&](int b) {
        if (b < nbb) {
            const int st = b % NS;
            for (int u = 0; u < B; u++) {
                const int y = ny - 2 - b * B - u;
                if (y >= 0) {
                    cp_async(&xs(st, u), x + (size_t)y * rstride, (int)sizeof(T));
                    cp_async(&ds(st, u), dc + (size_t)y * pstride, 8);
                }
            }
        }
        cp_async_commit();
    };
#pragma unroll
    for (int b = 0; b < NS - 1; b++) issue_b(b);
    for (int b = 0; b < nbb; b++) {
        issue_b(b + NS - 1);
        cp_async_wait<NS - 1>();
        const int st = b % NS;
#pragma unroll
        for (int u = 0; u < B; u++) {
            const int y = ny - 2 - b * B - u;
            if (y >= 0) {
                const double c = ds(st, u);  // c_y / D_y, tabulated with the pivots
                const double2 v = to_d2(xs(st, u));
                double2 r;
                r.x = __dsub_rn(v.x, __dmul_rn(prev.x, c));
                r.y = __dsub_rn(v.y, __dmul_rn(prev.y, c));
                prev = r;
                from_d2(x[(size_t)y * rstride], r);
            }
        }
    }
    cp_async_wait<0>();
}

// ring shape (planes per stage B x stages NS) of the streamed kernel
template <typename T, int B, int NS>
constexpr size_t thomas_async_smem() {
    return (size_t)NS * B * kThomasTile * (sizeof(T) + sizeof(double));
}

// arguments of a plan's FP64 spectrum rows for zfft_pass_tile, and of its Thomas lines
// kx0 .. kx0+rows-1 held in X as [y][kx - kx0][z] (prj_zsplit.cu)
ZfftArgs batch_z_args(const prj_plan* pl);
int batch_z_default_rows(int nz);  // rows per tile of the z kernels' default shape
ThomasArgs thomas_args(const prj_plan* pl, void* X, int kx0, int rows_per_plane);

}  // namespace prj

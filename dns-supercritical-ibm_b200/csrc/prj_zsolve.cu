// prj_zsolve.cu -- z transform + Thomas + inverse z transform, pipelined.
//
// One CTA owns one x-wavenumber kx and walks the wall-normal direction in
// chunks of `yb` planes.  A ring of `ns` shared-memory stages is filled by
// bulk (TMA) copies -- the spectral z-rows X[y][kx][:] and the pivot rows
// D[y][kx][:] of a chunk -- while the CTA works on the previous chunk:
//
//   forward pass  (y = 0 .. ny-1): FFT along z of the chunk's rows (all rows in
//                 parallel), then the Thomas forward recurrence across the
//                 rows, d'_y = (d_y - a_y d'_{y-1}) / D_y, written back in place;
//   backward pass (y = ny-1 .. 0): back substitution x_y = d'_y - c'_y x_{y+1}
//                 with c'_y = c_y / D_y, then the inverse FFT of the chunk's
//                 rows, written back in place.
//
// The recurrence keeps the reference's operation order and rounding
// (poisson_solver_multigpu.f90:401-419) through round-to-nearest intrinsics.
// Every mbarrier wait is bounded; on a timeout the CTA raises *err, waits
// (bounded) for its copies in flight and returns.
#include <cstdlib>

#include "prj_internal.h"
#include "tma_util.cuh"

namespace prj {

namespace {

struct ZPipeArgs {
    int nz, ny, nh, nzh, mzp;
    int yb, ns;
    FftDev f;
    const double2* tw;
    const double* bands;  // a, b, c, a00, b00, c00
    const double* piv;    // D[y][kx][kzs]
    double2* X;
    int* err;
    DifDev fd;            // in-place transform (DIF variant)
    const double2* dtw;
    const int* dpos;
};

// DIF = true: in-place transforms (no work buffer), spectrum read through the
// position table; DIF = false: out-of-place Stockham transforms with a work buffer.
template <int PPT, bool DIF>
__global__ void __launch_bounds__(512) k_zsolve_pipe(const ZPipeArgs a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int nz = a.nz, ny = a.ny, yb = a.yb, ns = a.ns, mzp = a.mzp, nh = a.nh;
    const uint32_t xrow = (uint32_t)nz * sizeof(double2);
    const uint32_t prow = (uint32_t)mzp * sizeof(double);
    const size_t stage_bytes = (size_t)yb * (xrow + prow);
    // after the stages: DIF -> position table (nz ints, padded to 16 B); Stockham -> work rows
    const size_t extra = DIF ? ((size_t)nz * sizeof(int) + 15) / 16 * 16 : (size_t)yb * xrow;
    double2* work = reinterpret_cast<double2*>(smraw + ns * stage_bytes);
    int* pos = reinterpret_cast<int*>(smraw + ns * stage_bytes);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smraw + ns * stage_bytes + extra);

    const int tid = threadIdx.x, nthr = blockDim.x;
    const int kx = blockIdx.x;
    const int nch = (ny + yb - 1) / yb;
    const double* ba = a.bands;
    const double* bc = a.bands + 2 * ny;
    const double* ba0 = a.bands + 3 * ny;
    const double* bc0 = a.bands + 5 * ny;

    if (DIF)
        for (int i = tid; i < nz; i += nthr) pos[i] = a.dpos[i];
    if (tid == 0) {
        for (int s = 0; s < ns; s++) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncthreads();

    uint32_t phase = 0;    // bit s: parity of the next completion of stage s
    uint32_t pending = 0;  // bit s: stage s has a load in flight (same value in every thread)

    auto stage_x = [&](int s) { return reinterpret_cast<double2*>(smraw + s * stage_bytes); };
    auto stage_d = [&](int s) { return reinterpret_cast<double*>(smraw + s * stage_bytes + (size_t)yb * xrow); };
    // load chunk c (planes [c yb, c yb + nr)) into stage s; thread 0 only
    auto issue = [&](int c, int s) {
        const int y0 = c * yb;
        const int nr = min(yb, ny - y0);
        fence_proxy_async_shared();
        mbar_arrive_expect_tx(&bars[s], (uint32_t)nr * (xrow + prow));
        for (int r = 0; r < nr; r++) {
            const size_t line = (size_t)(y0 + r) * nh + kx;
            bulk_g2s(stage_x(s) + (size_t)r * nz, a.X + line * nz, xrow, &bars[s]);
            bulk_g2s(stage_d(s) + (size_t)r * mzp, a.piv + line * mzp, prow, &bars[s]);
        }
    };
    // consume stage s; false (in every thread) if any thread gave up waiting
    auto acquire = [&](int s) -> bool {
        const bool ok = mbar_wait_bounded(&bars[s], (phase >> s) & 1u);
        phase ^= 1u << s;
        pending &= ~(1u << s);
        return !__syncthreads_or(!ok);
    };
    auto bail = [&]() {
        if (tid == 0) {
            atomicExch(a.err, 1);
            for (int s = 0; s < ns; s++)
                if (pending & (1u << s)) mbar_wait_bounded(&bars[s], (phase >> s) & 1u);
        }
    };

    double2 p0[PPT], p1[PPT];
#pragma unroll
    for (int q = 0; q < PPT; q++) { p0[q] = make_double2(0, 0); p1[q] = make_double2(0, 0); }

    // ------------------------------------------------------------ forward pass
    for (int c = 0; c < ns - 1 && c < nch; c++) {
        if (tid == 0) issue(c, c % ns);
        pending |= 1u << (c % ns);
    }
    for (int c = 0; c < nch; c++) {
        const int s = c % ns;
        if (c + ns - 1 < nch) {
            if (tid == 0) issue(c + ns - 1, (c + ns - 1) % ns);
            pending |= 1u << ((c + ns - 1) % ns);
        }
        if (!acquire(s)) { bail(); return; }
        const int y0 = c * yb;
        const int nr = min(yb, ny - y0);
        const double2* F;
        if (DIF) {
            dif_rows<-1>(stage_x(s), nr, nz, a.fd, a.dtw);
            F = stage_x(s);
        } else {
            F = fft_rows<-1>(stage_x(s), work, nr, nz, a.f, a.tw);
        }
        const double* Ds = stage_d(s);
        for (int r = 0; r < nr; r++) {
            const int y = y0 + r;
            double2* grow = a.X + ((size_t)y * nh + kx) * nz;
            const double av = ba[y], av00 = ba0[y];
#pragma unroll
            for (int q = 0; q < PPT; q++) {
                const int t = tid + q * nthr;
                if (t < a.nzh) {
                    const bool two = (t > 0) && (2 * t != nz);
                    const double D = Ds[(size_t)r * mzp + t];
                    double2 v0 = F[(size_t)r * nz + (DIF ? pos[t] : t)];
                    double2 v1 = two ? F[(size_t)r * nz + (DIF ? pos[nz - t] : nz - t)] : make_double2(0, 0);
                    if (y == 0) {
                        v0.x = __ddiv_rn(v0.x, D); v0.y = __ddiv_rn(v0.y, D);
                        v1.x = __ddiv_rn(v1.x, D); v1.y = __ddiv_rn(v1.y, D);
                    } else {
                        const double aa = (kx == 0 && t == 0) ? av00 : av;
                        v0.x = __ddiv_rn(__dsub_rn(v0.x, __dmul_rn(aa, p0[q].x)), D);
                        v0.y = __ddiv_rn(__dsub_rn(v0.y, __dmul_rn(aa, p0[q].y)), D);
                        v1.x = __ddiv_rn(__dsub_rn(v1.x, __dmul_rn(aa, p1[q].x)), D);
                        v1.y = __ddiv_rn(__dsub_rn(v1.y, __dmul_rn(aa, p1[q].y)), D);
                    }
                    p0[q] = v0; p1[q] = v1;
                    grow[t] = v0;
                    if (two) grow[nz - t] = v1;
                }
            }
        }
        __syncthreads();
    }
    // the backward pass reads the forward-sweep values back through bulk copies
    fence_proxy_async_global();
    __syncthreads();

    // ----------------------------------------------------------- backward pass
    // chunk counter continues from the forward pass: global chunk g uses stage g % ns
    for (int j = 0; j < ns - 1 && j < nch; j++) {
        const int s = (nch + j) % ns;
        if (tid == 0) issue(nch - 1 - j, s);
        pending |= 1u << s;
    }
    for (int j = 0; j < nch; j++) {
        const int s = (nch + j) % ns;
        if (j + ns - 1 < nch) {
            const int s2 = (nch + j + ns - 1) % ns;
            if (tid == 0) issue(nch - 1 - (j + ns - 1), s2);
            pending |= 1u << s2;
        }
        if (!acquire(s)) { bail(); return; }
        const int c = nch - 1 - j;
        const int y0 = c * yb;
        const int nr = min(yb, ny - y0);
        double2* Xs = stage_x(s);
        const double* Ds = stage_d(s);
        for (int r = nr - 1; r >= 0; r--) {
            const int y = y0 + r;
            const double cv = bc[y], cv00 = bc0[y];
#pragma unroll
            for (int q = 0; q < PPT; q++) {
                const int t = tid + q * nthr;
                if (t < a.nzh) {
                    const bool two = (t > 0) && (2 * t != nz);
                    const double2 d0 = Xs[(size_t)r * nz + t];
                    const double2 d1 = two ? Xs[(size_t)r * nz + nz - t] : make_double2(0, 0);
                    if (y == ny - 1) {
                        p0[q] = d0; p1[q] = d1;
                    } else {
                        const double C = __ddiv_rn((kx == 0 && t == 0) ? cv00 : cv, Ds[(size_t)r * mzp + t]);
                        p0[q].x = __dsub_rn(d0.x, __dmul_rn(p0[q].x, C));
                        p0[q].y = __dsub_rn(d0.y, __dmul_rn(p0[q].y, C));
                        p1[q].x = __dsub_rn(d1.x, __dmul_rn(p1[q].x, C));
                        p1[q].y = __dsub_rn(d1.y, __dmul_rn(p1[q].y, C));
                    }
                    Xs[(size_t)r * nz + t] = p0[q];
                    if (two) Xs[(size_t)r * nz + nz - t] = p1[q];
                }
            }
        }
        __syncthreads();
        if (DIF) {
            dif_rows<+1>(Xs, nr, nz, a.fd, a.dtw);
            for (int i = tid; i < nr * nz; i += nthr) {
                const int r = i / nz, z = i - r * nz;
                a.X[((size_t)(y0 + r) * nh + kx) * nz + z] = Xs[(size_t)r * nz + pos[z]];
            }
        } else {
            const double2* G = fft_rows<+1>(Xs, work, nr, nz, a.f, a.tw);
            for (int i = tid; i < nr * nz; i += nthr) {
                const int r = i / nz, z = i - r * nz;
                a.X[((size_t)(y0 + r) * nh + kx) * nz + z] = G[i];
            }
        }
        __syncthreads();
    }
}

template <int PPT, bool DIF>
cudaError_t launch_pipe(const ZPipeArgs& a, int nthr, size_t smem, cudaStream_t st) {
    cudaError_t e =
        cudaFuncSetAttribute(k_zsolve_pipe<PPT, DIF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_zsolve_pipe<PPT, DIF><<<a.nh, nthr, smem, st>>>(a);
    return cudaGetLastError();
}

template <bool DIF>
cudaError_t launch_ppt(const ZPipeArgs& a, int ppt, int nthr, size_t smem, cudaStream_t st) {
    switch (ppt) {
    case 1: return launch_pipe<1, DIF>(a, nthr, smem, st);
    case 2: return launch_pipe<2, DIF>(a, nthr, smem, st);
    default: return launch_pipe<4, DIF>(a, nthr, smem, st);
    }
}

}  // namespace

// Chooses the chunk size and ring depth for about 72 KB of shared memory (three
// CTAs per SM; the plan's z_planes / z_stages tuning overrides them) and
// returns cudaErrorNotSupported when even one plane per chunk with two stages
// does not fit, so the caller can use the unpipelined kernel.
cudaError_t launch_zsolve_pipelined(const prj_plan* pl, int* err_word, cudaStream_t st) {
    const Geometry& g = pl->g;
    ZPipeArgs a{};
    a.nz = g.nz; a.ny = g.ny; a.nh = g.nxh; a.nzh = g.nzh; a.mzp = g.mzp;
    a.f = pl->fz64.f; a.tw = pl->fz64.tw; a.bands = pl->t.bands; a.piv = pl->t.piv; a.X = pl->spec;
    a.err = err_word;
    const bool dif = pl->zd.ok;
    if (dif) { a.fd = pl->zd.f; a.dtw = pl->zd.tw; a.dpos = pl->zd.pos; }
    const size_t xrow = (size_t)g.nz * sizeof(double2), prow = (size_t)g.mzp * sizeof(double);
    auto bytes = [&](int yb, int ns) {
        const size_t extra = dif ? ((size_t)g.nz * sizeof(int) + 15) / 16 * 16 : (size_t)yb * xrow;
        return (size_t)ns * yb * (xrow + prow) + extra + 8 * (size_t)ns;
    };
    int yb = pl->z_planes, ns = pl->z_stages;
    if (yb < 1 || ns < 2 || ns > 8 || bytes(yb, ns) > 200 * 1024) {
        yb = 0;
        const int pref_ns = dif ? 2 : 3;
        for (int cand = 8; cand >= 1; cand /= 2)
            if (bytes(cand, pref_ns) <= 72 * 1024) { yb = cand; ns = pref_ns; break; }
        if (!yb)
            for (int cand = 2; cand >= 1; cand /= 2)
                if (bytes(cand, 2) <= 200 * 1024) { yb = cand; ns = 2; break; }
    }
    if (!yb) return cudaErrorNotSupported;
    a.yb = yb; a.ns = ns;
    int ppt = 1;
    while ((g.nzh + ppt - 1) / ppt > 512) ppt *= 2;
    if (ppt > 4) return cudaErrorNotSupported;
    int nthr = (g.nzh + ppt - 1) / ppt;
    nthr = (nthr + 31) / 32 * 32;
    if (nthr < 128) nthr = 128;
    const size_t smem = bytes(yb, ns);
    return dif ? launch_ppt<true>(a, ppt, nthr, smem, st) : launch_ppt<false>(a, ppt, nthr, smem, st);
}

}  // namespace prj

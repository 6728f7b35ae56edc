// zline_tiles.cuh -- the z direction of the solve for one x wavenumber, as a device
// function: z FFT, Thomas sweeps and inverse z FFT of the ny spectral z-rows X[y][kx][:].
//
//   forward phase, y ascending, chunks of yb planes:
//     rows (natural z order) copied into a shared-memory stage by one tensor-map copy
//     (TMA) and pivot rows by cp.async, NS stages in flight;
//     forward z FFT of the chunk's rows in place, every pass in shared memory;
//     d'_y = (d_y - a_y d'_{y-1}) / D_y for the chunk's planes, stored to the row
//     (slot order);
//   backward phase, y descending:
//     d' rows and the rows of c'_y = c_y / D_y (tabulated with the pivots) streamed
//     back the same way;
//     x_y = d'_y - c'_y x_{y+1} in the stage;
//     inverse z FFT in place, the last pass storing natural-order rows.
//
// The spectrum crosses HBM four times (rows in, d' out, d' in, rows out) against
// eight for the split kernels (z FFT in/out, Thomas in/out twice, inverse z
// in/out).  The butterflies, twiddle tables and the Thomas operation order
// (poisson_solver_multigpu.f90:401-419, round-to-nearest intrinsics) are those of
// k_zfft_pass and k_thomas, so the result is bitwise that of the split kernels.
// Every mbarrier wait is bounded (a clock budget).  k_zline
// (prj_zline.cu) runs one wavenumber per CTA; the persistent batch kernel
// (prj_batchk.cu) runs (case, wavenumber) tiles from its work queue.
#pragma once
#include <cuda.h>

#include "cp_async.cuh"
#include "div_rn.cuh"
#include "fft_pass.cuh"
#include "tma_util.cuh"

struct prj_plan;

namespace prj {

struct ZLineArgs {
    int ny, nh, mzp;
    int yb;               // planes per stage
    const double2* tw;    // z pass-plan twiddles
    const double* bands;  // a, b, c, a00, b00, c00
    const double* piv;    // D[y][kx][kzs]
    const double* pivc;   // c'[y][kx][kzs] = c_y / D_y
    const int* kz_of_slot;
    double2* X;           // [y][kx][z]
    int* err;             // raised (5) when a bounded mbarrier wait gives up
};

// lines per thread (default) and threads per CTA of a length-n plan; resident CTAs per
// SM asked of the register allocator
__host__ __device__ constexpr int zl_lpt(int n) { return n <= 128 ? 1 : n <= 512 ? 2 : n <= 1024 ? 4 : 8; }
__host__ __device__ constexpr int zl_threads(int n, int lpt) { return n / lpt < 32 ? 32 : n / lpt; }
__host__ __device__ constexpr int zl_minb(int nt) { return nt <= 64 ? 8 : nt <= 128 ? 5 : nt <= 384 ? 3 : 2; }

// Pivot rows in shared memory: rows of mzs = mzp rounded up to 16 doubles; the 16-byte
// piece j (kzs 2j, 2j+1) sits at piece zl_piece(j), which permutes the pieces of each
// 128-byte group by the group index.  The Thomas phase gathers pivots by wavenumber in
// the slots' digit-reversed order: the permutation spreads the 8 pieces that a stride of
// 8 groups apart would put on one bank pair (n = 384: 129 -> 68 wavefronts per plane for
// the CTA's pivot reads, against 24 conflict-free).
__host__ __device__ constexpr int zl_mzs(int mzp) { return (mzp + 15) & ~15; }
__host__ __device__ constexpr int zl_piece(int j) { return (j & ~7) | ((j ^ (j >> 3)) & 7); }

// For a z length n (mzp = nz/2 + 1 rounded up to even, as the plan sets it): the copied
// pieces land on distinct pieces inside the padded row, and every folded wavenumber a
// thread reads lies in a copied piece.  Checked at compile time for every pass-plan length.
constexpr bool zl_layout_ok(int n) {
    const int mzp = (n / 2 + 2) / 2 * 2, mzs = zl_mzs(mzp), hp = mzp / 2;
    bool used[1024] = {};
    if (mzs / 2 > 1024) return false;
    for (int j = 0; j < hp; j++) {
        const int p = zl_piece(j);
        if (p < 0 || p >= mzs / 2 || used[p]) return false;
        used[p] = true;
    }
    for (int kf = 0; kf <= n / 2; kf++)
        if ((kf >> 1) >= hp || 2 * zl_piece(kf >> 1) + (kf & 1) >= mzs) return false;
    return true;
}
#define PRJ_ZL_LAYOUT_CHECK(N, ...) static_assert(zl_layout_ok(N), "pivot stage layout of length " #N);
PRJ_PASS_PLANS(PRJ_ZL_LAYOUT_CHECK)
#undef PRJ_ZL_LAYOUT_CHECK

// Shared memory of a tile: 128 bytes of alignment slack, NS mbarriers (128 bytes),
// NS row stages of zl_slot_bytes each (128-byte aligned), then the pivot ring.  A stage
// holds yb rows in the padded layout of the FFT passes: each group of 8 complex values is
// followed by one pad slot, which is what a tensor-map box of 9 complex values per group
// (the 9th out of bounds, zero-filled) writes.
__host__ __device__ inline size_t zl_slot_bytes(int n, int yb) { return ((size_t)yb * n * 18 + 127) / 128 * 128; }

// The z solve of x wavenumber kx: NT threads (the CTA), LPT lines per thread (NT LPT >=
// n; slots past n idle in the Thomas phase), NS stages of a.yb planes in `zsm`
// (zline_smem bytes).  Each stage's rows arrive by one tensor-map copy (`tmap`:
// zline_tmap's 4-D view of the spectrum) issued by thread 0 and completed on an mbarrier;
// the pivot rows are cp.async copies (their pieces are permuted).  Every mbarrier wait is
// bounded: on a timeout the tile raises *a.err, waits (bounded) for its copies in flight
// and returns.
template <class PL, int NS, int LPT, int NT>
__device__ __forceinline__ void zline_tile(const ZLineArgs& a, const void* tmap, int kx, unsigned char* zsm) {
    constexpr int n = PL::n;
    static_assert(NT * LPT >= n, "every line has a thread");
    static_assert(n % 8 == 0, "the stage layout needs whole groups of 8");
    const int ny = a.ny, nh = a.nh, mzp = a.mzp, mzs = zl_mzs(mzp), yb = a.yb, tid = threadIdx.x;
    const int nch = (ny + yb - 1) / yb;
    unsigned char* base = zsm + ((128u - (smem_u32(zsm) & 127u)) & 127u);
    uint64_t* bars = reinterpret_cast<uint64_t*>(base);
    const size_t slot_bytes = zl_slot_bytes(n, yb);
    unsigned char* rslots = base + 128;
    double* dring = reinterpret_cast<double*>(rslots + NS * slot_bytes);
    auto stage = [&](int s) { return reinterpret_cast<double2*>(rslots + s * slot_bytes); };
    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < NS; s++) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncthreads();
    uint32_t phase = 0;    // bit s: parity of stage s's next completion
    uint32_t pending = 0;  // bit s: stage s has a copy in flight (the same in every thread)

    // this thread's lines
    int slot[LPT], kzs[LPT];
    bool is00[LPT];
#pragma unroll
    for (int q = 0; q < LPT; q++) {
        slot[q] = tid + q * NT;
        const int kz = slot[q] < n ? a.kz_of_slot[slot[q]] : 0;
        const int kf = kz <= n - kz ? kz : n - kz;
        kzs[q] = 2 * zl_piece(kf >> 1) + (kf & 1);  // position in a shared pivot row
        is00[q] = (kx == 0 && kz == 0);
    }
    const double* bA = a.bands;
    const double* bA0 = a.bands + 3 * ny;

    // chunk c (planes c yb ..) into stage s with the rows of table tab (pivots on the way
    // up, back-substitution factors on the way down): the rows by one tensor-map copy (a
    // box of yb planes, those past ny zero-filled), the pivots by every thread's cp.async
    // share; one cp.async group per call
    auto issue = [&](int c, int s, const double* tab) {
        if (c >= 0 && c < nch) {
            const int y0 = c * yb, nr = min(yb, ny - y0);
            if (tid == 0) {
                fence_proxy_async_shared();  // the stage's earlier reads before the copy's writes
                mbar_arrive_expect_tx(&bars[s], (uint32_t)(18 * n * yb));
                tma_load_4d(stage(s), tmap, 0, 0, kx, y0, &bars[s]);
            }
            pending |= 1u << s;
            const int hp = mzp / 2;  // 16-byte pieces of a pivot row
            double* dbuf = dring + (size_t)s * yb * mzs;
            for (int i = tid; i < nr * hp; i += NT) {
                const int r = i / hp, j = i - r * hp;
                cp_async(dbuf + (size_t)r * mzs + 2 * zl_piece(j), tab + ((size_t)(y0 + r) * nh + kx) * mzp + 2 * j, 16);
            }
        }
        cp_async_commit();
    };
    // stage s's copies complete (pivots: this thread's groups but the NS-1 newest); false
    // in every thread if any thread's wait gave up
    auto acquire = [&](int s) -> bool {
        cp_async_wait<NS - 1>();
        const bool ok = mbar_wait_bounded(&bars[s], (phase >> s) & 1u);
        phase ^= 1u << s;
        pending &= ~(1u << s);
        return !__syncthreads_or(!ok);
    };
    auto bail = [&]() {
        if (tid == 0) {
            atomicExch(a.err, 5);
#pragma unroll
            for (int s = 0; s < NS; s++)
                if (pending & (1u << s)) mbar_wait_bounded(&bars[s], (phase >> s) & 1u);
        }
        cp_async_wait<0>();
        __syncthreads();
        if (tid == 0)
#pragma unroll
            for (int s = 0; s < NS; s++) mbar_inval(&bars[s]);
    };

    double2 prev[LPT];
#pragma unroll
    for (int q = 0; q < LPT; q++) prev[q] = make_double2(0.0, 0.0);

    // ------------------------------------------------------------ forward phase
#pragma unroll
    for (int c = 0; c < NS - 1; c++) issue(c, c, a.piv);
    for (int c = 0; c < nch; c++) {
        issue(c + NS - 1, (c + NS - 1) % NS, a.piv);  // that stage was last read in iteration c - 1
        const int s = c % NS, y0 = c * yb, nr = min(yb, ny - y0);
        if (!acquire(s)) {
            bail();
            return;
        }
        double2* buf = stage(s);
        const double* dbuf = dring + (size_t)s * yb * mzs;
        dif_passes_shared<-1, PL, 0, PL::P>(buf, nr, n, a.tw);  // barrier after every pass
        for (int r = 0; r < nr; r++) {
            const int y = y0 + r;
            double2* grow = a.X + ((size_t)y * nh + kx) * n;
#pragma unroll
            for (int q = 0; q < LPT; q++) {
                if (slot[q] < n) {
                    double2 v = buf[sidx<true>(r * n + slot[q])];
                    const double D = dbuf[(size_t)r * mzs + kzs[q]];
                    const double rD = __drcp_rn(D);  // off the recurrence's chain
                    if (y == 0) {
                        v.x = div_by_recip(v.x, D, rD);
                        v.y = div_by_recip(v.y, D, rD);
                    } else {
                        const double av = is00[q] ? bA0[y] : bA[y];
                        v.x = div_by_recip(__dsub_rn(v.x, __dmul_rn(av, prev[q].x)), D, rD);
                        v.y = div_by_recip(__dsub_rn(v.y, __dmul_rn(av, prev[q].y)), D, rD);
                    }
                    prev[q] = v;
                    grow[slot[q]] = v;
                }
            }
        }
        __syncthreads();
    }
    cp_async_wait<0>();
    // the backward phase's tensor-map copies read back rows other threads of this CTA
    // stored
    __threadfence();
    fence_proxy_async_global();
    __syncthreads();

    // ----------------------------------------------------------- backward phase
    // j-th chunk from the top (chunk nch-1-j) uses stage (nch + j) % NS, continuing the
    // forward phase's rotation
#pragma unroll
    for (int j = 0; j < NS - 1; j++) issue(nch - 1 - j, (nch + j) % NS, a.pivc);
    for (int j = 0; j < nch; j++) {
        issue(nch - 1 - (j + NS - 1), (nch + j + NS - 1) % NS, a.pivc);
        const int s = (nch + j) % NS, c = nch - 1 - j, y0 = c * yb, nr = min(yb, ny - y0);
        if (!acquire(s)) {
            bail();
            return;
        }
        double2* buf = stage(s);
        const double* dbuf = dring + (size_t)s * yb * mzs;
        for (int r = nr - 1; r >= 0; r--) {
            const int y = y0 + r;
#pragma unroll
            for (int q = 0; q < LPT; q++) {
                if (slot[q] < n) {
                    double2& cell = buf[sidx<true>(r * n + slot[q])];
                    const double2 d = cell;
                    if (y == ny - 1) {
                        prev[q] = d;
                    } else {
                        const double C = dbuf[(size_t)r * mzs + kzs[q]];  // c_y / D_y
                        prev[q].x = __dsub_rn(d.x, __dmul_rn(prev[q].x, C));
                        prev[q].y = __dsub_rn(d.y, __dmul_rn(prev[q].y, C));
                    }
                    cell = prev[q];
                }
            }
        }
        __syncthreads();
        dit_passes_shared<+1, PL, PL::P - 1, 0>(buf, nr, n, a.tw);
        dit_last_pass<+1, PL>(buf, nr, n, a.tw, [&](int r, int e, double2 v) {
            a.X[((size_t)(y0 + r) * nh + kx) * n + e] = v;
        });
        __syncthreads();
    }
    cp_async_wait<0>();
    __syncthreads();
    if (tid == 0)
#pragma unroll
        for (int s = 0; s < NS; s++) mbar_inval(&bars[s]);
}

// arguments of a plan's z solves (FP64 spectrum, pivots, z pass plan; yb from the plan's
// z_planes tuning or 4; prj_zline.cu)
ZLineArgs zline_args(const prj_plan* pl);

// shared memory of a tile (alignment slack, mbarriers, row stages, pivot ring)
inline size_t zline_smem(int n, int mzp, int yb, int ns) {
    return 256 + (size_t)ns * zl_slot_bytes(n, yb) + (size_t)ns * yb * zl_mzs(mzp) * sizeof(double);
}

// the 4-D tensor map of the row copies over the spectrum X (n-point z rows,
// nh x wavenumbers, ny planes): dims {16 doubles (a group of 8 complex values), n/8
// groups, nh, ny}, box {18, n/8, 1, yb}; false if the driver refuses it
bool zline_tmap(void* tmap128, const double2* X, int n, int nh, int ny, int yb);


}  // namespace prj

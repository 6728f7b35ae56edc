// prj_zline.cu -- the z direction of the solve as one kernel per x wavenumber,
// built on the pass-plan butterflies (fft_pass.cuh).
//
// One CTA owns one x wavenumber kx: the ny spectral z-rows X[y][kx][:] and the nz
// Thomas lines (kx, slot) that run through them.  Each thread owns LPT lines
// (slots tid + q NT) and carries their recurrence in registers.
//
//   forward phase, y ascending, chunks of yb planes:
//     rows (natural z order) and pivot rows copied into a shared-memory stage by
//     cp.async, NS stages in flight;
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
// cp.async copies complete on their own, so no wait here can hang.
#include "div_rn.cuh"
#include "fft_pass.cuh"
#include "prj_internal.h"

namespace prj {

namespace {

struct ZLineArgs {
    int ny, nh, mzp;
    int yb;               // planes per stage
    const double2* tw;    // z pass-plan twiddles
    const double* bands;  // a, b, c, a00, b00, c00
    const double* piv;    // D[y][kx][kzs]
    const double* pivc;   // c'[y][kx][kzs] = c_y / D_y
    const int* kz_of_slot;
    double2* X;           // [y][kx][z]
};

__device__ __forceinline__ void zl_cp16(void* dst, const void* src) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void zl_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void zl_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

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

template <class PL, int NS, int LPT>
__global__ void __launch_bounds__(zl_threads(PL::n, LPT), zl_minb(zl_threads(PL::n, LPT))) k_zline(const ZLineArgs a) {
    constexpr int n = PL::n, NT = zl_threads(n, LPT);
    extern __shared__ __align__(16) unsigned char zsm[];
    const int ny = a.ny, nh = a.nh, mzp = a.mzp, mzs = zl_mzs(mzp), yb = a.yb, tid = threadIdx.x;
    const int kx = blockIdx.x;
    double2* ring = reinterpret_cast<double2*>(zsm);  // NS * yb rows of n, padded as one array
    double* dring = reinterpret_cast<double*>(zsm + (size_t)padded_len(NS * yb * n, true) * sizeof(double2));
    const int nch = (ny + yb - 1) / yb;

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
    // up, back-substitution factors on the way down); every thread copies a share; one
    // group per call
    auto issue = [&](int c, int s, const double* tab) {
        if (c >= 0 && c < nch) {
            const int y0 = c * yb, nr = min(yb, ny - y0);
            double2* buf = ring + sidx<true>(s * yb * n);
            for (int i = tid; i < nr * n; i += NT) {
                const int r = i / n, e = i - r * n;
                zl_cp16(&buf[sidx<true>(r * n + e)], a.X + ((size_t)(y0 + r) * nh + kx) * n + e);
            }
            const int hp = mzp / 2;  // 16-byte pieces of a pivot row
            double* dbuf = dring + (size_t)s * yb * mzs;
            for (int i = tid; i < nr * hp; i += NT) {
                const int r = i / hp, j = i - r * hp;
                zl_cp16(dbuf + (size_t)r * mzs + 2 * zl_piece(j), tab + ((size_t)(y0 + r) * nh + kx) * mzp + 2 * j);
            }
        }
        zl_commit();
    };

    double2 prev[LPT];
#pragma unroll
    for (int q = 0; q < LPT; q++) prev[q] = make_double2(0.0, 0.0);

    // ------------------------------------------------------------ forward phase
#pragma unroll
    for (int c = 0; c < NS - 1; c++) issue(c, c, a.piv);
    for (int c = 0; c < nch; c++) {
        issue(c + NS - 1, (c + NS - 1) % NS, a.piv);  // that stage was last read in iteration c - 1
        zl_wait<NS - 1>();
        __syncthreads();
        const int s = c % NS, y0 = c * yb, nr = min(yb, ny - y0);
        double2* buf = ring + sidx<true>(s * yb * n);
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
    zl_wait<0>();
    // the backward phase streams back rows other threads of this CTA stored
    __threadfence();
    __syncthreads();

    // ----------------------------------------------------------- backward phase
    // j-th chunk from the top (chunk nch-1-j) uses stage j % NS
#pragma unroll
    for (int j = 0; j < NS - 1; j++) issue(nch - 1 - j, j, a.pivc);
    for (int j = 0; j < nch; j++) {
        issue(nch - 1 - (j + NS - 1), (j + NS - 1) % NS, a.pivc);
        zl_wait<NS - 1>();
        __syncthreads();
        const int s = j % NS, c = nch - 1 - j, y0 = c * yb, nr = min(yb, ny - y0);
        double2* buf = ring + sidx<true>(s * yb * n);
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
    zl_wait<0>();
}

size_t zline_smem(int n, int mzp, int yb, int ns) {
    return (size_t)padded_len(ns * yb * n, true) * sizeof(double2) + (size_t)ns * yb * zl_mzs(mzp) * sizeof(double);
}

template <class PL, int NS, int LPT>
cudaError_t launch_zline_pl(const ZLineArgs& a, size_t smem, cudaStream_t st) {
    cudaError_t e =
        cudaFuncSetAttribute(k_zline<PL, NS, LPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_zline<PL, NS, LPT><<<a.nh, zl_threads(PL::n, LPT), smem, st>>>(a);
    return cudaGetLastError();
}

template <class PL>
cudaError_t launch_zline_ns(const ZLineArgs& a, int ns, size_t smem, cudaStream_t st) {
    constexpr int L = zl_lpt(PL::n);
    switch (ns) {
    case 2: return launch_zline_pl<PL, 2, L>(a, smem, st);
    case 3: return launch_zline_pl<PL, 3, L>(a, smem, st);
    default: return launch_zline_pl<PL, 4, L>(a, smem, st);
    }
}

}  // namespace

bool zline_supported(const prj_plan* pl) {
    if (!pl->use_pass || !pl->zd.ok || !pl->kz_of_slot || !pl->t.pivc) return false;
#define PRJ_ZL_HAS(N, ...)                                                          \
    if (pl->g.nz == N && same_radices<PassList<__VA_ARGS__>>(pl->zd.f))             \
        return zline_smem(N, pl->g.mzp, 1, 2) <= (size_t)200 * 1024;
    PRJ_PASS_ALL(PRJ_ZL_HAS)
#undef PRJ_ZL_HAS
    return false;
}

// cudaErrorNotSupported when nz has no pass plan (the caller runs the split kernels)
cudaError_t launch_zline(const prj_plan* pl, cudaStream_t st) {
    if (!pl->use_pass || !pl->zd.ok || !pl->kz_of_slot || !pl->t.pivc) return cudaErrorNotSupported;
    const Geometry& g = pl->g;
    ZLineArgs a{};
    a.ny = g.ny; a.nh = g.nxh; a.mzp = g.mzp;
    a.tw = pl->zd.tw; a.bands = pl->t.bands; a.piv = pl->t.piv; a.pivc = pl->t.pivc;
    a.kz_of_slot = pl->kz_of_slot; a.X = pl->spec;
    // planes per stage and stage count: the plan's z_planes / z_stages tuning, else 4 x 2;
    // the planes per stage shrink until the ring fits 72 KB (three CTAs per SM).  Measured
    // at 768x384x384 and not kept: deeper rings at fewer CTAs per SM, and one line per
    // thread (twice the threads, spilling at the register budget of three CTAs per SM).
    int yb = pl->z_planes > 0 ? pl->z_planes : 4, ns = pl->z_stages > 0 ? pl->z_stages : 2;
    const size_t cap = (size_t)72 * 1024;
    if (ns < 2 || ns > 4) ns = 2;
    if (yb < 1) yb = 1;
    if (yb > g.ny) yb = g.ny;
    while (yb > 1 && zline_smem(g.nz, g.mzp, yb, ns) > cap) yb--;
    const size_t smem = zline_smem(g.nz, g.mzp, yb, ns);
    if (smem > (size_t)200 * 1024) return cudaErrorNotSupported;
    a.yb = yb;
#define PRJ_ZL_CASE(N, ...)                                                  \
    if (g.nz == N && same_radices<PassList<__VA_ARGS__>>(pl->zd.f))          \
        return launch_zline_ns<PassList<__VA_ARGS__>>(a, ns, smem, st);
    PRJ_PASS_ALL(PRJ_ZL_CASE)
#undef PRJ_ZL_CASE
    return cudaErrorNotSupported;
}

}  // namespace prj

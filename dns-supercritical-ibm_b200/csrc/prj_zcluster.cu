// prj_zcluster.cu -- the z direction of the solve on a thread-block cluster per x
// wavenumber: z FFT, Thomas sweeps and inverse z FFT in one kernel, the work of one
// wavenumber spread over C = R_0 CTAs (R_0 the first radix of the z pass plan).
//
// The in-place DIF transform of a pass plan n = R_0 R_1 ... R_{P-1} starts with one
// pass of radix R_0 and span n: butterfly j (0 <= j < L1 = n / R_0) takes the
// elements j + q' L1 of the row and leaves its output q' at position j of block q'.
// Every later pass works inside one block of L1 elements, and block q ends up holding
// exactly the frequencies k = q (mod R_0), in slot order.  So:
//
//   CTA q of the cluster of x wavenumber kx owns block q of every z-row X[y][kx][:]:
//   the L1 Thomas lines (kx, slot q L1 + t), t < L1;
//   forward, per chunk of yb planes: it loads the inputs of its share J_q of the
//     first-pass butterflies (j in [q JW, q JW + JW), JW = ceil(L1 / C)) for all C
//     blocks, runs those butterflies and stores output q' into block q' of CTA q' in
//     distributed shared memory; after a cluster barrier it runs passes 1 .. P-1 on its
//     own block, then the forward Thomas recurrence d'_y = (d_y - a_y d'_{y-1}) / D_y
//     of its lines, d' stored to the row (slot order);
//   backward, chunks in descending y: it loads its block of the d' rows, runs the back
//     substitution x_y = d'_y - c'_y x_{y+1} and the inverse passes P-1 .. 1 inside the
//     block, sends position j of its block to the CTA that owns butterfly j of the last
//     inverse pass (radix R_0, span n), and after a cluster barrier runs those
//     butterflies and stores natural-order z values.
//
// The butterflies, twiddle tables and the Thomas operation order
// (poisson_solver_multigpu.f90:395-422) are those of k_zfft_pass / k_thomas / k_zline,
// applied to the same elements, so the result is bitwise that of the split kernels.
// The spectrum crosses HBM four times, as in k_zline, but a wavenumber has C CTAs of
// L1/LPT threads instead of one, so nx/2+1 = 385 wavenumbers make 2310 CTAs at
// nz = 384 and more of the chunk pipelines run side by side on every SM.
//
// Pivots: CTA q reads the pivots D and back-substitution factors c' of its lines.  The
// plan keeps, besides the folded tables D[y][kx][kzs], class tables
// Dc[y][kx][c][t] = D[y][kx][kzs(slot c L1 + t)] for c < NC = C/2 + 1: CTA q < NC
// reads row q in its own slot order; CTA q >= NC holds the frequencies n - k of CTA
// C - q (the same folded wavenumbers) and reads row C - q through the position table
// pos[q L1 + t].  That is (C/2+1)/C of a full slot-ordered row (256 instead of 384
// entries at n = 384), each loaded as one contiguous piece.
//
// Synchronisation: cp.async copies (they complete on their own), CTA barriers, and
// the hardware cluster barrier (barrier.cluster.arrive.release / wait.acquire), which
// every thread of every CTA of the cluster reaches the same number of times (the
// chunk loops have the same trip count in every CTA), so no wait depends on a flag.
// Remote stores go to the buffer of the current parity; the barrier of chunk c
// orders them after the receiver's last read of that buffer (chunk c - 2) and before
// its reads in chunk c.
#include <cstdlib>
#include <vector>

#include "div_rn.cuh"
#include "fft_pass.cuh"
#include "prj_internal.h"

namespace prj {

namespace {

template <class PL>
struct SubPlan;
template <int R0, int... Rs>
struct SubPlan<PassList<R0, Rs...>> {
    using type = PassList<Rs...>;
};

template <class PL>
struct ZclShape {
    static constexpr int n = PL::n;
    static constexpr int C = PL::radix(0);
    static constexpr int L1 = n / C;
    static constexpr int JW = (L1 + C - 1) / C;
    static constexpr int NC = C / 2 + 1;
};

struct ZclArgs {
    int ny, nh;
    int yb;               // planes per chunk
    const double2* tw;    // z pass-plan twiddles
    const double* bands;  // a, b, c, a00, b00, c00
    const double* dcls;   // D class tables [y][kx][c][t]
    const double* ccls;   // c' class tables, same layout
    const int* pos;       // pos[slot]: class row * L1 + position of the slot's line
    const int* kz_of_slot;
    double2* X;           // [y][kx][z]
};

__device__ __forceinline__ void zc_cp16(void* dst, const void* src) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void zc_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void zc_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ unsigned zc_rank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void zc_cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// shared::cluster address of the same shared-memory offset in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t zc_mapa(const void* local, unsigned rank) {
    uint32_t r;
    const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(local));
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    return r;
}
__device__ __forceinline__ void zc_st_remote(uint32_t addr, double2 v) {
    asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(addr), "d"(v.x), "d"(v.y) : "memory");
}

__host__ __device__ constexpr int zc_threads(int lines, int lpt) {
    return ((lines + lpt - 1) / lpt + 31) / 32 * 32;
}
// resident CTAs per SM asked of the register allocator: about 96 registers per thread
__host__ __device__ constexpr int zc_minb(int nt) { return 65536 / (nt * 96) < 1 ? 1 : 65536 / (nt * 96); }

// shared-memory layout (bytes), NS stages of yb planes
struct ZclSmem {
    size_t stage, blk, xin, piv, total;
};
template <class PL>
__host__ __device__ inline ZclSmem zcl_smem_layout(int yb, int ns) {
    using S = ZclShape<PL>;
    const size_t in_b = (size_t)yb * S::C * S::JW * sizeof(double2);                 // forward inputs per stage
    const size_t bb_b = (size_t)padded_len(yb * S::L1, true) * sizeof(double2);     // backward block per stage
    const size_t st_b = ((in_b > bb_b ? in_b : bb_b) + 15) / 16 * 16;
    ZclSmem m{};
    m.stage = st_b;
    m.blk = ((size_t)padded_len(yb * S::L1, true) * sizeof(double2) + 15) / 16 * 16;
    m.xin = ((size_t)yb * S::C * S::JW * sizeof(double2) + 15) / 16 * 16;
    m.piv = ((size_t)yb * S::L1 * sizeof(double) + 15) / 16 * 16;
    m.total = (size_t)ns * m.stage + 2 * m.blk + 2 * m.xin + (size_t)ns * m.piv;
    return m;
}

template <class PL, int NS, int LPT>
__global__ void __launch_bounds__(zc_threads(ZclShape<PL>::L1, LPT), zc_minb(zc_threads(ZclShape<PL>::L1, LPT)))
    k_zcl(const ZclArgs a) {
    using Sh = ZclShape<PL>;
    using SUB = typename SubPlan<PL>::type;
    constexpr int n = Sh::n, C = Sh::C, L1 = Sh::L1, JW = Sh::JW, NC = Sh::NC;
    constexpr int NT = zc_threads(L1, LPT);
    extern __shared__ __align__(16) unsigned char zsm[];
    const ZclSmem lay = zcl_smem_layout<PL>(a.yb, NS);
    const int ny = a.ny, nh = a.nh, yb = a.yb, tid = threadIdx.x;
    const unsigned q = zc_rank();
    const int kx = blockIdx.x / C;
    unsigned char* p = zsm;
    unsigned char* stage0 = p;
    p += (size_t)NS * lay.stage;
    double2* blk0 = reinterpret_cast<double2*>(p);
    p += 2 * lay.blk;
    double2* xin0 = reinterpret_cast<double2*>(p);
    p += 2 * lay.xin;
    double* piv0 = reinterpret_cast<double*>(p);
    auto stage_in = [&](int s) { return reinterpret_cast<double2*>(stage0 + (size_t)s * lay.stage); };
    auto blk = [&](int par) { return reinterpret_cast<double2*>(reinterpret_cast<unsigned char*>(blk0) + par * lay.blk); };
    auto xin = [&](int par) { return reinterpret_cast<double2*>(reinterpret_cast<unsigned char*>(xin0) + par * lay.xin); };
    auto pivs = [&](int s) { return reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(piv0) + s * lay.piv); };
    const int nch = (ny + yb - 1) / yb;
    const int j0 = (int)q * JW;
    const int jn = min(JW, L1 - j0);  // first / last pass butterflies of this CTA (may be < JW)
    const int cls = (int)q < NC ? (int)q : C - (int)q;
    const double2* twsub = a.tw + PL::twoff(1);

    // this thread's lines: t = tid + u NT of the block
    int tl[LPT], pp[LPT];
    bool is00[LPT];
#pragma unroll
    for (int u = 0; u < LPT; u++) {
        tl[u] = tid + u * NT;
        const int slot = (int)q * L1 + (tl[u] < L1 ? tl[u] : 0);
        pp[u] = a.pos[slot] - cls * L1;  // position in the class row
        is00[u] = (kx == 0 && a.kz_of_slot[slot] == 0 && tl[u] < L1);
    }
    const double* bA = a.bands;
    const double* bA0 = a.bands + 3 * ny;
    double2* Xk = a.X + (size_t)kx * n;  // row (y, kx) starts at Xk + y nh n
    const size_t ystr = (size_t)nh * n;

    // every CTA of the cluster has started before any remote store
    zc_cluster_sync();

    // ------------------------------------------------------------------ forward
    auto issue_f = [&](int c, int s) {
        if (c >= 0 && c < nch) {
            const int y0 = c * yb, nr = min(yb, ny - y0);
            double2* in = stage_in(s);
            const int per = C * jn;
            for (int i = tid; i < nr * per; i += NT) {
                const int r = i / per, rem = i - r * per, qq = rem / jn, jj = rem - qq * jn;
                zc_cp16(&in[(r * C + qq) * JW + jj], Xk + (size_t)(y0 + r) * ystr + j0 + jj + qq * L1);
            }
            double* pv = pivs(s);
            constexpr int hp = L1 / 2;  // 16-byte pieces of a class row
            for (int i = tid; i < nr * hp; i += NT) {
                const int r = i / hp, e = i - r * hp;
                zc_cp16(pv + (size_t)r * L1 + 2 * e, a.dcls + (((size_t)(y0 + r) * nh + kx) * NC + cls) * L1 + 2 * e);
            }
        }
        zc_commit();
    };

    double2 prev[LPT];
#pragma unroll
    for (int u = 0; u < LPT; u++) prev[u] = make_double2(0.0, 0.0);

#pragma unroll
    for (int c = 0; c < NS - 1; c++) issue_f(c, c);
    for (int c = 0; c < nch; c++) {
        issue_f(c + NS - 1, (c + NS - 1) % NS);  // that stage was last read in chunk c - 1
        zc_wait<NS - 1>();
        __syncthreads();
        const int s = c % NS, par = c & 1, y0 = c * yb, nr = min(yb, ny - y0);
        const double2* in = stage_in(s);
        double2* bk = blk(par);
        // first DIF pass (radix C, span n) of this CTA's butterflies; output q' to CTA q'
        for (int i = tid; i < nr * jn; i += NT) {
            const int r = i / jn, jj = i - r * jn, j = j0 + jj;
            double2 v[C];
#pragma unroll
            for (int qq = 0; qq < C; qq++) v[qq] = in[(r * C + qq) * JW + jj];
            dft_r<-1, C>(v);
            if (L1 > 1 && j) apply_twiddles<-1, C, L1>(v, a.tw, j);
            const double2* dst = &bk[sidx<true>(r * L1 + j)];
#pragma unroll
            for (int qq = 0; qq < C; qq++) zc_st_remote(zc_mapa(dst, qq), v[qq]);
        }
        zc_cluster_sync();
        // passes 1 .. P-1 inside this CTA's block
        dif_passes_shared<-1, SUB, 0, SUB::P>(bk, nr, L1, twsub);  // barrier after every pass
        const double* pv = pivs(s);
        for (int r = 0; r < nr; r++) {
            const int y = y0 + r;
            double2* grow = Xk + (size_t)y * ystr + (size_t)q * L1;
#pragma unroll
            for (int u = 0; u < LPT; u++) {
                if (tl[u] < L1) {
                    double2 v = bk[sidx<true>(r * L1 + tl[u])];
                    const double D = pv[(size_t)r * L1 + pp[u]];
                    const double rD = __drcp_rn(D);  // off the recurrence's chain
                    if (y == 0) {
                        v.x = div_by_recip(v.x, D, rD);
                        v.y = div_by_recip(v.y, D, rD);
                    } else {
                        const double av = is00[u] ? bA0[y] : bA[y];
                        v.x = div_by_recip(__dsub_rn(v.x, __dmul_rn(av, prev[u].x)), D, rD);
                        v.y = div_by_recip(__dsub_rn(v.y, __dmul_rn(av, prev[u].y)), D, rD);
                    }
                    prev[u] = v;
                    grow[tl[u]] = v;
                }
            }
        }
        __syncthreads();
    }
    zc_wait<0>();
    // the backward phase streams back the d' rows this CTA's threads stored
    __threadfence();
    __syncthreads();

    // ----------------------------------------------------------------- backward
    auto issue_b = [&](int c, int s) {
        if (c >= 0 && c < nch) {
            const int y0 = c * yb, nr = min(yb, ny - y0);
            double2* bb = stage_in(s);
            for (int i = tid; i < nr * L1; i += NT) {
                const int r = i / L1, e = i - r * L1;
                zc_cp16(&bb[sidx<true>(r * L1 + e)], Xk + (size_t)(y0 + r) * ystr + (size_t)q * L1 + e);
            }
            double* pv = pivs(s);
            constexpr int hp = L1 / 2;
            for (int i = tid; i < nr * hp; i += NT) {
                const int r = i / hp, e = i - r * hp;
                zc_cp16(pv + (size_t)r * L1 + 2 * e, a.ccls + (((size_t)(y0 + r) * nh + kx) * NC + cls) * L1 + 2 * e);
            }
        }
        zc_commit();
    };
#pragma unroll
    for (int j = 0; j < NS - 1; j++) issue_b(nch - 1 - j, j);
    for (int j = 0; j < nch; j++) {
        issue_b(nch - 1 - (j + NS - 1), (j + NS - 1) % NS);
        zc_wait<NS - 1>();
        __syncthreads();
        const int s = j % NS, par = j & 1, c = nch - 1 - j, y0 = c * yb, nr = min(yb, ny - y0);
        double2* bb = stage_in(s);
        const double* pv = pivs(s);
        for (int r = nr - 1; r >= 0; r--) {
            const int y = y0 + r;
#pragma unroll
            for (int u = 0; u < LPT; u++) {
                if (tl[u] < L1) {
                    double2& cell = bb[sidx<true>(r * L1 + tl[u])];
                    const double2 d = cell;
                    if (y == ny - 1) {
                        prev[u] = d;
                    } else {
                        const double Cf = pv[(size_t)r * L1 + pp[u]];  // c_y / D_y
                        prev[u].x = __dsub_rn(d.x, __dmul_rn(prev[u].x, Cf));
                        prev[u].y = __dsub_rn(d.y, __dmul_rn(prev[u].y, Cf));
                    }
                    cell = prev[u];
                }
            }
        }
        __syncthreads();
        dit_passes_shared<+1, SUB, SUB::P - 1, -1>(bb, nr, L1, twsub);  // passes P-1 .. 1, barrier after each
        // position e of this block goes to the owner of last-pass butterfly e
        double2* xb = xin(par);
        for (int i = tid; i < nr * L1; i += NT) {
            const int r = i / L1, e = i - r * L1, g = e / JW, jj = e - g * JW;
            zc_st_remote(zc_mapa(&xb[(r * C + (int)q) * JW + jj], g), bb[sidx<true>(r * L1 + e)]);
        }
        zc_cluster_sync();
        // last DIT pass (pass 0: radix C, span n) of this CTA's butterflies, natural order out
        for (int i = tid; i < nr * jn; i += NT) {
            const int r = i / jn, jj = i - r * jn, jg = j0 + jj;
            double2 v[C];
#pragma unroll
            for (int qq = 0; qq < C; qq++) v[qq] = xb[(r * C + qq) * JW + jj];
            if (L1 > 1 && jg) apply_twiddles<+1, C, L1>(v, a.tw, jg);
            dft_r<+1, C>(v);
            double2* row = Xk + (size_t)(y0 + r) * ystr + jg;
#pragma unroll
            for (int qq = 0; qq < C; qq++) row[qq * L1] = v[qq];
        }
    }
    zc_wait<0>();
    // no CTA leaves while another may still address its shared memory
    zc_cluster_sync();
}

}  // namespace

namespace {

// class tables of the pivots and back-substitution factors (layout of k_zcl)
__global__ void k_build_cls(int ny, int nh, int mzp, int n, int nc, int l1, const int* __restrict__ kz_of_slot,
                            const double* __restrict__ piv, const double* __restrict__ pivc, double* dcls,
                            double* ccls) {
    const size_t tot = (size_t)ny * nh * nc * l1;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < tot; i += (size_t)gridDim.x * blockDim.x) {
        const int t = (int)(i % l1);
        const size_t rest = i / l1;
        const int c = (int)(rest % nc);
        const size_t yk = rest / nc;  // y nh + kx
        const int kz = kz_of_slot[c * l1 + t];
        const int kf = kz <= n - kz ? kz : n - kz;
        dcls[i] = piv[yk * mzp + kf];
        ccls[i] = pivc[yk * mzp + kf];
    }
}

template <class PL, int NS, int LPT>
cudaError_t zcl_launch_pl(const ZclArgs& a, size_t smem, cudaStream_t st) {
    using Sh = ZclShape<PL>;
    auto kern = k_zcl<PL, NS, LPT>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)(a.nh * Sh::C));
    cfg.blockDim = dim3((unsigned)zc_threads(Sh::L1, LPT));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = Sh::C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, a);
}

// lines per thread: one up to 128 lines of a block, then two, four
template <class PL>
constexpr int zcl_lpt() {
    return ZclShape<PL>::L1 <= 128 ? 1 : ZclShape<PL>::L1 <= 256 ? 2 : 4;
}

template <class PL>
cudaError_t zcl_launch_ns(const ZclArgs& a, int ns, cudaStream_t st) {
    constexpr int L = zcl_lpt<PL>();
    const size_t smem = zcl_smem_layout<PL>(a.yb, ns).total;
    switch (ns) {
    case 2: return zcl_launch_pl<PL, 2, L>(a, smem, st);
    case 4: return zcl_launch_pl<PL, 4, L>(a, smem, st);
    default: return zcl_launch_pl<PL, 3, L>(a, smem, st);
    }
}

template <class PL>
size_t zcl_smem_bytes(int yb, int ns) {
    return zcl_smem_layout<PL>(yb, ns).total;
}

// cluster size, block length and class count of the pass plan of length n (0 if none)
bool zcl_shape_of(int n, int* C, int* L1, int* NC) {
    switch (n) {
#define PRJ_ZC_SHAPE(N, ...)                          \
    case N: {                                         \
        using Sh = ZclShape<PassList<__VA_ARGS__>>;   \
        *C = Sh::C; *L1 = Sh::L1; *NC = Sh::NC;       \
        return true;                                  \
    }
        PRJ_PASS_PLANS(PRJ_ZC_SHAPE)
#undef PRJ_ZC_SHAPE
    default:
        return false;
    }
}

}  // namespace

size_t zcl_smem(int nz, int yb, int ns) {
    switch (nz) {
#define PRJ_ZC_SMEM(N, ...) \
    case N: return zcl_smem_bytes<PassList<__VA_ARGS__>>(yb, ns);
        PRJ_PASS_PLANS(PRJ_ZC_SMEM)
#undef PRJ_ZC_SMEM
    default:
        return 0;
    }
}

bool zcl_supported(const prj_plan* pl) {
    if (!pl->use_pass || !pl->zd.ok || !pl->kz_of_slot || !pl->t.pivc) return false;
    int C = 0, L1 = 0, NC = 0;
    if (!zcl_shape_of(pl->g.nz, &C, &L1, &NC)) return false;
    switch (pl->g.nz) {
#define PRJ_ZC_SAME(N, ...) \
    case N: if (!same_radices<PassList<__VA_ARGS__>>(pl->zd.f)) return false; break;
        PRJ_PASS_PLANS(PRJ_ZC_SAME)
#undef PRJ_ZC_SAME
    default:
        return false;
    }
    return C >= 2 && C <= 8 && zcl_smem(pl->g.nz, 1, 2) <= (size_t)200 * 1024;
}

// class tables and position table of k_zcl (built once; tables of the plan's pivots)
cudaError_t zcl_prepare(prj_plan* pl, cudaStream_t st) {
    if (pl->zcl_dcls) return cudaSuccess;
    int C = 0, L1 = 0, NC = 0;
    if (!zcl_shape_of(pl->g.nz, &C, &L1, &NC)) return cudaErrorNotSupported;
    const Geometry& g = pl->g;
    const int n = g.nz;
    // slot -> wavenumber on the host (the plan's slot table), then the position table
    std::vector<int> kz(n), pos(n);
    cudaError_t e = cudaMemcpy(kz.data(), pl->kz_of_slot, n * sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return e;
    for (int q = 0; q < C; q++) {
        const int cls = q < NC ? q : C - q;
        for (int t = 0; t < L1; t++) {
            const int s = q * L1 + t;
            if (cls == q) {
                pos[s] = q * L1 + t;
                continue;
            }
            const int want = (n - kz[s]) % n;  // the same folded wavenumber in CTA C - q
            int found = -1;
            for (int t2 = 0; t2 < L1; t2++)
                if (kz[cls * L1 + t2] == want) { found = t2; break; }
            if (found < 0) return cudaErrorInvalidValue;  // a plan whose blocks are not frequency classes
            pos[s] = cls * L1 + found;
        }
    }
    const size_t ne = (size_t)g.ny * g.nxh * NC * L1;
    double *dc = nullptr, *cc = nullptr;
    int* dp = nullptr;
    if ((e = cudaMalloc((void**)&dc, ne * sizeof(double))) != cudaSuccess) return e;
    if ((e = cudaMalloc((void**)&cc, ne * sizeof(double))) != cudaSuccess) { cudaFree(dc); return e; }
    if ((e = cudaMalloc((void**)&dp, n * sizeof(int))) != cudaSuccess) { cudaFree(dc); cudaFree(cc); return e; }
    if ((e = cudaMemcpy(dp, pos.data(), n * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess) {
        cudaFree(dc); cudaFree(cc); cudaFree(dp);
        return e;
    }
    const int blocks = (int)std::min<size_t>((ne + 255) / 256, 148 * 16);
    k_build_cls<<<blocks, 256, 0, st>>>(g.ny, g.nxh, g.mzp, n, NC, L1, pl->kz_of_slot, pl->t.piv, pl->t.pivc, dc, cc);
    if ((e = cudaGetLastError()) != cudaSuccess) { cudaFree(dc); cudaFree(cc); cudaFree(dp); return e; }
    pl->zcl_dcls = dc;
    pl->zcl_ccls = cc;
    pl->zcl_pos = dp;
    pl->device_bytes += 2 * ne * sizeof(double) + n * sizeof(int);
    return cudaSuccess;
}

// cudaErrorNotSupported when nz has no pass plan or the tables are missing
cudaError_t launch_zcl(const prj_plan* pl, cudaStream_t st) {
    if (!pl->zcl_dcls || !zcl_supported(pl)) return cudaErrorNotSupported;
    const Geometry& g = pl->g;
    ZclArgs a{};
    a.ny = g.ny; a.nh = g.nxh;
    a.tw = pl->zd.tw; a.bands = pl->t.bands; a.dcls = pl->zcl_dcls; a.ccls = pl->zcl_ccls; a.pos = pl->zcl_pos;
    a.kz_of_slot = pl->kz_of_slot; a.X = pl->spec;
    int yb = pl->z_planes > 0 ? pl->z_planes : 4, ns = pl->z_stages > 0 ? pl->z_stages : 3;
    if (ns < 2 || ns > 4) ns = 3;
    if (yb > g.ny) yb = g.ny;
    while (yb > 1 && zcl_smem(g.nz, yb, ns) > (size_t)100 * 1024) yb--;
    a.yb = yb;
    switch (g.nz) {
#define PRJ_ZC_CASE(N, ...)                                                  \
    case N: {                                                                \
        using PL = PassList<__VA_ARGS__>;                                    \
        if (!same_radices<PL>(pl->zd.f)) return cudaErrorNotSupported;       \
        return zcl_launch_ns<PL>(a, ns, st);                                 \
    }
        PRJ_PASS_PLANS(PRJ_ZC_CASE)
#undef PRJ_ZC_CASE
    default:
        return cudaErrorNotSupported;
    }
}

}  // namespace prj

// prj_zline.cu -- the z direction of the solve as one kernel per x wavenumber,
// built on the pass-plan butterflies (fft_pass.cuh).
//
// One CTA owns one x wavenumber kx: the ny spectral z-rows X[y][kx][:] and the nz
// Thomas lines (kx, slot) that run through them (zline_tile, zline_tiles.cuh: z FFT,
// both Thomas sweeps and the inverse z FFT, the spectrum crossing HBM four times).
// Each thread owns LPT lines (slots tid + q NT) and carries their recurrence in
// registers.
#include "div_rn.cuh"
#include "fft_pass.cuh"
#include "prj_internal.h"
#include "zline_tiles.cuh"

namespace prj {

namespace {

template <class PL, int NS, int LPT>
__global__ void __launch_bounds__(zl_threads(PL::n, LPT), zl_minb(zl_threads(PL::n, LPT))) k_zline(const ZLineArgs a) {
    extern __shared__ __align__(16) unsigned char zsm[];
    zline_tile<PL, NS, LPT, zl_threads(PL::n, LPT)>(a, blockIdx.x, zsm);
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

ZLineArgs zline_args(const prj_plan* pl) {
    const Geometry& g = pl->g;
    ZLineArgs a{};
    a.ny = g.ny; a.nh = g.nxh; a.mzp = g.mzp;
    a.yb = pl->z_planes > 0 ? pl->z_planes : 4;
    a.tw = pl->zd.tw; a.bands = pl->t.bands; a.piv = pl->t.piv; a.pivc = pl->t.pivc;
    a.kz_of_slot = pl->kz_of_slot; a.X = pl->spec;
    return a;
}

// cudaErrorNotSupported when nz has no pass plan (the caller runs the split kernels)
cudaError_t launch_zline(const prj_plan* pl, cudaStream_t st) {
    if (!pl->use_pass || !pl->zd.ok || !pl->kz_of_slot || !pl->t.pivc) return cudaErrorNotSupported;
    const Geometry& g = pl->g;
    ZLineArgs a = zline_args(pl);
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

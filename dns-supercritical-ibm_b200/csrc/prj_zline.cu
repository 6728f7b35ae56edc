// prj_zline.cu -- the z direction of the solve as one kernel per x wavenumber,
// built on the pass-plan butterflies (fft_pass.cuh).
//
// One CTA owns one x wavenumber kx: the ny spectral z-rows X[y][kx][:] and the nz
// Thomas lines (kx, slot) that run through them (zline_tile, zline_tiles.cuh: z FFT,
// both Thomas sweeps and the inverse z FFT, the spectrum crossing HBM four times).
// Each thread owns LPT lines (slots tid + q NT) and carries their recurrence in
// registers.  The rows of each chunk of planes arrive by one TMA copy through a 4-D
// tensor map of the spectrum (zline_tmap, encoded on the host for every launch with the
// driver's cuTensorMapEncodeTiled); a map the driver refuses sends the solve to the split
// kernels.
#include <cuda.h>

#include "div_rn.cuh"
#include "fft_pass.cuh"
#include "prj_internal.h"
#include "zline_tiles.cuh"

namespace prj {

namespace {

// `tmap` (zline_tmap) is a kernel parameter: the TMA unit reads it from parameter space
template <class PL, int NS, int LPT>
__global__ void __launch_bounds__(zl_threads(PL::n, LPT), zl_minb(zl_threads(PL::n, LPT)))
    k_zline(const __grid_constant__ ZLineArgs a, const __grid_constant__ CUtensorMap tmap) {
    extern __shared__ __align__(128) unsigned char zsm[];
    zline_tile<PL, NS, LPT, zl_threads(PL::n, LPT)>(a, &tmap, blockIdx.x, zsm);
}

template <class PL, int NS, int LPT>
cudaError_t launch_zline_pl(const ZLineArgs& a, const CUtensorMap& tm, size_t smem, cudaStream_t st) {
    cudaError_t e =
        cudaFuncSetAttribute(k_zline<PL, NS, LPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_zline<PL, NS, LPT><<<a.nh, zl_threads(PL::n, LPT), smem, st>>>(a, tm);
    return cudaGetLastError();
}

template <class PL>
cudaError_t launch_zline_ns(const ZLineArgs& a, const CUtensorMap& tm, int ns, size_t smem, cudaStream_t st) {
    constexpr int L = zl_lpt(PL::n);
    switch (ns) {
    case 2: return launch_zline_pl<PL, 2, L>(a, tm, smem, st);
    case 3: return launch_zline_pl<PL, 3, L>(a, tm, smem, st);
    default: return launch_zline_pl<PL, 4, L>(a, tm, smem, st);
    }
}


}  // namespace

bool zline_supported(const prj_plan* pl) {
    if (!pl->use_pass || !pl->zd.ok || !pl->kz_of_slot || !pl->t.pivc || !pl->spec) return false;
    CUtensorMap tm{};
    if (!zline_tmap(&tm, pl->spec, pl->g.nz, pl->g.nxh, pl->g.ny, 1)) return false;  // the driver's answer
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
    a.err = reinterpret_cast<int*>(pl->stat_buf + kStatErrSlot);
    return a;
}

bool tmap_encode_f64(void* tmap128, const void* base, int rank, const uint64_t* dims, const uint64_t* strides,
                     const uint32_t* box) {
    using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static const Encode enc = []() -> Encode {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<Encode>(fn);
    }();
    if (!enc || !base || rank < 1 || rank > 5 || ((uintptr_t)base & 15u) != 0) return false;
    cuuint64_t d[5], st[4];
    cuuint32_t b[5], e[5];
    for (int i = 0; i < rank; i++) {
        d[i] = dims[i];
        b[i] = box[i];
        e[i] = 1;
        if (i + 1 < rank) st[i] = strides[i];
    }
    return enc(static_cast<CUtensorMap*>(tmap128), CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (cuuint32_t)rank,
               const_cast<void*>(base), d, st, b, e, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool zline_tmap(void* tmap128, const double2* X, int n, int nh, int ny, int yb) {
    if (n % 8 != 0 || n / 8 > 256 || yb < 1 || yb > 256) return false;
    const uint64_t dims[4] = {16, (uint64_t)(n / 8), (uint64_t)nh, (uint64_t)ny};
    const uint64_t strides[3] = {128, (uint64_t)n * 16, (uint64_t)nh * (uint64_t)n * 16};  // bytes
    const uint32_t box[4] = {18, (uint32_t)(n / 8), 1, (uint32_t)yb};
    return tmap_encode_f64(tmap128, X, 4, dims, strides, box);
}

// cudaErrorNotSupported when nz has no pass plan (the caller runs the split kernels)
cudaError_t launch_zline(const prj_plan* pl, cudaStream_t st) {
    if (!pl->use_pass || !pl->zd.ok || !pl->kz_of_slot || !pl->t.pivc || !pl->spec) return cudaErrorNotSupported;
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
    CUtensorMap tm{};
    if (!zline_tmap(&tm, pl->spec, g.nz, g.nxh, g.ny, yb)) return cudaErrorNotSupported;  // split kernels
#define PRJ_ZL_CASE(N, ...)                                                  \
    if (g.nz == N && same_radices<PassList<__VA_ARGS__>>(pl->zd.f))          \
        return launch_zline_ns<PassList<__VA_ARGS__>>(a, tm, ns, smem, st);
    PRJ_PASS_ALL(PRJ_ZL_CASE)
#undef PRJ_ZL_CASE
    return cudaErrorNotSupported;
}

}  // namespace prj

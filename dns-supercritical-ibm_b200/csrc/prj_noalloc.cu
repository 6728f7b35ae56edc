// prj_noalloc.cu -- the FP64 Poisson solve for callers that cannot allocate
// device memory.
//
// Some host programs own all device memory themselves: an OpenACC or Fortran
// runtime that maps every array up front, a solver embedded in a time loop
// that must not call cudaMalloc (which can synchronise the whole device and
// fail under a memory cap), or a caller running where no allocator may be
// invoked.  prj_poisson_fp64_noalloc serves them: it takes the bands, the grid
// spacings and the device array P, and does all of its work in one fixed
// scratch array that is part of the library image instead of in a plan.
//
// The scratch array is a file-scope __device__ array of
// PRJ_NOALLOC_SCRATCH_BYTES (64 MiB).  Every GPU on which the library is used
// holds it until the process exits.  In host code its name only stands for the
// symbol; the device address is resolved with cudaGetSymbolAddress once per
// device, on that device's first call, and passed to the kernels.  Every call
// shares the array and finds there what the previous call left; the entry
// point therefore re-initialises every region it reads (tables, pivot table,
// the min-pivot slot) before use.  Two calls whose work overlapped on the GPU
// would race on the array: this entry point is synchronous and takes a process
// lock for its whole duration, so calls made through it never overlap.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/projection.h"
#include "div_rn.cuh"
#include "prj_internal.h"

namespace {

constexpr size_t kScratchBytes = PRJ_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;
constexpr size_t kHostTableBytes = (size_t)8 << 20;

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_dev_ptr[kMaxDevices] = {};
alignas(256) unsigned char g_host_tables[kHostTableBytes];  // staging of the small tables, no heap
// failures are reported through prj_last_error_string, like every other entry point
int na_fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return prj::record_error(code, buf);
}

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

// radix sequence, same rule as the planned path
int na_factorize(int n, int* fac) {
    int nf = 0, m = n;
    while (m % 8 == 0 && m != 16) { fac[nf++] = 8; m /= 8; }
    while (m % 4 == 0) { fac[nf++] = 4; m /= 4; }
    while (m % 2 == 0) { fac[nf++] = 2; m /= 2; }
    for (int r : {3, 5}) while (m % r == 0) { fac[nf++] = r; m /= r; }
    for (int r = 7; m > 1; r += 2) {
        while (m % r == 0) { fac[nf++] = r; m /= r; }
        if ((long)r * r > m && m > 1) { fac[nf++] = m; m = 1; }
        if (nf >= prj::kMaxStages) return -1;
    }
    return nf;
}

double2 na_cexpm(long double num, long double den) {
    const long double a = 6.283185307179586476925286766559005768L * num / den;
    return make_double2((double)cosl(a), (double)(-sinl(a)));
}

// number of twiddle entries of a complex FFT of length n (stage twiddles + roots)
long na_tw_count(int n, prj::FftDev* f) {
    int fac[prj::kMaxStages + 8];
    const int nf = na_factorize(n, fac);
    if (nf < 0 || nf > prj::kMaxStages) return -1;
    std::memset(f, 0, sizeof(*f));
    f->n = n;
    f->nst = nf;
    long cnt = 0;
    int p = 1;
    for (int s = 0; s < nf; s++) {
        const int R = fac[s];
        if (R > 64) return -2;
        f->radix[s] = R;
        f->p[s] = p;
        f->twoff[s] = (int)cnt;
        cnt += (long)p * (R - 1);
        if (!(R == 2 || R == 3 || R == 4 || R == 5 || R == 8)) cnt += R;
        p *= R;
    }
    return cnt > 0 ? cnt : 1;
}

void na_tw_fill(const prj::FftDev& f, double2* out) {
    long c = 0;
    for (int s = 0; s < f.nst; s++) {
        const int R = f.radix[s], p = f.p[s];
        for (int k = 0; k < p; k++)
            for (int r = 1; r < R; r++) out[c++] = na_cexpm((long double)r * k, (long double)p * R);
        if (!(R == 2 || R == 3 || R == 4 || R == 5 || R == 8))
            for (int m = 0; m < R; m++) out[c++] = na_cexpm((long double)m, (long double)R);
    }
    if (c == 0) out[0] = na_cexpm(0, 1);
}

}  // namespace

extern "C" int prj_poisson_fp64_noalloc(int nx, int nz, int ny, double dx, double dz, const double* band_a,
                                        const double* band_b, const double* band_c, const double* band_a00,
                                        const double* band_b00, const double* band_c00, double* d_P,
                                        void* stream) {
    if (nx < 1 || nx > 8192 || nz < 1 || nz > 4094 || ny < 2 || ny > 65536)
        return na_fail(PRJ_ERR_ARG, "grid %d x %d x %d outside the limits of prj_plan_create", nx, nz, ny);
    if (!(dx > 0) || !(dz > 0) || !std::isfinite(dx) || !std::isfinite(dz))
        return na_fail(PRJ_ERR_ARG, "dx=%g, dz=%g must be finite and positive", dx, dz);
    const double* bandv[6] = {band_a, band_b, band_c, band_a00, band_b00, band_c00};
    for (int i = 0; i < 6; i++) {
        if (!bandv[i]) return na_fail(PRJ_ERR_ARG, "band pointer %d is NULL", i);
        for (int k = 0; k < ny; k++)
            if (!std::isfinite(bandv[i][k])) return na_fail(PRJ_ERR_ARG, "band array %d holds a non-finite value", i);
    }
    if (!d_P) return na_fail(PRJ_ERR_ARG, "P is NULL");

    // geometry and FFT descriptors, exactly as prj_plan_create builds them
    prj_plan pl;  // stack descriptor: every device pointer below points into the scratch array
    prj::Geometry& g = pl.g;
    g.nx = nx; g.nz = nz; g.ny = ny; g.dx = dx; g.dz = dz;
    g.nxh = nx / 2 + 1;
    g.nzh = nz / 2 + 1;
    g.mzp = (g.nzh + 1) / 2 * 2;
    pl.fx64.n = nx;
    pl.fx64.nh = nx / 2 + 1;
    pl.fx64.even = (nx % 2 == 0);
    pl.fx64.m = pl.fx64.even ? nx / 2 : nx;
    const long ntwx = na_tw_count(pl.fx64.m, &pl.fx64.f);
    const long ntwz = na_tw_count(nz, &pl.fz64.f);
    if (ntwx < 0 || ntwz < 0) return na_fail(PRJ_ERR_UNSUPPORTED, "FFT length with a prime factor > 64");
    {
        const size_t per_row = (size_t)2 * (pl.fx64.m + 1) * sizeof(double2);
        int tz = (int)((100 * 1024) / per_row);
        pl.tz_fwd = tz > 16 ? 16 : (tz < 1 ? 1 : tz);
    }

    // scratch layout
    const size_t o_stat = 0;
    const size_t o_twx = align256(o_stat + 8 * sizeof(double));
    const size_t o_post = align256(o_twx + (size_t)ntwx * sizeof(double2));
    const size_t o_twz = align256(o_post + (size_t)(pl.fx64.m + 1) * sizeof(double2));
    const size_t o_ax = align256(o_twz + (size_t)ntwz * sizeof(double2));
    const size_t o_az = align256(o_ax + (size_t)g.nxh * sizeof(double));
    const size_t o_bands = align256(o_az + (size_t)g.nzh * sizeof(double));
    const size_t o_piv = align256(o_bands + (size_t)6 * ny * sizeof(double));
    const size_t o_spec = align256(o_piv + (size_t)ny * g.nxh * g.mzp * sizeof(double));
    const size_t need = align256(o_spec + (size_t)ny * g.nxh * nz * sizeof(double2));
    if (need > kScratchBytes)
        return na_fail(PRJ_ERR_ARG,
                       "grid %d x %d x %d needs %zu bytes of scratch; the no-allocation solve holds %zu bytes "
                       "(use prj_plan_create / prj_poisson_fp64 for larger grids)",
                       nx, nz, ny, need, kScratchBytes);
    const size_t table_bytes = o_piv - o_twx;
    if (table_bytes > kHostTableBytes) return na_fail(PRJ_ERR_ARG, "tables of %zu bytes exceed the staging area", table_bytes);

    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return na_fail(PRJ_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return na_fail(PRJ_ERR_UNSUPPORTED, "device %d beyond %d", dev, kMaxDevices);
    if (!g_noalloc_dev_ptr[dev]) {
        // first call on this device (current device): resolve the array's device address
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return na_fail(PRJ_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
        g_noalloc_dev_ptr[dev] = ptr;
    }
    unsigned char* base = static_cast<unsigned char*>(g_noalloc_dev_ptr[dev]);

    // host tables in the static staging area (same values as the planned path)
    unsigned char* h = g_host_tables;
    std::memset(h, 0, table_bytes);
    na_tw_fill(pl.fx64.f, reinterpret_cast<double2*>(h + (o_twx - o_twx)));
    double2* post = reinterpret_cast<double2*>(h + (o_post - o_twx));
    for (int k = 0; k <= pl.fx64.m; k++) post[k] = na_cexpm((long double)k, (long double)nx);
    na_tw_fill(pl.fz64.f, reinterpret_cast<double2*>(h + (o_twz - o_twx)));
    const double const_pi = 4.0 * std::atan(1.0);
    const double inv_dx = 1.0 / dx, inv_dz = 1.0 / dz;
    double* ax = reinterpret_cast<double*>(h + (o_ax - o_twx));
    double* az = reinterpret_cast<double*>(h + (o_az - o_twx));
    for (int i = 0; i < g.nxh; i++) {
        const double s = std::sin(i * const_pi / nx);
        ax[i] = -4 * (inv_dx * inv_dx) * (s * s);
    }
    for (int j = 0; j < g.nzh; j++) {
        const double s = std::sin(j * const_pi / nz);
        az[j] = -4 * (inv_dz * inv_dz) * (s * s);
    }
    double* bands = reinterpret_cast<double*>(h + (o_bands - o_twx));
    for (int i = 0; i < 6; i++) std::memcpy(bands + (size_t)i * ny, bandv[i], sizeof(double) * ny);

    pl.stat_buf = reinterpret_cast<double*>(base + o_stat);
    pl.fx64.tw = reinterpret_cast<double2*>(base + o_twx);
    pl.fx64.post = reinterpret_cast<double2*>(base + o_post);
    pl.fz64.tw = reinterpret_cast<double2*>(base + o_twz);
    pl.t.ax = reinterpret_cast<double*>(base + o_ax);
    pl.t.az = reinterpret_cast<double*>(base + o_az);
    pl.t.bands = reinterpret_cast<double*>(base + o_bands);
    pl.t.piv = reinterpret_cast<double*>(base + o_piv);
    pl.spec = reinterpret_cast<double2*>(base + o_spec);

    cudaStream_t st = (cudaStream_t)stream;
    if ((e = cudaMemcpyAsync(base + o_twx, h, table_bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return na_fail(PRJ_ERR_CUDA, "table upload: %s", cudaGetErrorString(e));
    // pivot table; its launcher also resets the min-pivot slot
    if ((e = prj::launch_build_pivots(&pl, st)) != cudaSuccess)
        return na_fail(PRJ_ERR_CUDA, "pivot table: %s", cudaGetErrorString(e));
    double mm[2] = {0.0, 0.0};  // smallest and largest |pivot|
    if ((e = cudaMemcpyAsync(mm, pl.stat_buf, sizeof(mm), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return na_fail(PRJ_ERR_CUDA, "pivot table: %s", cudaGetErrorString(e));
    const double minpiv = mm[0];
    if (!(minpiv > 0) || !std::isfinite(minpiv))
        return na_fail(PRJ_ERR_NUMERIC, "zero or non-finite Thomas pivot (min_abs_div_bacp = %g)", minpiv);
    if (!(minpiv >= prj::kDivRecipMinD) || !(mm[1] <= prj::kDivRecipMaxD))
        return na_fail(PRJ_ERR_NUMERIC, "Thomas pivots |D| in [%g, %g] leave the range [2^-40, 2^1000] of the "
                                        "correctly rounded division", minpiv, mm[1]);
    // the error word of the bounded device waits (the z kernel's copy pipeline): cleared
    // here, because the array keeps whatever the previous call left, and read back below
    int* err_word = reinterpret_cast<int*>(pl.stat_buf + prj::kStatErrSlot);
    if ((e = cudaMemsetAsync(err_word, 0, sizeof(int), st)) != cudaSuccess)
        return na_fail(PRJ_ERR_CUDA, "error word: %s", cudaGetErrorString(e));
    if ((e = prj::launch_fwd_x(&pl, prj::FwdSource::Pressure, d_P, nullptr, nullptr, nullptr, nullptr, st)) != cudaSuccess ||
        (e = prj::launch_zsolve(&pl, st)) != cudaSuccess || (e = prj::launch_bwd_x(&pl, d_P, st)) != cudaSuccess)
        return na_fail(PRJ_ERR_CUDA, "solve: %s", cudaGetErrorString(e));
    int dev_err = 0;
    if ((e = cudaMemcpyAsync(&dev_err, err_word, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return na_fail(PRJ_ERR_CUDA, "solve: %s", cudaGetErrorString(e));
    if (dev_err)
        return na_fail(PRJ_ERR_TIMEOUT, "a bounded device-side wait of the z solve gave up (code %d); P is not solved",
                       dev_err);
    return PRJ_OK;
}

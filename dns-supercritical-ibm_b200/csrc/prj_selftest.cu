// prj_selftest.cu -- diagnostic of the bounded device-side waits.
//
// The pipelined kernels (bulk copies completing on mbarriers) never spin without
// a limit: after a clock budget a wait gives up, the kernel raises an error word
// and returns, and the host reports PRJ_ERR_TIMEOUT with the context intact.
// prj_selftest_wait_timeout exercises that path on purpose without any fault: one
// thread waits, with a short budget, on an mbarrier that nothing arrives on.
#include "../../include/projection.h"
#include "prj_internal.h"
#include "div_rn.cuh"
#include "tma_util.cuh"

namespace prj {
namespace {

__global__ void k_wait_selftest(long long budget, int* err) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);  // expects one arrival that never comes
        mbar_fence_init();
    }
    __syncthreads();
    const bool ok = mbar_wait_bounded(&bar, 0, budget);
    if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicExch(err, 3);
}

// splitmix64: a reproducible stream of 64-bit words per index
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// a double with a random sign and mantissa and an exponent in [-span, span] about 1
// (span <= 1022: normal numbers); every eighth value has an all-ones or all-zeros
// mantissa (the rounding edges)
__device__ __forceinline__ double random_double(unsigned long long w, unsigned long long w2, int span) {
    unsigned long long mant = w & 0xfffffffffffffull;
    const int sel = (int)(w2 & 7);
    if (sel == 0) mant = 0xfffffffffffffull;
    if (sel == 1) mant = 0;
    const int ex = 1023 + (int)((w2 >> 8) % (unsigned long long)(2 * span + 1)) - span;
    const unsigned long long bits = ((w >> 63) << 63) | ((unsigned long long)ex << 52) | mant;
    return __longlong_as_double((long long)bits);
}

// a double with a random sign and mantissa and any exponent field 0 .. 2047 (zeros,
// subnormals, normals across the whole range, infinities and NaNs)
__device__ __forceinline__ double any_double(unsigned long long w, unsigned long long w2) {
    unsigned long long mant = w & 0xfffffffffffffull;
    const int sel = (int)(w2 & 7);
    if (sel == 0) mant = 0xfffffffffffffull;
    if (sel == 1) mant = 0;
    const unsigned long long ex = (w2 >> 8) % 2048ull;
    return __longlong_as_double((long long)(((w >> 63) << 63) | (ex << 52) | mant));
}

// a divisor anywhere in the pivot range of div_by_recip, |D| in [2^-40, 2^1000]: exponent
// uniform in [-40, 999], one value in 32 exactly at a bound
__device__ __forceinline__ double pivot_range_double(unsigned long long w, unsigned long long w2) {
    const int sel = (int)((w2 >> 50) & 31);
    const double sgn = (w >> 63) ? -1.0 : 1.0;
    if (sel == 0) return sgn * kDivRecipMinD;
    if (sel == 1) return sgn * kDivRecipMaxD;
    return ldexp(random_double(w, w2, 0), -40 + (int)((w2 >> 8) % 1040ull));
}

// pairs of three kinds by index: u within 2^+-200 and D within 2^+-40 of 1 (the spectra
// and pivots of a solve); u anywhere in the double range (zeros, subnormals, infinities,
// NaNs) with D anywhere in the pivot range; and quotients near the bounds 2^-900 and
// 2^1000 of the fast path's window
__global__ void k_div_selftest(long long n, unsigned long long seed, unsigned long long* bad, double* first) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long k = seed * 0x100000000ull + (unsigned long long)i * 4;
        const unsigned long long wu = mix64(k), wu2 = mix64(k + 1), wd = mix64(k + 2), wd2 = mix64(k + 3);
        double u, D;
        switch (i % 4) {
        case 0:
        case 1:
            u = random_double(wu, wu2, 200);
            D = random_double(wd, wd2, 40);
            break;
        case 2:
            u = any_double(wu, wu2);
            D = pivot_range_double(wd, wd2);
            break;
        default: {
            // u / D within 2^40 of 2^-900 or of 2^1000 (ldexp rounds to subnormals, zero or
            // infinity past the double range)
            D = pivot_range_double(wd, wd2);
            int eD = 0;
            frexp(D, &eD);
            const int eq = ((wu2 >> 40) & 1 ? 1000 : -900) + (int)((wu2 >> 41) % 81ull) - 40;
            u = ldexp(random_double(wu, wu2, 0), eq + eD - 1);
            break;
        }
        }
        if (((wu2 >> 20) & 31) == 0) u = (wu >> 63) ? -0.0 : 0.0;  // signed zero numerators
        const double want = __ddiv_rn(u, D);
        const double got = div_by_recip(u, D, __drcp_rn(D));
        if (__double_as_longlong(want) != __double_as_longlong(got)) {
            if (atomicAdd(bad, 1ull) == 0) {
                first[0] = u;
                first[1] = D;
            }
        }
    }
}

}  // namespace
}  // namespace prj

extern "C" int prj_selftest_division(int device, long long n, unsigned long long seed, long long* mismatches,
                                     double* first_u, double* first_d) {
    if (n < 1 || !mismatches) return prj::record_error(PRJ_ERR_ARG, "need n >= 1 and a result pointer");
    int prev = 0;
    cudaGetDevice(&prev);
    cudaError_t e = cudaSetDevice(device);
    unsigned long long* d_bad = nullptr;
    double* d_first = nullptr;
    unsigned long long h_bad = 0;
    double h_first[2] = {0.0, 0.0};
    if (e == cudaSuccess) e = cudaMalloc((void**)&d_bad, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc((void**)&d_first, 2 * sizeof(double));
    if (e == cudaSuccess) e = cudaMemset(d_bad, 0, sizeof(unsigned long long));
    if (e == cudaSuccess) {
        prj::k_div_selftest<<<148 * 8, 256>>>(n, seed, d_bad, d_first);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(&h_bad, d_bad, sizeof(h_bad), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(h_first, d_first, sizeof(h_first), cudaMemcpyDeviceToHost);
    if (d_bad) cudaFree(d_bad);
    if (d_first) cudaFree(d_first);
    cudaSetDevice(prev);
    if (e != cudaSuccess) return prj::record_error(PRJ_ERR_CUDA, cudaGetErrorString(e));
    *mismatches = (long long)h_bad;
    if (first_u) *first_u = h_bad ? h_first[0] : 0.0;
    if (first_d) *first_d = h_bad ? h_first[1] : 0.0;
    return PRJ_OK;
}

extern "C" int prj_selftest_wait_timeout(int device, long long budget_cycles) {
    if (budget_cycles < 1 || budget_cycles > prj::kWaitBudgetCycles)
        return prj::record_error(PRJ_ERR_ARG, "budget_cycles must be in [1, 4e9]");
    int prev = 0;
    cudaGetDevice(&prev);
    cudaError_t e = cudaSetDevice(device);
    int* d_err = nullptr;
    int h_err = 0;
    if (e == cudaSuccess) e = cudaMalloc((void**)&d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(d_err, 0, sizeof(int));
    if (e == cudaSuccess) {
        prj::k_wait_selftest<<<1, 32>>>(budget_cycles, d_err);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (d_err) cudaFree(d_err);
    cudaSetDevice(prev);
    if (e != cudaSuccess) return prj::record_error(PRJ_ERR_CUDA, cudaGetErrorString(e));
    if (h_err) return prj::record_error(PRJ_ERR_TIMEOUT, "bounded device wait gave up (as intended by the self-test)");
    return PRJ_OK;
}

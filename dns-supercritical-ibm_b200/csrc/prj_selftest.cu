// prj_selftest.cu -- diagnostic of the bounded device-side waits.
//
// The pipelined kernels (bulk copies completing on mbarriers) never spin without
// a limit: after a clock budget a wait gives up, the kernel raises an error word
// and returns, and the host reports PRJ_ERR_TIMEOUT with the context intact.
// prj_selftest_wait_timeout exercises that path on purpose without any fault: one
// thread waits, with a short budget, on an mbarrier that nothing arrives on.
#include "../../include/projection.h"
#include "prj_internal.h"
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

}  // namespace
}  // namespace prj

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

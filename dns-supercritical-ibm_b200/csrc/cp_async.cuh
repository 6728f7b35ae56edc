// cp_async.cuh -- per-thread asynchronous global -> shared copies (cp.async, 8 or 16
// bytes, grouped by commit_group / wait_group).  A copy completes on its own, so a
// wait on this thread's groups cannot hang.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace prj {

__device__ __forceinline__ void cp_async(void* dst, const void* src, int bytes) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    if (bytes == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// no action (the default hook of the tiles that can stage their next input)
struct NoHook {
    __device__ __forceinline__ void operator()() const {}
};

}  // namespace prj

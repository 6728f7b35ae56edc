// tma_util.cuh -- bulk (TMA) copies and mbarriers for sm_100a, inline PTX.
//
// Only non-multicast, CTA-local forms are used: cp.async.bulk and
// cp.async.bulk.tensor from global to this CTA's shared memory with mbarrier
// completion.  Every wait is bounded by
// a clock budget; a caller that gives up reports an error instead of hanging.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace prj {

// ~2 s at 1.9 GHz: far above any legitimate wait of these kernels
constexpr long long kWaitBudgetCycles = 4000000000LL;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// one arrival that also announces `bytes` of incoming transactions
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// the first 128-byte boundary at or after p (a shared-memory address)
__device__ __forceinline__ unsigned char* align128(unsigned char* p) {
    return p + ((128u - (smem_u32(p) & 127u)) & 127u);
}

// Wait for completion of the phase with parity `phase`; false after `budget` cycles.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase,
                                                  long long budget = kWaitBudgetCycles) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, phase)) {
        if (clock64() - t0 > budget) return false;
    }
    return true;
}

// global -> shared bulk copy; dst/src 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// global -> shared copy of one box of a 4-D tensor map (cp.async.bulk.tensor, no
// multicast): box coordinates c0..c3 (c0 in elements, a multiple of 16 bytes), completion
// counted on `bar`; `tmap` is the generic address of the CUtensorMap in param, const or
// global memory; `dst` 128-byte aligned
__device__ __forceinline__ void tma_load_4d(void* dst, const void* tmap, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

// global -> shared copy of one box of a 3-D tensor map (as tma_load_4d)
__device__ __forceinline__ void tma_load_3d(void* dst, const void* tmap, int c0, int c1, int c2, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

// Host: encode a tiled tensor map of FP64 elements (the driver's cuTensorMapEncodeTiled,
// looked up once through the runtime): rank dims (innermost first), rank-1 byte strides,
// the box; no interleave, swizzle or fill value (out-of-bounds elements read as zero).
// False if the driver refuses it.
bool tmap_encode_f64(void* tmap128, const void* base, int rank, const uint64_t* dims, const uint64_t* strides,
                     const uint32_t* box);

// order this thread's generic-proxy accesses before later async-proxy (bulk copy) accesses
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

}  // namespace prj

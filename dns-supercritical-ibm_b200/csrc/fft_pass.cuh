// fft_pass.cuh -- compile-time pass plans of the in-place DIF/DIT transforms.
//
// A length n = R_0 R_1 ... R_{P-1} is transformed in P passes with the stage
// semantics of fft_dif.cuh (span L_s = n / (R_0 ... R_{s-1}); a butterfly of pass s
// takes the R_s elements j + q L_s/R_s of one span block).  With the radices known
// at compile time:
//   * the first pass of a DIF transform reads its elements straight from global
//     memory (they are n/R_0 apart, so a warp's loads are coalesced) and the last
//     pass writes its R_{P-1} outputs, contiguous in slot order, straight to global
//     memory; only the passes in between go through shared memory;
//   * the DIT inverse runs the passes in reverse: the first reads contiguous slots
//     from global memory, the last writes natural order to global memory;
//   * index arithmetic divides by constants and the slot of frequency k
//     (digit reversal) is computed, not looked up.
// Twiddles are the plan's tables (fft_host.h dif_fill, same radices), so the
// result equals the runtime-radix kernels up to rounding order.
#pragma once
#include "fft_dif.cuh"

namespace prj {

template <int DIR, int R, typename V>
__device__ __forceinline__ void dft_r(V* a) {
    if constexpr (R == 2) dft2<DIR>(a[0], a[1]);
    else if constexpr (R == 3) dft3<DIR>(a[0], a[1], a[2]);
    else if constexpr (R == 4) dft4<DIR>(a[0], a[1], a[2], a[3]);
    else if constexpr (R == 5) dft5<DIR>(a[0], a[1], a[2], a[3], a[4]);
    else if constexpr (R == 6) dft6<DIR>(a);
    else {
        static_assert(R == 8, "radix 2, 3, 4, 5, 6 or 8");
        dft8<DIR>(a);
    }
}

template <int... Rs>
struct PassList {
    static constexpr int P = sizeof...(Rs);
    static constexpr int n = (Rs * ...);
    __host__ __device__ static constexpr int radix(int s) {
        constexpr int r[] = {Rs...};
        return r[s];
    }
    __host__ __device__ static constexpr int span(int s) {
        int L = n;
        for (int t = 0; t < s; t++) L /= radix(t);
        return L;
    }
    // offset of pass s's twiddles in the plan's table (fft_host.h dif_plan)
    __host__ __device__ static constexpr int twoff(int s) {
        int c = 0;
        for (int t = 0; t < s; t++) c += (span(t) / radix(t)) * (radix(t) - 1);
        return c;
    }
    // slot of index k after the DIF transform: digits of k (radix R_0 least
    // significant) weighted by span_s / R_s
    __host__ __device__ static constexpr int slot(int k) {
        int p = 0;
        for (int s = 0; s < P; s++) {
            const int R = radix(s);
            const int q = k % R;
            k /= R;
            p += q * (span(s) / R);
        }
        return p;
    }
};

// slot(k) for a run-time k with compile-time divisors
template <class PL, int S = 0>
__device__ __forceinline__ int pass_slot(int k) {
    if constexpr (S == PL::P) {
        return 0;
    } else {
        constexpr int R = PL::radix(S);
        constexpr int w = PL::span(S) / R;
        return (k % R) * w + pass_slot<PL, S + 1>(k / R);
    }
}

// a[q] *= w1^q with w1 = exp(-+2 pi i j / L) the first row of the stage table
// (w[j]); the powers come from a product tree of depth <= 3 (about 3 ulp), so a
// butterfly loads one twiddle instead of R-1 (the loads were the larger share of
// the L1 traffic of these kernels)
template <int DIR, int R, int MM, typename V>
__device__ __forceinline__ void apply_twiddles(V* a, const V* __restrict__ w, int j) {
    V p[R];
    p[1] = w[j];
    if constexpr (R > 2) p[2] = cmul(p[1], p[1]);
    if constexpr (R > 3) p[3] = cmul(p[1], p[2]);
    if constexpr (R > 4) p[4] = cmul(p[2], p[2]);
    if constexpr (R > 5) p[5] = cmul(p[2], p[3]);
    if constexpr (R > 6) p[6] = cmul(p[3], p[3]);
    if constexpr (R > 7) p[7] = cmul(p[3], p[4]);
#pragma unroll
    for (int q = 1; q < R; q++) a[q] = twiddle<DIR>(a[q], p[q]);
}

// One pass s of nrows rows held in shared memory (row stride rs, padded slots):
// DIT = false: DFT then twiddles; DIT = true: twiddles then DFT.
template <int DIR, bool DIT, class PL, int S, typename V>
__device__ __forceinline__ void pass_shared(V* buf, int nrows, int rs, const V* __restrict__ tw) {
    constexpr int R = PL::radix(S), L = PL::span(S), mm = L / R, NB = PL::n / R;
    const V* tws = tw + PL::twoff(S);
    for (int idx = threadIdx.x; idx < nrows * NB; idx += blockDim.x) {
        const int row = idx / NB, bi = idx - row * NB;
        const int blk = bi / mm, j = bi - blk * mm;
        const int g0 = row * rs + blk * L + j;
        V a[R];
#pragma unroll
        for (int q = 0; q < R; q++) a[q] = buf[sidx<true>(g0 + q * mm)];
        if (DIT && mm > 1 && j) apply_twiddles<DIR, R, mm>(a, tws, j);
        dft_r<DIR, R>(a);
        if (!DIT && mm > 1 && j) apply_twiddles<DIR, R, mm>(a, tws, j);
#pragma unroll
        for (int q = 0; q < R; q++) buf[sidx<true>(g0 + q * mm)] = a[q];
    }
}

// Passes S .. E-1 in shared memory, a barrier after each (DIF order).
template <int DIR, class PL, int S, int E, typename V>
__device__ __forceinline__ void dif_passes_shared(V* buf, int nrows, int rs, const V* __restrict__ tw) {
    if constexpr (S < E) {
        pass_shared<DIR, false, PL, S>(buf, nrows, rs, tw);
        __syncthreads();
        dif_passes_shared<DIR, PL, S + 1, E>(buf, nrows, rs, tw);
    }
}

// Passes S down to E+1 in shared memory, a barrier after each (DIT order).
template <int DIR, class PL, int S, int E, typename V>
__device__ __forceinline__ void dit_passes_shared(V* buf, int nrows, int rs, const V* __restrict__ tw) {
    if constexpr (S > E) {
        pass_shared<DIR, true, PL, S>(buf, nrows, rs, tw);
        __syncthreads();
        dit_passes_shared<DIR, PL, S - 1, E>(buf, nrows, rs, tw);
    }
}

// First DIF pass from a source functor: ld(row, e) -> V for natural index e.
// Results go to shared memory.  No barrier.
template <int DIR, class PL, typename V, class Ld>
__device__ __forceinline__ void dif_first_pass(V* buf, int nrows, int rs, const V* __restrict__ tw, Ld ld) {
    constexpr int R = PL::radix(0), mm = PL::n / R;
    for (int idx = threadIdx.x; idx < nrows * mm; idx += blockDim.x) {
        const int row = idx / mm, j = idx - row * mm;
        V a[R];
#pragma unroll
        for (int q = 0; q < R; q++) a[q] = ld(row, j + q * mm);
        dft_r<DIR, R>(a);
        if (mm > 1 && j) apply_twiddles<DIR, R, mm>(a, tw, j);
#pragma unroll
        for (int q = 0; q < R; q++) buf[sidx<true>(row * rs + j + q * mm)] = a[q];
    }
}

// Last DIF pass (span R, no twiddles) from shared memory to a sink functor:
// st(row, slot, value) for the R contiguous slots of each block.  No barrier.
template <int DIR, class PL, typename V, class St>
__device__ __forceinline__ void dif_last_pass(const V* buf, int nrows, int rs, St st) {
    constexpr int S = PL::P - 1, R = PL::radix(S), NB = PL::n / R;
    for (int idx = threadIdx.x; idx < nrows * NB; idx += blockDim.x) {
        const int row = idx / NB, blk = idx - row * NB;
        const int g0 = row * rs + blk * R;
        V a[R];
#pragma unroll
        for (int q = 0; q < R; q++) a[q] = buf[sidx<true>(g0 + q)];
        dft_r<DIR, R>(a);
#pragma unroll
        for (int q = 0; q < R; q++) st(row, blk * R + q, a[q]);
    }
}

// First DIT pass (pass P-1, span R, no twiddles) from a source functor reading
// slot order: ld(row, slot).  Results to shared memory.  No barrier.
template <int DIR, class PL, typename V, class Ld>
__device__ __forceinline__ void dit_first_pass(V* buf, int nrows, int rs, Ld ld) {
    constexpr int S = PL::P - 1, R = PL::radix(S), NB = PL::n / R;
    for (int idx = threadIdx.x; idx < nrows * NB; idx += blockDim.x) {
        const int row = idx / NB, blk = idx - row * NB;
        V a[R];
#pragma unroll
        for (int q = 0; q < R; q++) a[q] = ld(row, blk * R + q);
        dft_r<DIR, R>(a);
#pragma unroll
        for (int q = 0; q < R; q++) buf[sidx<true>(row * rs + blk * R + q)] = a[q];
    }
}

// Last DIT pass (pass 0, span n) from shared memory to a sink functor in natural
// order: st(row, e, value).  No barrier.
template <int DIR, class PL, typename V, class St>
__device__ __forceinline__ void dit_last_pass(const V* buf, int nrows, int rs, const V* __restrict__ tw, St st) {
    constexpr int R = PL::radix(0), mm = PL::n / R;
    for (int idx = threadIdx.x; idx < nrows * mm; idx += blockDim.x) {
        const int row = idx / mm, j = idx - row * mm;
        V a[R];
#pragma unroll
        for (int q = 0; q < R; q++) a[q] = buf[sidx<true>(row * rs + j + q * mm)];
        if (mm > 1 && j) apply_twiddles<DIR, R, mm>(a, tw, j);
        dft_r<DIR, R>(a);
#pragma unroll
        for (int q = 0; q < R; q++) st(row, j + q * mm, a[q]);
    }
}

// threads per CTA and minimum resident CTAs per SM of the pass-plan kernels (6: 85
// registers, and 6 CTAs of ~28 KB shared memory per SM; measured best of 4-8)
constexpr int kPassThreads = 128;
#ifndef PRJ_PASS_MINB
#define PRJ_PASS_MINB 6
#endif

// true when a runtime plan has exactly the radices of PL
template <class PL>
inline bool same_radices(const DifDev& f) {
    if (f.nst != PL::P || f.n != PL::n) return false;
    for (int s = 0; s < PL::P; s++)
        if (f.radix[s] != PL::radix(s)) return false;
    return true;
}

// Lengths with a compile-time pass plan: X(n, radices...).  The host plans these
// lengths with the same radices (fft_host.h), so twiddle tables and slot orders
// agree with the runtime-radix kernels.  The radix order is the one whose passes
// address the padded shared-memory rows (slot g + g/8) without bank conflicts, or
// with the fewest (counted for 16-byte accesses, eight lanes per wavefront): a
// pass of span L and radix R strides its butterflies by L/R elements, and with the
// odd radices early every later stride is a multiple of 8 or spread by the padding.
#define PRJ_PASS_PLANS(X)       \
    X(16, 4, 4)                 \
    X(24, 6, 4)                 \
    X(32, 8, 4)                 \
    X(48, 6, 8)                 \
    X(64, 8, 8)                 \
    X(96, 2, 6, 8)              \
    X(128, 4, 4, 8)             \
    X(192, 3, 8, 8)             \
    X(256, 8, 4, 8)             \
    X(384, 6, 8, 8)             \
    X(512, 8, 8, 8)             \
    X(768, 8, 6, 2, 8)          \
    X(1024, 4, 8, 4, 8)         \
    X(1536, 4, 8, 6, 8)

// Other radix orders of some of those lengths, compiled as well, that a plan's tuning
// (x_order / z_order) can select: order k >= 1 of length n is the k-th entry of n below.
// The autotuner times them against the default orders above.  Different orders round
// differently (every one within the parity bounds); a given order gives the same bits in
// every kernel family.
#define PRJ_PASS_ALTS(X)        \
    X(64, 4, 4, 4)              \
    X(96, 8, 6, 2)              \
    X(128, 8, 8, 2)             \
    X(192, 6, 4, 8)             \
    X(256, 4, 8, 8)             \
    X(256, 8, 8, 4)             \
    X(384, 8, 6, 8)             \
    X(384, 8, 8, 6)

// every compiled pass plan: the default orders, then the other orders
#define PRJ_PASS_ALL(X) PRJ_PASS_PLANS(X) PRJ_PASS_ALTS(X)

// Row stride (in elements) of the x kernels' shared-memory rows of m complex values:
// a multiple of 8, so every row starts on a padding boundary and the passes of
// consecutive rows see the same bank pattern; the +8 offsets consecutive rows by
// one bank group for the row-fastest split and load phases.
__host__ __device__ constexpr int pass_row_stride(int m) { return m + 8; }

}  // namespace prj

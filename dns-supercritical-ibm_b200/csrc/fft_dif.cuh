// fft_dif.cuh -- in-place mixed-radix decimation-in-frequency FFT for one CTA.
//
// Rows of length n live in shared memory (row stride rs).  Stage s has span
// L_s = n / (R_0 ... R_{s-1}); each butterfly takes the R_s elements
// j + r L_s/R_s of one span block, runs an R_s-point DFT and scales output q by
// exp(-+2 pi i q j / L_s), writing back to the same R_s slots.  Butterflies of a
// stage touch disjoint slots, so a stage needs one barrier and no second
// buffer.  The result is in digit-reversed order: frequency (or, for the
// inverse, time) index k sits at slot pos[k]; consumers read through `pos`.
//
// Twiddles per stage: tw[(q - 1) L/R + j] = exp(-2 pi i q j / L), j < L/R,
// 1 <= q < R.  The inverse transform uses the conjugates.  Radices 2, 3, 4, 5
// 6 and 8 only; other lengths use the out-of-place path of fft_device.cuh.
#pragma once
#include "fft_device.cuh"

namespace prj {

// Division by a run-time invariant d by multiply-high and shift (Granlund and
// Montgomery, "Division by invariant integers using multiplication", 1994):
// q = umulhi(x, m) >> s with s = ceil(log2 d) - 1, m = ceil(2^(31 + ceil(log2 d)) / d).
// Exact for 0 <= x < 2^22 and 1 <= d < 8200 (checked exhaustively on the host).
struct FastDiv {
    unsigned d, m, s;
};

__host__ __device__ inline FastDiv make_fastdiv(unsigned d) {
    FastDiv f{d, 0u, 0u};
    if (d > 1) {
        unsigned l = 0;
        while ((1u << l) < d) l++;
        const unsigned long long p = 31ull + l;
        f.m = (unsigned)(((1ull << p) + d - 1) / d);
        f.s = l - 1;
    }
    return f;
}

__device__ __forceinline__ int fdiv(int x, const FastDiv& f) {
    return f.d == 1 ? x : (int)(__umulhi((unsigned)x, f.m) >> f.s);
}

struct DifDev {
    int n;
    int nst;
    int radix[kMaxStages];
    int span[kMaxStages];
    int twoff[kMaxStages];
    FastDiv nbdiv[kMaxStages];  // n / radix
    FastDiv mmdiv[kMaxStages];  // span / radix
};

template <int DIR, typename V>
__device__ __forceinline__ V twiddle(V a, V w) {
    return DIR < 0 ? cmul(a, w) : cmulc(a, w);
}

// Shared-memory slot of element g.  PAD inserts one empty 16-byte slot after
// every 8 elements, so strides that are multiples of 8 elements (the late
// stages and the digit-reversal gathers) spread over all bank groups.
template <bool PAD>
__device__ __forceinline__ int sidx(int g) {
    return PAD ? g + (g >> 3) : g;
}

// elements per row buffer of n slots with optional padding
__host__ __device__ inline int padded_len(int n, bool pad) { return pad ? n + (n >> 3) + 1 : n; }

// One butterfly of radix R on elements g0 + r mm (r < R) of buf; w = the stage's twiddles.
// DIT = false: DFT, then twiddles (decimation in frequency);
// DIT = true: twiddles, then DFT (its transpose).
template <int DIR, bool DIT, bool PAD, int R, typename V>
__device__ __forceinline__ void bfly_r(V* __restrict__ buf, int g0, int mm, int j, const V* __restrict__ w) {
    V a[R];
#pragma unroll
    for (int r = 0; r < R; r++) a[r] = buf[sidx<PAD>(g0 + r * mm)];
    if (DIT && j) {
#pragma unroll
        for (int q = 1; q < R; q++) a[q] = twiddle<DIR>(a[q], w[(q - 1) * mm + j]);
    }
    if (R == 2) dft2<DIR>(a[0], a[1]);
    else if (R == 3) dft3<DIR>(a[0], a[1], a[2]);
    else if (R == 4) dft4<DIR>(a[0], a[1], a[2], a[3]);
    else if (R == 5) dft5<DIR>(a[0], a[1], a[2], a[3], a[4]);
    else if (R == 6) dft6<DIR>(a);
    else dft8<DIR>(a);
    if (!DIT && j) {
#pragma unroll
        for (int q = 1; q < R; q++) a[q] = twiddle<DIR>(a[q], w[(q - 1) * mm + j]);
    }
#pragma unroll
    for (int r = 0; r < R; r++) buf[sidx<PAD>(g0 + r * mm)] = a[r];
}

template <int DIR, bool DIT, bool PAD, typename V>
__device__ __forceinline__ void bfly(V* __restrict__ buf, int g0, int mm, int R, int j, const V* __restrict__ w) {
    switch (R) {
    case 2: bfly_r<DIR, DIT, PAD, 2>(buf, g0, mm, j, w); break;
    case 3: bfly_r<DIR, DIT, PAD, 3>(buf, g0, mm, j, w); break;
    case 4: bfly_r<DIR, DIT, PAD, 4>(buf, g0, mm, j, w); break;
    case 5: bfly_r<DIR, DIT, PAD, 5>(buf, g0, mm, j, w); break;
    case 6: bfly_r<DIR, DIT, PAD, 6>(buf, g0, mm, j, w); break;
    case 8: bfly_r<DIR, DIT, PAD, 8>(buf, g0, mm, j, w); break;
    default:
        // other radices are planned on the out-of-place Stockham path (fft_device.cuh);
        // the host never builds a DifDev containing them (dif_supported)
        break;
    }
}

// In-place transform of `nrows` rows of n elements (row r starts at element
// r * rs; with PAD, element g of the buffer lives at slot g + g/8).  DIT = false:
// decimation in frequency, natural order in, digit-reversed out.  DIT = true:
// decimation in time with the same plan, digit-reversed in, natural out; with
// DIR = +1 it inverts the DIF transform up to the factor n.  Starts and ends
// with the CTA synchronised.
template <int DIR, bool DIT, bool PAD, typename V>
__device__ void inplace_rows(V* buf, int nrows, int rs, const DifDev& f, const V* __restrict__ tw) {
    const int nthr = blockDim.x, tid = threadIdx.x;
    const int n = f.n;
    for (int t = 0; t < f.nst; t++) {
        const int s = DIT ? f.nst - 1 - t : t;
        const int R = f.radix[s], L = f.span[s];
        const int mm = L / R;
        const int nb = n / R;
        const V* tws = tw + f.twoff[s];
        const FastDiv dnb = f.nbdiv[s], dmm = f.mmdiv[s];
        for (int idx = tid; idx < nb * nrows; idx += nthr) {
            const int row = fdiv(idx, dnb);
            const int bi = idx - row * nb;
            const int b = fdiv(bi, dmm);
            const int j = bi - b * mm;
            bfly<DIR, DIT, PAD>(buf, row * rs + b * L + j, mm, R, j, tws);
        }
        __syncthreads();
    }
}

template <int DIR, typename V>
__device__ void dif_rows(V* buf, int nrows, int rs, const DifDev& f, const V* __restrict__ tw) {
    inplace_rows<DIR, false, false>(buf, nrows, rs, f, tw);
}

template <int DIR, typename V>
__device__ void dit_rows(V* buf, int nrows, int rs, const DifDev& f, const V* __restrict__ tw) {
    inplace_rows<DIR, true, false>(buf, nrows, rs, f, tw);
}

}  // namespace prj

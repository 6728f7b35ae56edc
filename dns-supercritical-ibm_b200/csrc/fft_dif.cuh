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
// Twiddles per stage: tw[j (R-1) + q - 1] = exp(-2 pi i q j / L), j < L/R,
// 1 <= q < R.  The inverse transform uses the conjugates.  Radices 2, 3, 4, 5
// and 8 only; other lengths use the out-of-place path of fft_device.cuh.
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

template <int DIR, typename V>
__device__ __forceinline__ void dif_bfly(V* __restrict__ p, int mm, int R, int j, const V* __restrict__ w) {
    switch (R) {
    case 2: {
        V a0 = p[0], a1 = p[mm];
        dft2<DIR>(a0, a1);
        if (j) a1 = twiddle<DIR>(a1, w[0]);
        p[0] = a0; p[mm] = a1;
    } break;
    case 3: {
        V a0 = p[0], a1 = p[mm], a2 = p[2 * mm];
        dft3<DIR>(a0, a1, a2);
        if (j) { a1 = twiddle<DIR>(a1, w[0]); a2 = twiddle<DIR>(a2, w[1]); }
        p[0] = a0; p[mm] = a1; p[2 * mm] = a2;
    } break;
    case 4: {
        V a0 = p[0], a1 = p[mm], a2 = p[2 * mm], a3 = p[3 * mm];
        dft4<DIR>(a0, a1, a2, a3);
        if (j) { a1 = twiddle<DIR>(a1, w[0]); a2 = twiddle<DIR>(a2, w[1]); a3 = twiddle<DIR>(a3, w[2]); }
        p[0] = a0; p[mm] = a1; p[2 * mm] = a2; p[3 * mm] = a3;
    } break;
    case 5: {
        V a[5];
#pragma unroll
        for (int r = 0; r < 5; r++) a[r] = p[r * mm];
        dft5<DIR>(a[0], a[1], a[2], a[3], a[4]);
        if (j) {
#pragma unroll
            for (int q = 1; q < 5; q++) a[q] = twiddle<DIR>(a[q], w[q - 1]);
        }
#pragma unroll
        for (int r = 0; r < 5; r++) p[r * mm] = a[r];
    } break;
    case 8: {
        V a[8];
#pragma unroll
        for (int r = 0; r < 8; r++) a[r] = p[r * mm];
        dft8<DIR>(a);
        if (j) {
#pragma unroll
            for (int q = 1; q < 8; q++) a[q] = twiddle<DIR>(a[q], w[q - 1]);
        }
#pragma unroll
        for (int r = 0; r < 8; r++) p[r * mm] = a[r];
    } break;
    default:
        // other radices are planned on the out-of-place Stockham path (fft_device.cuh);
        // the host never builds a DifDev containing them (dif_supported)
        break;
    }
}

// In-place transform of `nrows` rows (stride rs).  Starts and ends with the
// CTA synchronised.
template <int DIR, typename V>
__device__ void dif_rows(V* buf, int nrows, int rs, const DifDev& f, const V* __restrict__ tw) {
    const int nthr = blockDim.x, tid = threadIdx.x;
    const int n = f.n;
    for (int s = 0; s < f.nst; s++) {
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
            dif_bfly<DIR>(buf + (size_t)row * rs + b * L + j, mm, R, j, tws + j * (R - 1));
        }
        __syncthreads();
    }
}

// One DIT butterfly: the transpose of dif_bfly (twiddles first, then the DFT).
template <int DIR, typename V>
__device__ __forceinline__ void dit_bfly(V* __restrict__ p, int mm, int R, int j, const V* __restrict__ w) {
    switch (R) {
    case 2: {
        V a0 = p[0], a1 = p[mm];
        if (j) a1 = twiddle<DIR>(a1, w[0]);
        dft2<DIR>(a0, a1);
        p[0] = a0; p[mm] = a1;
    } break;
    case 3: {
        V a0 = p[0], a1 = p[mm], a2 = p[2 * mm];
        if (j) { a1 = twiddle<DIR>(a1, w[0]); a2 = twiddle<DIR>(a2, w[1]); }
        dft3<DIR>(a0, a1, a2);
        p[0] = a0; p[mm] = a1; p[2 * mm] = a2;
    } break;
    case 4: {
        V a0 = p[0], a1 = p[mm], a2 = p[2 * mm], a3 = p[3 * mm];
        if (j) { a1 = twiddle<DIR>(a1, w[0]); a2 = twiddle<DIR>(a2, w[1]); a3 = twiddle<DIR>(a3, w[2]); }
        dft4<DIR>(a0, a1, a2, a3);
        p[0] = a0; p[mm] = a1; p[2 * mm] = a2; p[3 * mm] = a3;
    } break;
    case 5: {
        V a[5];
#pragma unroll
        for (int r = 0; r < 5; r++) a[r] = p[r * mm];
        if (j) {
#pragma unroll
            for (int q = 1; q < 5; q++) a[q] = twiddle<DIR>(a[q], w[q - 1]);
        }
        dft5<DIR>(a[0], a[1], a[2], a[3], a[4]);
#pragma unroll
        for (int r = 0; r < 5; r++) p[r * mm] = a[r];
    } break;
    case 8: {
        V a[8];
#pragma unroll
        for (int r = 0; r < 8; r++) a[r] = p[r * mm];
        if (j) {
#pragma unroll
            for (int q = 1; q < 8; q++) a[q] = twiddle<DIR>(a[q], w[q - 1]);
        }
        dft8<DIR>(a);
#pragma unroll
        for (int r = 0; r < 8; r++) p[r * mm] = a[r];
    } break;
    default:
        break;
    }
}

// In-place decimation-in-time transform with the same plan as dif_rows: input in
// digit-reversed order (index k at slot pos[k]), output in natural order.  With
// DIR = +1 it inverts dif_rows<-1> up to the factor n (unnormalised inverse).
template <int DIR, typename V>
__device__ void dit_rows(V* buf, int nrows, int rs, const DifDev& f, const V* __restrict__ tw) {
    const int nthr = blockDim.x, tid = threadIdx.x;
    const int n = f.n;
    for (int s = f.nst - 1; s >= 0; s--) {
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
            dit_bfly<DIR>(buf + (size_t)row * rs + b * L + j, mm, R, j, tws + j * (R - 1));
        }
        __syncthreads();
    }
}

}  // namespace prj

// fft_device.cuh -- shared-memory mixed-radix Stockham FFT for one CTA.
//
// The CTA holds `nrows` complex rows of length n in shared memory (row stride
// `rs` elements) and transforms all of them together.  Each stage of radix R
// reads R inputs strided by n/R, applies the stage twiddles, runs an R-point
// DFT in registers and writes R outputs in autosorted order, so the last stage
// leaves the spectrum in natural order (no bit reversal).  Stages ping-pong
// between two buffers; the function returns the buffer holding the result.
//
// Twiddles are precomputed on the host in extended precision and stored per
// stage as tw[k*(R-1) + r-1] = exp(-2 pi i r k / (p R)), k < p, 1 <= r < R,
// followed (for radices without a hard-coded kernel) by the R roots
// exp(-2 pi i m / R).  The inverse transform uses the conjugates.
#pragma once
#include <cuda_runtime.h>

namespace prj {

constexpr int kMaxStages = 24;

struct FftDev {
    int n;                      // complex length
    int nst;                    // number of stages
    int radix[kMaxStages];
    int p[kMaxStages];          // product of the radices of the earlier stages
    int twoff[kMaxStages];      // offset (complex elements) of the stage twiddles
};

template <typename T> struct C2;
template <> struct C2<double> { using t = double2; };
template <> struct C2<float> { using t = float2; };

template <typename V> __device__ __forceinline__ V cmk(decltype(V::x) r, decltype(V::x) i) { V v; v.x = r; v.y = i; return v; }
template <typename V> __device__ __forceinline__ V cadd(V a, V b) { return cmk<V>(a.x + b.x, a.y + b.y); }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { return cmk<V>(a.x - b.x, a.y - b.y); }
template <typename V> __device__ __forceinline__ V cmul(V a, V b) { return cmk<V>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
// a * conj(b)
template <typename V> __device__ __forceinline__ V cmulc(V a, V b) { return cmk<V>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); }
template <typename V> __device__ __forceinline__ V cscale(V a, decltype(V::x) s) { return cmk<V>(a.x * s, a.y * s); }
template <typename V> __device__ __forceinline__ V cconj(V a) { return cmk<V>(a.x, -a.y); }
// multiply by i*DIR  (DIR = -1: -i, DIR = +1: +i)
template <int DIR, typename V> __device__ __forceinline__ V cmuli(V a) {
    return DIR > 0 ? cmk<V>(-a.y, a.x) : cmk<V>(a.y, -a.x);
}

// ---------------------------------------------------------------- DFT kernels
template <int DIR, typename V> __device__ __forceinline__ void dft2(V& a0, V& a1) {
    V t = a0; a0 = cadd(t, a1); a1 = csub(t, a1);
}

template <int DIR, typename V> __device__ __forceinline__ void dft3(V& a0, V& a1, V& a2) {
    using R = decltype(V::x);
    const R c = R(-0.5), s = R(0.86602540378443864676372317075294);
    V t1 = cadd(a1, a2);
    V t2 = csub(a0, cscale(t1, -c));
    V t3 = cmuli<DIR>(cscale(csub(a1, a2), s));
    a0 = cadd(a0, t1);
    a1 = cadd(t2, t3);
    a2 = csub(t2, t3);
}

template <int DIR, typename V> __device__ __forceinline__ void dft4(V& a0, V& a1, V& a2, V& a3) {
    V t0 = cadd(a0, a2), t1 = csub(a0, a2);
    V t2 = cadd(a1, a3), t3 = cmuli<DIR>(csub(a1, a3));
    a0 = cadd(t0, t2); a2 = csub(t0, t2);
    a1 = cadd(t1, t3); a3 = csub(t1, t3);
}

template <int DIR, typename V> __device__ __forceinline__ void dft5(V& a0, V& a1, V& a2, V& a3, V& a4) {
    using R = decltype(V::x);
    const R c1 = R(0.30901699437494742410229341718282), c2 = R(-0.80901699437494742410229341718282);
    const R s1 = R(0.95105651629515357211643933337938), s2 = R(0.58778525229247312916870595463907);
    V p14 = cadd(a1, a4), m14 = csub(a1, a4), p23 = cadd(a2, a3), m23 = csub(a2, a3);
    V b1 = cadd(a0, cadd(cscale(p14, c1), cscale(p23, c2)));
    V b2 = cadd(a0, cadd(cscale(p14, c2), cscale(p23, c1)));
    V q1 = cmuli<DIR>(cadd(cscale(m14, s1), cscale(m23, s2)));
    V q2 = cmuli<DIR>(csub(cscale(m14, s2), cscale(m23, s1)));
    a0 = cadd(a0, cadd(p14, p23));
    a1 = cadd(b1, q1); a4 = csub(b1, q1);
    a2 = cadd(b2, q2); a3 = csub(b2, q2);
}

template <int DIR, typename V> __device__ __forceinline__ void dft8(V* a) {
    using R = decltype(V::x);
    const R h = R(0.70710678118654752440084436210485);
    dft4<DIR>(a[0], a[2], a[4], a[6]);
    dft4<DIR>(a[1], a[3], a[5], a[7]);
    // odd part times w8^k, w8 = exp(DIR 2 pi i / 8)
    V o1 = cmk<V>(h * (a[3].x - DIR * a[3].y), h * (a[3].y + DIR * a[3].x));
    V o2 = cmuli<DIR>(a[5]);
    V o3 = cmk<V>(h * (-a[7].x - DIR * a[7].y), h * (-a[7].y + DIR * a[7].x));
    V e0 = a[0], e1 = a[2], e2 = a[4], e3 = a[6];
    a[0] = cadd(e0, a[1]); a[4] = csub(e0, a[1]);
    a[1] = cadd(e1, o1);   a[5] = csub(e1, o1);
    a[2] = cadd(e2, o2);   a[6] = csub(e2, o2);
    a[3] = cadd(e3, o3);   a[7] = csub(e3, o3);
}

// 6-point DFT by the prime-factor map n = (3 n1 + 2 n2) mod 6, k = (3 k1 + 4 k2) mod 6:
// two 3-point DFTs and three 2-point DFTs, no internal twiddles.
template <int DIR, typename V>
__device__ __forceinline__ void dft6(V* a) {
    V e0 = a[0], e1 = a[2], e2 = a[4];
    V o0 = a[3], o1 = a[5], o2 = a[1];
    dft3<DIR>(e0, e1, e2);
    dft3<DIR>(o0, o1, o2);
    a[0] = cadd(e0, o0); a[3] = csub(e0, o0);
    a[4] = cadd(e1, o1); a[1] = csub(e1, o1);
    a[2] = cadd(e2, o2); a[5] = csub(e2, o2);
}

// ------------------------------------------------------------ one radix stage
// i: butterfly index in [0, n/R); k = i mod p.  Inputs src[i + r n/R];
// outputs dst[(i - k) R + k + r p].
template <int DIR, typename V>
__device__ __forceinline__ void stage_bfly(const V* __restrict__ src, V* __restrict__ dst, int n, int R, int p,
                                           const V* __restrict__ tw, int i) {
    const int k = i % p;
    const int stride = n / R;
    const int obase = (i - k) * R + k;
    const V* w = tw + k * (R - 1);
    switch (R) {
    case 2: {
        V a0 = src[i], a1 = src[i + stride];
        if (k) a1 = DIR < 0 ? cmul(a1, w[0]) : cmulc(a1, w[0]);
        dft2<DIR>(a0, a1);
        dst[obase] = a0; dst[obase + p] = a1;
    } break;
    case 3: {
        V a0 = src[i], a1 = src[i + stride], a2 = src[i + 2 * stride];
        if (k) {
            if (DIR < 0) { a1 = cmul(a1, w[0]); a2 = cmul(a2, w[1]); }
            else { a1 = cmulc(a1, w[0]); a2 = cmulc(a2, w[1]); }
        }
        dft3<DIR>(a0, a1, a2);
        dst[obase] = a0; dst[obase + p] = a1; dst[obase + 2 * p] = a2;
    } break;
    case 4: {
        V a0 = src[i], a1 = src[i + stride], a2 = src[i + 2 * stride], a3 = src[i + 3 * stride];
        if (k) {
            if (DIR < 0) { a1 = cmul(a1, w[0]); a2 = cmul(a2, w[1]); a3 = cmul(a3, w[2]); }
            else { a1 = cmulc(a1, w[0]); a2 = cmulc(a2, w[1]); a3 = cmulc(a3, w[2]); }
        }
        dft4<DIR>(a0, a1, a2, a3);
        dst[obase] = a0; dst[obase + p] = a1; dst[obase + 2 * p] = a2; dst[obase + 3 * p] = a3;
    } break;
    case 5: {
        V a[5];
#pragma unroll
        for (int r = 0; r < 5; r++) a[r] = src[i + r * stride];
        if (k) {
#pragma unroll
            for (int r = 1; r < 5; r++) a[r] = DIR < 0 ? cmul(a[r], w[r - 1]) : cmulc(a[r], w[r - 1]);
        }
        dft5<DIR>(a[0], a[1], a[2], a[3], a[4]);
#pragma unroll
        for (int r = 0; r < 5; r++) dst[obase + r * p] = a[r];
    } break;
    case 8: {
        V a[8];
#pragma unroll
        for (int r = 0; r < 8; r++) a[r] = src[i + r * stride];
        if (k) {
#pragma unroll
            for (int r = 1; r < 8; r++) a[r] = DIR < 0 ? cmul(a[r], w[r - 1]) : cmulc(a[r], w[r - 1]);
        }
        dft8<DIR>(a);
#pragma unroll
        for (int r = 0; r < 8; r++) dst[obase + r * p] = a[r];
    } break;
    default: {
        // any radix: direct R-point DFT with the stage's root table
        const V* roots = tw + p * (R - 1);
        for (int q = 0; q < R; q++) {
            V acc = cmk<V>(0, 0);
            for (int r = 0; r < R; r++) {
                V u = src[i + r * stride];
                if (r && k) u = DIR < 0 ? cmul(u, w[r - 1]) : cmulc(u, w[r - 1]);
                const int e = (r * q) % R;
                acc = cadd(acc, DIR < 0 ? cmul(u, roots[e]) : cmulc(u, roots[e]));
            }
            dst[obase + q * p] = acc;
        }
    } break;
    }
}

// Transform `nrows` rows (row stride rs) held in a; b is scratch of the same
// shape.  Returns the buffer with the result.  Starts and ends with all
// threads of the CTA synchronised.
template <int DIR, typename V>
__device__ V* fft_rows(V* a, V* b, int nrows, int rs, const FftDev& f, const V* __restrict__ tw) {
    const int nthr = blockDim.x;
    const int tid = threadIdx.x;
    V* src = a;
    V* dst = b;
    for (int s = 0; s < f.nst; s++) {
        const int R = f.radix[s];
        const int nb = f.n / R;
        const int tot = nb * nrows;
        const V* tws = tw + f.twoff[s];
        for (int idx = tid; idx < tot; idx += nthr) {
            const int row = idx / nb;
            const int i = idx - row * nb;
            stage_bfly<DIR>(src + row * rs, dst + row * rs, f.n, R, f.p[s], tws, i);
        }
        __syncthreads();
        V* t = src; src = dst; dst = t;
    }
    return src;
}

}  // namespace prj

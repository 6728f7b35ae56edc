// fft_host.h -- host-side planning of the in-place DIF transforms: radix
// sequence, per-stage twiddles (extended precision, rounded once) and the
// digit-reversal position table.  Header-only so both the planned entry
// points and the no-allocation entry point fill their tables the same way,
// into caller-provided memory.
#pragma once
#include <cmath>
#include <cstring>

#include "fft_dif.cuh"
#include "fft_pass.cuh"

namespace prj {

// radices of the compile-time pass plan of length n in radix order `order` (0: the
// default of PRJ_PASS_PLANS, k >= 1: the k-th entry of n in PRJ_PASS_ALTS); 0 if none
inline int pass_radices(int n, int* fac, int cap, int order = 0) {
    int seen = 0;
#define PRJ_PASS_RADICES(N, ...)                                  \
    if (n == N && seen++ == order) {                              \
        const int r[] = {__VA_ARGS__};                            \
        const int nr = (int)(sizeof(r) / sizeof(r[0]));           \
        if (nr > cap) return -1;                                  \
        for (int i = 0; i < nr; i++) fac[i] = r[i];               \
        return nr;                                                \
    }
    PRJ_PASS_ALL(PRJ_PASS_RADICES)
#undef PRJ_PASS_RADICES
    return 0;
}

// radix orders compiled for length n (0 when n has no pass plan)
inline int pass_orders(int n) {
    int c = 0;
#define PRJ_PASS_COUNT(N, ...) \
    if (n == N) c++;
    PRJ_PASS_ALL(PRJ_PASS_COUNT)
#undef PRJ_PASS_COUNT
    return c;
}

// radix sequence of a length-n transform: the pass plan's radices (in radix order
// `order`) where one exists, else 8 first, then 4, 2, 3, 5, then any remaining primes;
// returns the number of stages or -1
inline int fft_factorize(int n, int* fac, int cap, int order = 0) {
    const int np = pass_radices(n, fac, cap, order);
    if (np != 0) return np;
    int nf = 0, m = n;
    auto push = [&](int r) { if (nf < cap) fac[nf] = r; nf++; };
    while (m % 8 == 0 && m != 16) { push(8); m /= 8; }
    while (m % 4 == 0) { push(4); m /= 4; }
    while (m % 2 == 0) { push(2); m /= 2; }
    for (int r : {3, 5}) while (m % r == 0) { push(r); m /= r; }
    for (int r = 7; m > 1; r += 2) {
        while (m % r == 0) { push(r); m /= r; }
        if ((long)r * r > m && m > 1) { push(m); m = 1; }
    }
    return nf <= cap ? nf : -1;
}

// true when every radix of n has a hard-coded DIF butterfly (2, 3, 4, 5, 6, 8)
inline bool dif_supported(int n) {
    int fac[64];
    const int nf = fft_factorize(n, fac, 64);
    if (nf < 0 || nf > kMaxStages) return false;
    for (int s = 0; s < nf; s++)
        if (!(fac[s] == 2 || fac[s] == 3 || fac[s] == 4 || fac[s] == 5 || fac[s] == 6 || fac[s] == 8)) return false;
    return true;
}

// fills the stage descriptor (radix order `order` where n has a pass plan); returns the
// number of twiddles (>= 1) or -1
inline long dif_plan(int n, DifDev* f, int order = 0) {
    int fac[kMaxStages];
    const int nf = fft_factorize(n, fac, kMaxStages, order);
    if (nf < 0) return -1;
    std::memset(f, 0, sizeof(*f));
    f->n = n;
    f->nst = nf;
    long cnt = 0;
    int L = n;
    for (int s = 0; s < nf; s++) {
        const int R = fac[s];
        f->radix[s] = R;
        f->span[s] = L;
        f->twoff[s] = (int)cnt;
        f->nbdiv[s] = make_fastdiv((unsigned)(n / R));
        f->mmdiv[s] = make_fastdiv((unsigned)(L / R));
        cnt += (long)(L / R) * (R - 1);
        L /= R;
    }
    return cnt > 0 ? cnt : 1;
}

// twiddle entries of a stage descriptor (what dif_plan returned for it)
inline long dif_twiddle_count(const DifDev& f) {
    long cnt = 0;
    for (int s = 0; s < f.nst; s++) cnt += (long)(f.span[s] / f.radix[s]) * (f.radix[s] - 1);
    return cnt > 0 ? cnt : 1;
}

// twiddles (forward sign; stage s at twoff[s], entry (q-1) mm + j, so the butterflies of
// consecutive j read consecutive entries) and positions: pos[k] = slot of index k after the transform
template <typename V>
inline void dif_fill(const DifDev& f, V* tw, int* pos) {
    const long double two_pi = 6.283185307179586476925286766559005768L;
    long c = 0;
    for (int s = 0; s < f.nst; s++) {
        const int R = f.radix[s], L = f.span[s], mm = L / R;
        for (int q = 1; q < R; q++)
            for (int j = 0; j < mm; j++) {
                const long double a = two_pi * (long double)q * j / (long double)L;
                tw[c].x = (decltype(tw[c].x))cosl(a);
                tw[c].y = (decltype(tw[c].y))(-sinl(a));
                c++;
            }
    }
    if (c == 0) { tw[0].x = 1; tw[0].y = 0; }
    for (int p = 0; p < f.n; p++) {
        int rem = p, k = 0, mult = 1;
        for (int s = 0; s < f.nst; s++) {
            const int R = f.radix[s];
            const int blk = f.span[s] / R;  // slots per digit value at this stage
            const int q = rem / blk;
            rem -= q * blk;
            k += q * mult;
            mult *= R;
        }
        pos[k] = p;
    }
}

// exp(-2 pi i k / n), k = 0..m (post-processing twiddles of a real transform)
template <typename V>
inline void real_post_fill(int n, int m, V* post) {
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int k = 0; k <= m; k++) {
        const long double a = two_pi * (long double)k / (long double)n;
        post[k].x = (decltype(post[k].x))cosl(a);
        post[k].y = (decltype(post[k].y))(-sinl(a));
    }
}

}  // namespace prj

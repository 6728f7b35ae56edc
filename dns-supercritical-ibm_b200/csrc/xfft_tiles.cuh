// xfft_tiles.cuh -- the pass-plan x transforms as per-tile device functions.
//
// A tile is tz x-rows (z0 .. z0+tz-1) of one y plane.  fwd_xp_tile: source (P, or
// the divergence of u_hat) -> packed complex -> DIF passes -> split X_k, X_{m-k} ->
// transposed store into the spectrum X[y][kx][z].  bwd_xp_tile: transposed load ->
// inverse split (scaled) -> DIT passes -> P rows.  The kernels k_fwd_xp / k_bwd_xp
// (prj_xfft.cu) run one tile per CTA; the persistent batch kernel (prj_batchk.cu)
// runs tiles of many cases from a work queue with the same code, so both give the
// same bits.  m = nx/2 has a compile-time plan PL; rows sit at stride
// pass_row_stride(m) in shared memory (`sm`, 16-byte aligned).
#pragma once
#include "cp_async.cuh"
#include "fft_dif.cuh"
#include "fft_pass.cuh"
#include "residual.cuh"
#include "tma_util.cuh"

struct prj_plan;

namespace prj {

#ifndef PRJ_X_UNROLL
#define PRJ_X_UNROLL 4
#endif
constexpr int kUnroll = PRJ_X_UNROLL;  // items whose global loads are in flight per thread in the load phases
// items per thread whose five field-row loads the divergence phase issues together
constexpr int kDivUnroll = 2;

__device__ __forceinline__ size_t hidx_d(int nx, int nz, int i, int j, int k) {
    return (size_t)(i + 1) + (size_t)(nx + 2) * ((size_t)(j + 1) + (size_t)(nz + 2) * (size_t)(k + 1));
}

struct XArgs {
    int nx, nz, ny, nh, m, tz, rs, even;
    DifDev f;
    const double2* tw;
    const int* pos;
    const double2* post;
    const double* P;
    const double* Uh;
    const double* Vh;
    const double* Wh;
    const double* inv_dy_p;
    double inv_dx, inv_dz, inv_dt, vbot, vtop, scale;
    double2* X;      // FP64 rows kx < kxs: X[(y kxs + kx) nz + z]
    float2* X32;     // FP32 rows kx >= kxs: X32[(y (nh - kxs) + kx - kxs) nz + z]
    int kxs;         // nh on the FP64 path
    int y0;          // first y plane of this launch (grid.y planes from y0)
    double* psum;    // bwd_xp_tile: per-tile sums of the written P values, [y][z tile], or null
    double* Pout;
    double* Bout;    // k_fwd_xd: copy of the source field (P layout), or null
    // fwd_xp_tile's residual source (SRC 3): r = B - A P of the pinned operator (residual.cuh)
    const double* B;       // right-hand side (P layout)
    const double* pm;      // plane means of P (ny)
    const double* bands;   // a, b, c, a00, b00, c00 (6 ny)
    double idx2, idz2;     // 1/dx^2, 1/dz^2
    int accum;       // k_bwd_xd: Pout += result instead of Pout = result
    double* sq;      // k_bwd_xd with accum: sq[0] += sum(update^2), sq[1] += sum(result^2), or null
};

// arguments of the pass-plan x tiles of a plan's FP64 Poisson solve of P in place (the
// persistent batch kernel's cases; prj_xfft.cu)
XArgs batch_x_args(const prj_plan* pl, double* P);

__device__ __forceinline__ void spec_store(const XArgs& a, int y, int kx, int z, double2 v) {
    if (kx < a.kxs) a.X[((size_t)y * a.kxs + kx) * a.nz + z] = v;
    else a.X32[((size_t)y * (a.nh - a.kxs) + (kx - a.kxs)) * a.nz + z] = make_float2((float)v.x, (float)v.y);
}

__device__ __forceinline__ double2 spec_load(const XArgs& a, int y, int kx, int z) {
    if (kx < a.kxs) return a.X[((size_t)y * a.kxs + kx) * a.nz + z];
    const float2 f = a.X32[((size_t)y * (a.nh - a.kxs) + (kx - a.kxs)) * a.nz + z];
    return make_double2(f.x, f.y);
}

// element g of the tz x rows buffer lives at slot sidx<true>(g) (bank-conflict padding)

// Staged inputs of the persistent batch kernel, which runs several tiles of one stage in
// a row and has the next tile's input copied into shared memory S (by the TMA unit) while
// the current tile computes: the forward's P rows z0 .. z0+nr-1 of plane y, contiguous in
// P, as S[r m + e]; the inverse's spectrum X[y][k][z0 + r] as S[k tz + r], k = 0 .. m.

// fwd_xp_tile: source (P, or the divergence of u_hat) -> packed complex -> DIF
// passes -> split X_k, X_{m-k} -> transposed store.  SRC 0 reads P in the first
// pass; SRC 1 stages the divergence in shared memory first; SRC 2 reads P from S
// (staged as above) and calls after_first() once S is no longer read (after the first
// pass); SRC 3 stages the residual B - A P (residual.cuh) in shared memory first.
// Tile (bx, by): rows z0 = bx tz .., plane y0 + by.
template <int SRC, class PL, class Hook = NoHook>
__device__ __forceinline__ void fwd_xp_tile(const XArgs& a, unsigned char* sm, int bx, int by,
                                            const double2* S = nullptr, Hook after_first = Hook{}) {
    double2* A = reinterpret_cast<double2*>(sm);
    constexpr int m = PL::n, nx = 2 * m, rs = pass_row_stride(m);
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int y = a.y0 + by, z0 = bx * a.tz;
    const int nr = min(a.tz, a.nz - z0);
    const double2* tw = a.tw;
    if (SRC == 1) {
        // divergence of the x pair (2e, 2e+1) of row z0 + r, as packed complex element e
        // (the operation order of div_at).  Each field row is read as the aligned pair
        // (interior 2e+1, 2e+2) -- halo'd positions 2e+2, 2e+3, 16-byte aligned because
        // the halo'd row length nx + 2 is even -- and interior 2e comes from the lane
        // holding item e-1 by shuffle (a scalar load where that lane holds another row
        // or is outside the warp).  The periodic wrap u(nx) = u(0) is a scalar load.
        const size_t hrow = (size_t)nx + 2, hplane = hrow * (size_t)(a.nz + 2);
        const double idy = a.inv_dy_p[y];
        const bool wb = (y == 0), wt = (y + 1 == a.ny);
        const int total = nr * m;
        const int lane = tid & 31;
        const unsigned full = 0xffffffffu;
        // all field loads of a group of kDivUnroll items are issued before any shuffle or
        // arithmetic (measured at 768x384x384: 0.88 ms against 0.98 ms for loads interleaved
        // with the arithmetic at 4 items, and 1.19 / 1.45 ms with 3 / 4 items grouped, which
        // spill)
        for (int base = tid - lane; base < total; base += kDivUnroll * nthr) {
            double2 pu[kDivUnroll], pw0[kDivUnroll], pw1[kDivUnroll], pv0[kDivUnroll], pv1[kDivUnroll];
#pragma unroll
            for (int u = 0; u < kDivUnroll; u++) {
                const int idx = base + u * nthr + lane;
                const bool in = idx < total;
                const int r = in ? idx / m : 0, e = in ? idx - r * m : 0;
                const int z = z0 + r, zp = (z + 1 == a.nz) ? 0 : z + 1;
                const size_t c0 = (size_t)(y + 1) * hplane + (size_t)(z + 1) * hrow + 1;
                const size_t cz = (size_t)(y + 1) * hplane + (size_t)(zp + 1) * hrow + 1;
                const size_t c1 = c0 + hplane;
                pu[u] = pw0[u] = pw1[u] = pv0[u] = pv1[u] = make_double2(0.0, 0.0);
                if (in) {
                    pu[u] = *reinterpret_cast<const double2*>(a.Uh + c0 + 2 * e + 1);
                    pw0[u] = *reinterpret_cast<const double2*>(a.Wh + c0 + 2 * e + 1);
                    pw1[u] = *reinterpret_cast<const double2*>(a.Wh + cz + 2 * e + 1);
                    if (!wb) pv0[u] = *reinterpret_cast<const double2*>(a.Vh + c0 + 2 * e + 1);
                    if (!wt) pv1[u] = *reinterpret_cast<const double2*>(a.Vh + c1 + 2 * e + 1);
                }
            }
#pragma unroll
            for (int u = 0; u < kDivUnroll; u++) {
                const int idx = base + u * nthr + lane;
                const bool in = idx < total;
                const int r = in ? idx / m : 0, e = in ? idx - r * m : 0;
                const int z = z0 + r, zp = (z + 1 == a.nz) ? 0 : z + 1;
                const size_t c0 = (size_t)(y + 1) * hplane + (size_t)(z + 1) * hrow + 1;
                const size_t cz = (size_t)(y + 1) * hplane + (size_t)(zp + 1) * hrow + 1;
                const size_t c1 = c0 + hplane;
                double u0 = __shfl_up_sync(full, pu[u].y, 1), w00 = __shfl_up_sync(full, pw0[u].y, 1);
                double w10 = __shfl_up_sync(full, pw1[u].y, 1), v00 = __shfl_up_sync(full, pv0[u].y, 1);
                double v10 = __shfl_up_sync(full, pv1[u].y, 1);
                if (!in) continue;
                if (lane == 0 || e == 0) {
                    u0 = a.Uh[c0 + 2 * e];
                    w00 = a.Wh[c0 + 2 * e];
                    w10 = a.Wh[cz + 2 * e];
                    if (!wb) v00 = a.Vh[c0 + 2 * e];
                    if (!wt) v10 = a.Vh[c1 + 2 * e];
                }
                if (wb) v00 = a.vbot;
                const double v01 = wb ? a.vbot : pv0[u].x;
                if (wt) v10 = a.vtop;
                const double v11 = wt ? a.vtop : pv1[u].x;
                const double u1 = pu[u].x;
                const double u2 = (e == m - 1) ? a.Uh[c0] : pu[u].y;
                double s0 = __dmul_rn(__dsub_rn(u1, u0), a.inv_dx);
                s0 = __dadd_rn(s0, __dmul_rn(__dsub_rn(w10, w00), a.inv_dz));
                s0 = __dadd_rn(s0, __dmul_rn(__dsub_rn(v10, v00), idy));
                double s1 = __dmul_rn(__dsub_rn(u2, u1), a.inv_dx);
                s1 = __dadd_rn(s1, __dmul_rn(__dsub_rn(pw1[u].x, pw0[u].x), a.inv_dz));
                s1 = __dadd_rn(s1, __dmul_rn(__dsub_rn(v11, v01), idy));
                const double2 vv = make_double2(__dmul_rn(a.inv_dt, s0), __dmul_rn(a.inv_dt, s1));
                if (a.Bout) {
                    double* b = a.Bout + ((size_t)y * a.nz + z) * nx + 2 * e;
                    b[0] = vv.x;
                    b[1] = vv.y;
                }
                A[sidx<true>(r * rs + e)] = vv;
            }
        }
        __syncthreads();
        dif_passes_shared<-1, PL, 0, PL::P>(A, nr, rs, tw);
    } else if (SRC == 3) {
        // the residual at the x pair (2e, 2e+1) of row z0 + r, as packed complex element e:
        // P, B and the z and wall-normal neighbour rows read as aligned pairs, the x
        // neighbours 2e-1 and 2e+2 (periodic) as scalars
        const int ny = a.ny, nz = a.nz;
        const double ak = a.bands[y], bk = a.bands[ny + y], ck = a.bands[2 * ny + y];
        const double pin = residual_pin(a.bands, a.pm, ny, y);
        const bool hkm = y > 0, hkp = y + 1 < ny;
        const size_t plane = (size_t)nz * nx;
        const int total = nr * m;
        for (int idx = tid; idx < total; idx += nthr) {
            const int r = idx / m, e = idx - r * m;
            const int z = z0 + r, zp = (z + 1 == nz) ? 0 : z + 1, zm = (z == 0) ? nz - 1 : z - 1;
            const size_t row = (size_t)y * plane + (size_t)z * nx;
            const double* p0 = a.P + row;
            const double2 pc = *reinterpret_cast<const double2*>(p0 + 2 * e);
            const double pxm = p0[e == 0 ? nx - 1 : 2 * e - 1];
            const double pxp = p0[e == m - 1 ? 0 : 2 * e + 2];
            const double2 pjp = *reinterpret_cast<const double2*>(a.P + (size_t)y * plane + (size_t)zp * nx + 2 * e);
            const double2 pjm = *reinterpret_cast<const double2*>(a.P + (size_t)y * plane + (size_t)zm * nx + 2 * e);
            double2 pkm = make_double2(0.0, 0.0), pkp = make_double2(0.0, 0.0);
            if (hkm) pkm = *reinterpret_cast<const double2*>(p0 - plane + 2 * e);
            if (hkp) pkp = *reinterpret_cast<const double2*>(p0 + plane + 2 * e);
            const double2 b = *reinterpret_cast<const double2*>(a.B + row + 2 * e);
            const double r0 = residual_at(b.x, pc.x, pc.y, pxm, pjp.x, pjm.x, pkm.x, pkp.x, hkm, hkp, a.idx2, a.idz2,
                                          ak, bk, ck, pin);
            const double r1 = residual_at(b.y, pc.y, pxp, pc.x, pjp.y, pjm.y, pkm.y, pkp.y, hkm, hkp, a.idx2, a.idz2,
                                          ak, bk, ck, pin);
            A[sidx<true>(r * rs + e)] = make_double2(r0, r1);
        }
        __syncthreads();
        dif_passes_shared<-1, PL, 0, PL::P>(A, nr, rs, tw);
    } else {
        const double2* src = reinterpret_cast<const double2*>(a.P) + ((size_t)y * a.nz + z0) * m;
        double2* bout = a.Bout ? reinterpret_cast<double2*>(a.Bout) + ((size_t)y * a.nz + z0) * m : nullptr;
        if constexpr (SRC == 2) {
            dif_first_pass<-1, PL>(A, nr, rs, tw, [&](int r, int e) { return S[(size_t)r * m + e]; });
        } else {
            dif_first_pass<-1, PL>(A, nr, rs, tw, [&](int r, int e) {
                const double2 v = src[(size_t)r * m + e];
                if (bout) bout[(size_t)r * m + e] = v;
                return v;
            });
        }
        __syncthreads();
        after_first();
        dif_passes_shared<-1, PL, 1, PL::P>(A, nr, rs, tw);
    }
    // split: X_k = E_k + W^k O_k, X_{m-k} = conj(E_k) + W^{m-k} conj(O_k); row index fastest
    constexpr int half = m / 2;
    for (int idx = tid; idx < nr * (half + 1); idx += nthr) {
        const int k = idx / nr, r = idx - k * nr;
        const int base = r * rs;
        const int z = z0 + r;
        if (k == 0) {
            const double2 c = A[sidx<true>(base)];
            spec_store(a, y, 0, z, make_double2(c.x + c.y, 0.0));
            spec_store(a, y, m, z, make_double2(c.x - c.y, 0.0));
        } else {
            const int kk = m - k;
            const double2 zk = A[sidx<true>(base + pass_slot<PL>(k))];
            const double2 zm = cconj(A[sidx<true>(base + pass_slot<PL>(kk))]);
            const double2 e = cscale(cadd(zk, zm), 0.5);
            const double2 d = csub(zk, zm);
            const double2 o = make_double2(0.5 * d.y, -0.5 * d.x);
            spec_store(a, y, k, z, cadd(e, cmul(a.post[k], o)));
            if (kk != k) spec_store(a, y, kk, z, cadd(cconj(e), cmul(a.post[kk], cconj(o))));
        }
    }
}

// bwd_xp_tile: transposed load of X_k, X_{m-k} -> inverse split (scaled) into slot
// order -> DIT passes -> P rows (x pairs as double2), optionally accumulated; the
// tile's partial sum of P goes to psum[y][bx] (tiles_per_plane entries per plane).
// EXTRAS = false: plain P = result (no accumulation, partial sums or norms), the form of
// the persistent batch kernel.  STAGED: the spectrum comes from S (staged as above), and
// after_split() is called once S is no longer read.
template <class PL, bool EXTRAS = true, bool STAGED = false, class Hook = NoHook>
__device__ __forceinline__ void bwd_xp_tile(const XArgs& a, unsigned char* sm, int bx, int by, int tiles_per_plane,
                                            const double2* S = nullptr, Hook after_split = Hook{}) {
    double2* A = reinterpret_cast<double2*>(sm);
    constexpr int m = PL::n, rs = pass_row_stride(m), half = m / 2;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int y = a.y0 + by, z0 = bx * a.tz;
    const int nr = min(a.tz, a.nz - z0);
    const double s = a.scale;
    const int total = nr * (half + 1);
    // X_k and X_{m-k} of kUnroll items loaded together (independent loads in flight)
    for (int base0 = tid; base0 < total; base0 += kUnroll * nthr) {
        double2 xa[kUnroll], xb[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
            const int idx = base0 + u * nthr;
            if (idx < total) {
                const int k = idx / nr, r = idx - k * nr;
                if constexpr (STAGED) {
                    xa[u] = S[k * a.tz + r];
                    xb[u] = S[(m - k) * a.tz + r];
                } else {
                    xa[u] = spec_load(a, y, k, z0 + r);
                    xb[u] = spec_load(a, y, m - k, z0 + r);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
            const int idx = base0 + u * nthr;
            if (idx >= total) continue;
            const int k = idx / nr, r = idx - k * nr;
            const int base = r * rs;
            if (k == 0) {
                const double x0 = xa[u].x, xm = xb[u].x;
                A[sidx<true>(base)] = make_double2((x0 + xm) * s, (x0 - xm) * s);
            } else {
                const int kk = m - k;
                const double2 xk = xa[u], xkk = xb[u];
                const double2 e1 = cadd(xk, cconj(xkk));
                const double2 o1 = cmulc(csub(xk, cconj(xkk)), a.post[k]);
                A[sidx<true>(base + pass_slot<PL>(k))] = cscale(make_double2(e1.x - o1.y, e1.y + o1.x), s);
                if (kk != k) {
                    const double2 e2 = cadd(xkk, cconj(xk));
                    const double2 o2 = cmulc(csub(xkk, cconj(xk)), a.post[kk]);
                    A[sidx<true>(base + pass_slot<PL>(kk))] = cscale(make_double2(e2.x - o2.y, e2.y + o2.x), s);
                }
            }
        }
    }
    __syncthreads();
    after_split();
    dit_passes_shared<+1, PL, PL::P - 1, 0>(A, nr, rs, a.tw);
    double2* out = reinterpret_cast<double2*>(a.Pout) + ((size_t)y * a.nz + z0) * m;
    double sq0 = 0.0, sq1 = 0.0, ps = 0.0;
    if constexpr (!EXTRAS) {
        dit_last_pass<+1, PL>(A, nr, rs, a.tw, [&](int r, int e, double2 v) { out[(size_t)r * m + e] = v; });
        return;
    }
    dit_last_pass<+1, PL>(A, nr, rs, a.tw, [&](int r, int e, double2 v) {
        double2* o = out + (size_t)r * m + e;
        if (a.accum) {
            const double2 old = *o;
            const double2 nv = make_double2(old.x + v.x, old.y + v.y);
            sq0 += v.x * v.x + v.y * v.y;
            sq1 += nv.x * nv.x + nv.y * nv.y;
            ps += nv.x + nv.y;
            *o = nv;
        } else {
            ps += v.x + v.y;
            *o = v;
        }
    });
    if (a.psum) {
        // the tile's sum in a fixed order (per thread, then warp butterfly, then warps in order)
        __shared__ double wsum[kPassThreads / 32];
        for (int o = 16; o > 0; o >>= 1) ps += __shfl_xor_sync(0xffffffffu, ps, o);
        if ((tid & 31) == 0) wsum[tid >> 5] = ps;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int w = 0; w < nthr / 32; w++) t += wsum[w];
            a.psum[(size_t)y * tiles_per_plane + bx] = t;
        }
    }
    if (a.sq) {
        for (int o = 16; o > 0; o >>= 1) {
            sq0 += __shfl_xor_sync(0xffffffffu, sq0, o);
            sq1 += __shfl_xor_sync(0xffffffffu, sq1, o);
        }
        if ((tid & 31) == 0) {
            atomicAdd(a.sq, sq0);
            atomicAdd(a.sq + 1, sq1);
        }
    }
}

// spectrum boxes of an inverse x tile: k = 0 .. m in boxes of at most 256 wavenumbers;
// with more than one box, a multiple of 8 wavenumbers per box, so every box lands on a
// 128-byte boundary of S (rows past m are zero-filled and unread)
inline int x_boxes(int m) { return (m + 1 + 255) / 256; }
inline int x_box_k(int m) {
    const int b = x_boxes(m), k = (m + 1 + b - 1) / b;
    return b == 1 ? k : (k + 7) / 8 * 8;
}

// Tiles t = first, first + stride, ... < end of an x transform (tile (t % tpp, t / tpp)) as a
// pipeline: the next tile's input is copied into the staging buffer S (128-byte aligned at or
// after sm + soff, sbytes long, followed by an mbarrier) by the TMA unit -- FWD: the tile's P
// rows, contiguous, by one bulk copy; inverse: its spectrum block X[y][k][z0 ..] by `boxes`
// boxes of box_k wavenumbers of the 3-D tensor map `xmap` ({2 nz doubles, nh, ny}, box
// {2 tz, box_k, 1}; FP64 rows only) -- while the current tile runs its FFT passes and stores.
// The tiles compute as fwd_xp_tile<2> / bwd_xp_tile<STAGED>, so the results are those of the
// one-tile kernels.  A wait that runs out raises *err (6) and ends the run.
template <class PL, bool FWD, bool EXTRAS>
__device__ __forceinline__ void x_tiles_tma(const XArgs& a, const void* xmap, int tpp, int boxes, int box_k,
                                            unsigned char* sm, int soff, int sbytes, int first, int stride, int end,
                                            int* err) {
    constexpr int m = PL::n;
    const int tid = threadIdx.x;
    if (first >= end) return;
    double2* S = reinterpret_cast<double2*>(align128(sm + soff));
    uint64_t* bar = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(S) + sbytes);
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    uint32_t phase = 0;
    auto stage = [&](int t) {  // thread 0
        const int bx = t % tpp, by = t / tpp;
        const int y = a.y0 + by, z0 = bx * a.tz;
        fence_proxy_async_shared();  // S's earlier reads before the copy's writes
        if constexpr (FWD) {
            const int nr = min(a.tz, a.nz - z0);
            const uint32_t bytes = (uint32_t)nr * m * (uint32_t)sizeof(double2);
            mbar_arrive_expect_tx(bar, bytes);
            bulk_g2s(S, reinterpret_cast<const double2*>(a.P) + ((size_t)y * a.nz + z0) * m, bytes, bar);
        } else {
            mbar_arrive_expect_tx(bar, (uint32_t)(boxes * box_k * a.tz) * (uint32_t)sizeof(double2));
            for (int b = 0; b < boxes; b++) tma_load_3d(S + (size_t)b * box_k * a.tz, xmap, 2 * z0, b * box_k, y, bar);
        }
    };
    if (tid == 0) stage(first);
    for (int t = first; t < end; t += stride) {
        const bool ok = mbar_wait_bounded(bar, phase);
        if (__syncthreads_or(!ok)) {  // S holds tile t for every thread (else: give up the run)
            if (tid == 0) {
                atomicExch(err, 6);
                mbar_wait_bounded(bar, phase);
            }
            break;
        }
        phase ^= 1u;
        const int nt = t + stride;
        auto next = [&] {
            if (tid == 0 && nt < end) stage(nt);
        };
        // (the next iteration's barrier orders this tile's reads of its area before the next
        // tile's writes)
        if constexpr (FWD) fwd_xp_tile<2, PL>(a, sm, t % tpp, t / tpp, S, next);
        else bwd_xp_tile<PL, EXTRAS, true>(a, sm, t % tpp, t / tpp, tpp, S, next);
    }
    __syncthreads();
    if (tid == 0) mbar_inval(bar);
}

}  // namespace prj

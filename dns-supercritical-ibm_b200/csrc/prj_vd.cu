// prj_vd.cu -- variable-density pressure splitting (use_incompressible = false).
//
// The Poisson operator stays the constant-coefficient one of the plan; only the
// right-hand side and the correction change (mod_cfd_subroutines.f90):
//   rho_min  = min rho over the interior                               (:476-486)
//   RHS      = rho_min/dt (div u_hat - div_now)
//              + sum_d D_d[(1 - rho_min avg(1/rho)) D_d Ps],  Ps = 2 P_now - P_old   (:538-573)
//   u        = u_hat - dt grad(P/rho_min + (avg(1/rho) - 1/rho_min) Ps)             (:1153-1197)
//   P_next   = P with periodic x/z halos and wall ghost planes (P_per, :1087-1118),
//              the caller's next P_now (the reference copies P_now -> P_old and
//              P_per -> P_now, :1199-1221; here the caller swaps pointers).
// rho, P_now, P_old and div_now are halo'd fields whose halos the caller fills,
// read as given (the reference reads them after its halo exchanges).  Every
// expression keeps the reference's operation order with round-to-nearest
// intrinsics.  rho_min stays on the device (an order-preserving integer image of
// the double, reduced with atomicMin), so the step needs no host round trip.
#include "prj_internal.h"

namespace prj {

namespace {

__device__ __forceinline__ size_t hix(int nx, int nz, int i, int j, int k) {
    return (size_t)(i + 1) + (size_t)(nx + 2) * ((size_t)(j + 1) + (size_t)(nz + 2) * (size_t)(k + 1));
}

// order-preserving map of doubles to unsigned 64-bit integers (and back)
__device__ __forceinline__ unsigned long long ord_of(double d) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(d);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double of_ord(unsigned long long o) {
    const unsigned long long b = (o >> 63) ? (o & 0x7fffffffffffffffull) : ~o;
    return __longlong_as_double((long long)b);
}

// one read of rho: ih = 0.5 / rho on the whole halo'd box (the quotient both stencils form
// for every neighbour, computed once: the same correctly rounded values), and rho_min, the
// minimum over the interior (mod_cfd_subroutines.f90:476-486), reduced by fmin and an
// atomicMin on the order-preserving integer image, both exact and order-free.  One warp per
// halo'd x-row (the row's plane and z index from one division per row, not per element).
__global__ void __launch_bounds__(256) k_rho_prep(int nx, int nz, int ny, const double* __restrict__ rho,
                                                  double* __restrict__ ih, unsigned long long* out) {
    const int hx = nx + 2, hz = nz + 2, rows = hz * (ny + 2), lane = threadIdx.x & 31;
    const int nw = (int)((gridDim.x * blockDim.x) >> 5);
    double m = 1e20;  // mod_cfd_subroutines.f90:476
    for (int r = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); r < rows; r += nw) {
        const int z = r % hz, y = r / hz;
        const bool inner = z >= 1 && z <= nz && y >= 1 && y <= ny;
        const double* src = rho + (size_t)r * hx;
        double* dst = ih + (size_t)r * hx;
        // eight loads in flight per lane before the quotients
        constexpr int U = 8;
        for (int x0 = lane; x0 < hx; x0 += 32 * U) {
            double v[U];
#pragma unroll
            for (int u = 0; u < U; u++) v[u] = x0 + 32 * u < hx ? src[x0 + 32 * u] : 1.0;
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int x = x0 + 32 * u;
                if (x < hx) {
                    dst[x] = __ddiv_rn(0.5, v[u]);
                    if (inner && x >= 1 && x <= nx) m = fmin(m, v[u]);
                }
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) atomicMin(out, ord_of(m));
}

struct VdArgs {
    int nx, nz, ny;
    const double* Uh;
    const double* Vh;
    const double* Wh;
    const double* rho;
    const double* ih;       // 0.5 / rho (halo'd)
    const double* Pn;
    const double* Po;
    const double* div_now;
    const double* inv_dy_p;
    const double* pad;      // inv_dy_p_pad (ny+1)
    const unsigned long long* rho_min;
    const double* lo;
    const double* hi;
    const double* P;
    double* Pout;           // RHS (k_vd_rhs)
    double* U;
    double* V;
    double* W;
    double* Pnext;
    double dt, inv_dt, inv_dx, inv_dz, inv_dx2, inv_dz2;
    double wall[6];
};

__device__ __forceinline__ double ps(const VdArgs& a, size_t h) {
    return __dsub_rn(__dmul_rn(2.0, a.Pn[h]), a.Po[h]);
}
// 1 - rho_min (0.5/rho_nbr + 0.5/rho_c), given hn = 0.5/rho_nbr and hc = 0.5/rho_c (each
// quotient computed once per point: the same correctly rounded value the reference forms)
__device__ __forceinline__ double rho_w(double rmin, double hn, double hc) {
    return __dsub_rn(1.0, __dmul_rn(rmin, __dadd_rn(hn, hc)));
}

// RHS of the constant-coefficient Poisson equation, one CTA per (y, z) row
__global__ void __launch_bounds__(128) k_vd_rhs(const VdArgs a) {
    const int nx = a.nx, nz = a.nz, ny = a.ny;
    const int k = blockIdx.x, j = blockIdx.y;
    const int jp = (j + 1 == nz) ? 0 : j + 1;
    const double rmin = of_ord(*a.rho_min);
    const double idy = a.inv_dy_p[k], padp = a.pad[k + 1], padm = a.pad[k];
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        const int ip = (i + 1 == nx) ? 0 : i + 1;
        const size_t h = hix(nx, nz, i, j, k);
        const double vp = (k + 1 == ny) ? a.wall[4] : a.Vh[hix(nx, nz, i, j, k + 1)];
        const double v0 = (k == 0) ? a.wall[1] : a.Vh[h];
        double dv = __dmul_rn(__dsub_rn(a.Uh[hix(nx, nz, ip, j, k)], a.Uh[h]), a.inv_dx);
        dv = __dadd_rn(dv, __dmul_rn(__dsub_rn(a.Wh[hix(nx, nz, i, jp, k)], a.Wh[h]), a.inv_dz));
        dv = __dadd_rn(dv, __dmul_rn(__dsub_rn(vp, v0), idy));
        const size_t hxp = hix(nx, nz, i + 1, j, k), hxm = hix(nx, nz, i - 1, j, k);
        const size_t hzp = hix(nx, nz, i, j + 1, k), hzm = hix(nx, nz, i, j - 1, k);
        const size_t hyp = hix(nx, nz, i, j, k + 1), hym = hix(nx, nz, i, j, k - 1);
        const double p00 = ps(a, h);
        const double h0 = a.ih[h];
        const double X = __dsub_rn(__dmul_rn(rho_w(rmin, a.ih[hxp], h0), __dsub_rn(ps(a, hxp), p00)),
                                   __dmul_rn(rho_w(rmin, a.ih[hxm], h0), __dsub_rn(p00, ps(a, hxm))));
        const double Z = __dsub_rn(__dmul_rn(rho_w(rmin, a.ih[hzp], h0), __dsub_rn(ps(a, hzp), p00)),
                                   __dmul_rn(rho_w(rmin, a.ih[hzm], h0), __dsub_rn(p00, ps(a, hzm))));
        const double Y =
            __dsub_rn(__dmul_rn(__dmul_rn(rho_w(rmin, a.ih[hyp], h0), __dsub_rn(ps(a, hyp), p00)), padp),
                      __dmul_rn(__dmul_rn(rho_w(rmin, a.ih[hym], h0), __dsub_rn(p00, ps(a, hym))), padm));
        const double L = __dadd_rn(__dadd_rn(__dmul_rn(X, a.inv_dx2), __dmul_rn(Z, a.inv_dz2)), __dmul_rn(Y, idy));
        const double t1 = __dmul_rn(__dmul_rn(a.inv_dt, dv), rmin);
        const double t2 = __dmul_rn(__dmul_rn(a.inv_dt, rmin), a.div_now[h]);
        a.Pout[((size_t)k * nz + j) * nx + i] = __dadd_rn(__dsub_rn(t1, t2), L);
    }
}

// P/rho_min + (avg(1/rho) - 1/rho_min) Ps at halo'd index h, P_per value p
__device__ __forceinline__ double pmix(const VdArgs& a, double p, size_t h, double irn, double irm) {
    return __dadd_rn(__dmul_rn(p, irm), __dmul_rn(__dsub_rn(irn, irm), ps(a, h)));
}

// correction + boundary fill + P_next on the whole halo'd box, one CTA per halo'd x-row
__global__ void __launch_bounds__(128) k_vd_correct(const VdArgs a) {
    const int nx = a.nx, nz = a.nz, ny = a.ny;
    const int jh = blockIdx.y;
    const int k = (int)blockIdx.x - 1;
    const size_t rowh = (size_t)(nx + 2) * ((size_t)jh + (size_t)(nz + 2) * (size_t)(k + 1));
    const int j = jh - 1;
    const int jw = j < 0 ? nz - 1 : (j == nz ? 0 : j);
    const int kc = k < 0 ? 0 : (k == ny ? ny - 1 : k);
    const double* Pc = a.P + ((size_t)kc * nz + jw) * nx;
    if (k < 0 || k == ny) {
        const double u = k < 0 ? a.wall[0] : a.wall[3];
        const double v = k < 0 ? a.wall[1] : a.wall[4];
        const double w = k < 0 ? a.wall[2] : a.wall[5];
        for (int ih = threadIdx.x; ih < nx + 2; ih += blockDim.x) {
            const int i = ih - 1;
            const int iw = i < 0 ? nx - 1 : (i == nx ? 0 : i);
            a.U[rowh + ih] = u;
            a.V[rowh + ih] = v;
            a.W[rowh + ih] = w;
            a.Pnext[rowh + ih] = Pc[iw];
        }
        return;
    }
    const double irm = __ddiv_rn(1.0, of_ord(*a.rho_min));
    const int jm = jw == 0 ? nz - 1 : jw - 1;
    const double* Pjm = a.P + ((size_t)k * nz + jm) * nx;
    const double* Pkm = a.P + ((size_t)(k > 0 ? k - 1 : 0) * nz + jw) * nx;
    const double hi = a.hi[k], lo = a.lo[k];
    for (int ih = threadIdx.x; ih < nx + 2; ih += blockDim.x) {
        const int i = ih - 1;
        const int iw = i < 0 ? nx - 1 : (i == nx ? 0 : i);
        const int im = iw == 0 ? nx - 1 : iw - 1;
        const size_t h = hix(nx, nz, iw, jw, k);
        const double p0 = Pc[iw];
        const double r0 = a.ih[h];
        // x face (MCS:1158-1164): neighbours at iw - 1 in the caller's halo'd arrays
        size_t hm = hix(nx, nz, iw - 1, jw, k);
        double irn = __dadd_rn(r0, a.ih[hm]);
        double pf = pmix(a, p0, h, irn, irm), pb = pmix(a, Pc[im], hm, irn, irm);
        const double u = __dsub_rn(a.Uh[h], __dmul_rn(__dmul_rn(a.dt, __dsub_rn(pf, pb)), a.inv_dx));
        // z face (:1168-1175)
        hm = hix(nx, nz, iw, jw - 1, k);
        irn = __dadd_rn(r0, a.ih[hm]);
        pf = pmix(a, p0, h, irn, irm);
        pb = pmix(a, Pjm[iw], hm, irn, irm);
        const double w = __dsub_rn(a.Wh[h], __dmul_rn(__dmul_rn(a.dt, __dsub_rn(pf, pb)), a.inv_dz));
        // y face (:1179-1186), k >= kmin_Vhat = 1; V(0) is the bottom wall
        double v = a.wall[1];
        if (k > 0) {
            hm = hix(nx, nz, iw, jw, k - 1);
            irn = __dadd_rn(r0, a.ih[hm]);
            pf = pmix(a, p0, h, irn, irm);
            pb = pmix(a, Pkm[iw], hm, irn, irm);
            v = __dsub_rn(a.Vh[h], __dmul_rn(a.dt, __dadd_rn(__dmul_rn(hi, pf), __dmul_rn(lo, pb))));
        }
        a.U[rowh + ih] = u;
        a.V[rowh + ih] = v;
        a.W[rowh + ih] = w;
        a.Pnext[rowh + ih] = p0;
    }
}

}  // namespace

cudaError_t launch_vd_prep(const prj_plan* pl, const double* rho, double* ih, unsigned long long* slot,
                           cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(slot, 0xff, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    const Geometry& g = pl->g;
    // eight warps per CTA, one halo'd row per warp at a time, one wave of resident CTAs
    int dev = 0, sms = 0, per = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_rho_prep, 256, 0)) != cudaSuccess) return e;
    const long long rows = (long long)(g.nz + 2) * (g.ny + 2);
    const unsigned blocks = (unsigned)std::max(1LL, std::min<long long>((rows + 7) / 8, (long long)std::max(per, 1) * sms));
    k_rho_prep<<<blocks, 256, 0, st>>>(g.nx, g.nz, g.ny, rho, ih, slot);
    return cudaGetLastError();
}

static VdArgs vd_args(const prj_plan* pl, const VdFields& f, const StepScalars& sc, const unsigned long long* slot) {
    const Geometry& g = pl->g;
    VdArgs a{};
    a.nx = g.nx; a.nz = g.nz; a.ny = g.ny;
    a.rho = f.rho; a.ih = pl->vd_ih; a.Pn = f.P_now; a.Po = f.P_old; a.div_now = f.div_now;
    a.inv_dy_p = pl->t.inv_dy_p; a.pad = pl->vd_pad; a.rho_min = slot;
    a.lo = pl->t.dpdy_lo; a.hi = pl->t.dpdy_hi;
    a.dt = sc.dt; a.inv_dt = sc.inv_dt;
    a.inv_dx = 1.0 / g.dx; a.inv_dz = 1.0 / g.dz;
    a.inv_dx2 = a.inv_dx * a.inv_dx; a.inv_dz2 = a.inv_dz * a.inv_dz;
    for (int i = 0; i < 6; i++) a.wall[i] = sc.wall[i];
    return a;
}

cudaError_t launch_vd_rhs(const prj_plan* pl, const double* Uh, const double* Vh, const double* Wh, const VdFields& f,
                          const StepScalars& sc, const unsigned long long* slot, double* P, cudaStream_t st) {
    VdArgs a = vd_args(pl, f, sc, slot);
    a.Uh = Uh; a.Vh = Vh; a.Wh = Wh; a.Pout = P;
    k_vd_rhs<<<dim3((unsigned)pl->g.ny, (unsigned)pl->g.nz), 128, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_vd_correction(const prj_plan* pl, const double* P, const double* Uh, const double* Vh,
                                 const double* Wh, const VdFields& f, const StepScalars& sc,
                                 const unsigned long long* slot, double* U, double* V, double* W, cudaStream_t st) {
    VdArgs a = vd_args(pl, f, sc, slot);
    a.P = P; a.Uh = Uh; a.Vh = Vh; a.Wh = Wh;
    a.U = U; a.V = V; a.W = W; a.Pnext = f.P_next;
    k_vd_correct<<<dim3((unsigned)(pl->g.ny + 2), (unsigned)(pl->g.nz + 2)), 128, 0, st>>>(a);
    return cudaGetLastError();
}

double vd_rho_min_host(unsigned long long o) {
    const unsigned long long b = (o >> 63) ? (o & 0x7fffffffffffffffull) : ~o;
    double d;
    std::memcpy(&d, &b, sizeof(d));
    return d;
}

}  // namespace prj

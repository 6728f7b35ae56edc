// prj_abi.cu -- host side of the engine: FFT planning, plan set-up and the
// extern "C" entry points declared in include/projection.h.
//
// The plan builder takes over the work of init_spec_poisson_multigpu
// (src/poisson_solver_mgpu_dtdma/poisson_solver_multigpu.f90:33-326) for one
// rank: FFT plans, the a_x / a_z wavenumber tables (:133-155, computed here in
// host double precision with the C library's sin, as the reference does on the
// CPU build), and the Thomas pivot table (the analogue of poi_C, :164-179).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/projection.h"
#include "fft_host.h"
#include "div_rn.cuh"
#include "prj_internal.h"

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    if (e == cudaErrorMemoryAllocation)
        return fail(PRJ_ERR_OOM, "%s: %s", what, cudaGetErrorString(e));
    return fail(PRJ_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call, what)                                   \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

// radix sequence of a complex FFT of length n (8 first, then 4, 2, 3, 5, others)
std::vector<int> factorize(int n) {
    std::vector<int> f;
    int m = n;
    while (m % 8 == 0 && m != 16) { f.push_back(8); m /= 8; }
    while (m % 4 == 0) { f.push_back(4); m /= 4; }
    while (m % 2 == 0) { f.push_back(2); m /= 2; }
    for (int r : {3, 5}) while (m % r == 0) { f.push_back(r); m /= r; }
    for (int r = 7; m > 1; r += 2) {
        while (m % r == 0) { f.push_back(r); m /= r; }
        if ((long)r * r > m && m > 1) { f.push_back(m); m = 1; }
    }
    return f;
}

const long double kTwoPi = 6.283185307179586476925286766559005768L;

template <typename T>
using C2 = typename prj::C2<T>::t;

template <typename T>
C2<T> cexpm(long double num, long double den) {  // exp(-2 pi i num/den)
    const long double a = kTwoPi * num / den;
    C2<T> v;
    v.x = (T)cosl(a);
    v.y = (T)(-sinl(a));
    return v;
}

// Build stage tables on the host; returns the device twiddle buffer.
template <typename T>
int make_cfft(int n, prj::FftDev* f, C2<T>** d_tw, size_t* bytes) {
    std::vector<int> fac = factorize(n);
    if ((int)fac.size() > prj::kMaxStages) return fail(PRJ_ERR_UNSUPPORTED, "FFT length %d needs too many stages", n);
    std::memset(f, 0, sizeof(*f));
    f->n = n;
    f->nst = (int)fac.size();
    std::vector<C2<T>> tw;
    int p = 1;
    for (int s = 0; s < f->nst; s++) {
        const int R = fac[s];
        if (R > 64) return fail(PRJ_ERR_UNSUPPORTED, "FFT length %d has prime factor %d > 64", n, R);
        f->radix[s] = R;
        f->p[s] = p;
        f->twoff[s] = (int)tw.size();
        for (int k = 0; k < p; k++)
            for (int r = 1; r < R; r++) tw.push_back(cexpm<T>((long double)r * k, (long double)p * R));
        const bool hard = (R == 2 || R == 3 || R == 4 || R == 5 || R == 8);
        if (!hard)
            for (int m = 0; m < R; m++) tw.push_back(cexpm<T>((long double)m, (long double)R));
        p *= R;
    }
    if (tw.empty()) tw.push_back(cexpm<T>(0, 1));
    *bytes += tw.size() * sizeof(C2<T>);
    CK(cudaMalloc((void**)d_tw, tw.size() * sizeof(C2<T>)), "cudaMalloc(twiddles)");
    CK(cudaMemcpy(*d_tw, tw.data(), tw.size() * sizeof(C2<T>), cudaMemcpyHostToDevice), "cudaMemcpy(twiddles)");
    return PRJ_OK;
}

template <typename T>
int make_rfft(int n, prj::RealFftPlan<T>* r, size_t* bytes) {
    r->n = n;
    r->nh = n / 2 + 1;
    r->even = (n % 2 == 0);
    r->m = r->even ? n / 2 : n;
    int rc = make_cfft<T>(r->m, &r->f, &r->tw, bytes);
    if (rc) return rc;
    std::vector<C2<T>> post((size_t)r->m + 1);
    for (int k = 0; k <= r->m; k++) post[k] = cexpm<T>((long double)k, (long double)n);
    *bytes += post.size() * sizeof(C2<T>);
    CK(cudaMalloc((void**)&r->post, post.size() * sizeof(C2<T>)), "cudaMalloc(post twiddles)");
    CK(cudaMemcpy(r->post, post.data(), post.size() * sizeof(C2<T>), cudaMemcpyHostToDevice), "cudaMemcpy(post)");
    return PRJ_OK;
}

template <typename P>
void dfree(P*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
}

// in-place DIF tables of a length-n transform in radix order `order` (left unset when a
// radix is unsupported)
int make_dif(int n, prj::DifFft* d, size_t* bytes, int order = 0) {
    d->ok = false;
    if (!prj::dif_supported(n)) return PRJ_OK;
    const long ntw = prj::dif_plan(n, &d->f, order);
    if (ntw < 0) return PRJ_OK;
    std::vector<double2> tw((size_t)ntw);
    std::vector<int> pos((size_t)n);
    prj::dif_fill(d->f, tw.data(), pos.data());
    CK(cudaMalloc((void**)&d->tw, tw.size() * sizeof(double2)), "cudaMalloc(DIF twiddles)");
    CK(cudaMemcpy(d->tw, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice), "cudaMemcpy(DIF twiddles)");
    CK(cudaMalloc((void**)&d->pos, pos.size() * sizeof(int)), "cudaMalloc(DIF positions)");
    CK(cudaMemcpy(d->pos, pos.data(), pos.size() * sizeof(int), cudaMemcpyHostToDevice), "cudaMemcpy(DIF positions)");
    *bytes += tw.size() * sizeof(double2) + pos.size() * sizeof(int);
    d->ok = true;
    return PRJ_OK;
}

// slot -> wavenumber table of the length-n in-place plan (inverse of its position table)
int make_slot_table(int n, int** d_out, size_t* bytes, int order = 0) {
    prj::DifDev f{};
    const long ntw = prj::dif_plan(n, &f, order);
    if (ntw < 0) return fail(PRJ_ERR_UNSUPPORTED, "no in-place plan for length %d", n);
    std::vector<double2> tw((size_t)ntw);
    std::vector<int> pos((size_t)n), kz((size_t)n);
    prj::dif_fill(f, tw.data(), pos.data());
    for (int k = 0; k < n; k++) kz[pos[k]] = k;
    CK(cudaMalloc((void**)d_out, kz.size() * sizeof(int)), "cudaMalloc(slot table)");
    CK(cudaMemcpy(*d_out, kz.data(), kz.size() * sizeof(int), cudaMemcpyHostToDevice), "cudaMemcpy(slot table)");
    *bytes += kz.size() * sizeof(int);
    return PRJ_OK;
}

// default z-direction kernels (prj_tuning.z_mode changes them; split and line need the
// in-place plan): the per-wavenumber kernel when there are at least two x wavenumbers
// (its CTAs) per SM, else the split kernels.  Measured on B200, the per-wavenumber kernel
// took 1.12 / 1.41 / 6.91 ms against 1.31 / 1.49 / 7.87 ms for nx/2+1 = 385 / 513 / 769,
// but 0.30 / 0.45 ms against 0.21 / 0.37 ms for 193 / 257.
int z_mode(bool split_ok, bool line_pref) { return split_ok ? (line_pref ? 3 : 0) : 1; }

void free_plan_buffers(prj_plan* pl) {
    dfree(pl->t.bands);
    dfree(pl->t.inv_dy_p);
    dfree(pl->t.dpdy_lo);
    dfree(pl->t.dpdy_hi);
    dfree(pl->t.ax);
    dfree(pl->t.az);
    dfree(pl->t.piv);
    dfree(pl->t.pivc);
    dfree(pl->fx64.tw);
    dfree(pl->fx64.post);
    dfree(pl->fz64.tw);
    dfree(pl->xd.tw);
    dfree(pl->xd.pos);
    dfree(pl->zd.tw);
    dfree(pl->zd.pos);
    dfree(pl->kz_of_slot);
    dfree(pl->spec32);
    dfree(pl->pbar);
    dfree(pl->psum);
    dfree(pl->mix_b);
    dfree(pl->mix_r);
    pl->xd.ok = pl->zd.ok = false;
    dfree(pl->spec);
    dfree(pl->stat_buf);
    dfree(pl->vd_pad);
    dfree(pl->vd_ih);
    for (cudaStream_t& hs : pl->hp_st) {
        if (hs) cudaStreamSynchronize(hs);
    }
    for (double*& hb : pl->hp_stage) dfree(hb);
    for (cudaEvent_t& he : pl->hp_ev) {
        if (he) cudaEventDestroy(he);
        he = nullptr;
    }
    for (cudaStream_t& hs : pl->hp_st) {
        if (hs) cudaStreamDestroy(hs);
        hs = nullptr;
    }
    dfree(pl->host_stage);
    pl->host_stage_elems = 0;
}

bool finite_all(const double* v, int n) {
    for (int i = 0; i < n; i++)
        if (!std::isfinite(v[i])) return false;
    return true;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

int check_plan(const prj_plan* pl) {
    if (!pl) return fail(PRJ_ERR_ARG, "plan is NULL");
    if (!pl->spec) return fail(PRJ_ERR_STATE, "plan has no device buffers");
    return PRJ_OK;
}

// Stage timing: events around one kernel launch when the plan's record is on.
struct StageTimer {
    prj_plan* pl;
    int stage;
    cudaStream_t st;
    cudaEvent_t t0 = nullptr;
    StageTimer(prj_plan* p, int s, cudaStream_t stream) : pl(p), stage(s), st(stream) {
        if (!pl->timing) return;
        t0 = take();
        if (t0) cudaEventRecord(t0, st);
    }
    cudaEvent_t take() {
        cudaEvent_t e = nullptr;
        if (!pl->event_pool.empty()) {
            e = pl->event_pool.back();
            pl->event_pool.pop_back();
        } else if (cudaEventCreate(&e) != cudaSuccess) {
            e = nullptr;
        }
        return e;
    }
    ~StageTimer() {
        if (!t0) return;
        cudaEvent_t t1 = take();
        if (!t1) { pl->event_pool.push_back(t0); return; }
        cudaEventRecord(t1, st);
        pl->rec.push_back(prj::StageRecord{stage, t0, t1});
    }
};

// Mixed-path set-up on first use: FP64 rows are the x-wavenumbers whose lines
// are badly conditioned, |a_x(kx)| < tau * max_k |b_k| (their condition number
// exceeds about 1/tau; with FP32 storage their error would not contract under
// refinement); kx = 0 (the pinned mean mode) is always FP64.
int ensure_mixed(prj_plan* pl) {
    if (pl->spec32 || pl->kxs_mixed == pl->g.nxh) return PRJ_OK;
    const prj::Geometry& g = pl->g;
    std::vector<double> ax(g.nxh), bands((size_t)6 * g.ny);
    CK(cudaMemcpy(ax.data(), pl->t.ax, ax.size() * sizeof(double), cudaMemcpyDeviceToHost), "mixed set-up");
    CK(cudaMemcpy(bands.data(), pl->t.bands, bands.size() * sizeof(double), cudaMemcpyDeviceToHost), "mixed set-up");
    double bmax = 0.0;
    for (int k = 0; k < g.ny; k++) bmax = std::max(bmax, std::fabs(bands[(size_t)g.ny + k]));
    const double tau = pl->mixed_tau;
    int kxs = g.nxh;
    for (int kx = 1; kx < g.nxh; kx++)
        if (std::fabs(ax[kx]) >= tau * bmax) { kxs = kx; break; }
    pl->kxs_mixed = kxs;
    const size_t n32 = (size_t)(g.nxh - kxs) * g.nz * g.ny;
    if (n32) {
        CK(cudaMalloc((void**)&pl->spec32, n32 * sizeof(float2)), "cudaMalloc(FP32 spectrum)");
        pl->device_bytes += n32 * sizeof(float2);
    }
    if (!pl->pbar) {
        CK(cudaMalloc((void**)&pl->pbar, (size_t)g.ny * sizeof(double)), "cudaMalloc(plane means)");
        pl->device_bytes += (size_t)g.ny * sizeof(double);
    }
    return PRJ_OK;
}

int run_zsolve_mixed(prj_plan* pl, cudaStream_t st) {
    {
        StageTimer tm(pl, prj::kStZfftFwd, st);
        CK(prj::launch_zfft_mixed(pl, -1, st), "z transform");
    }
    {
        StageTimer tm(pl, prj::kStThomas, st);
        CK(prj::launch_thomas_mixed(pl, st), "Thomas sweeps");
    }
    {
        StageTimer tm(pl, prj::kStZfftInv, st);
        CK(prj::launch_zfft_mixed(pl, +1, st), "inverse z transform");
    }
    return PRJ_OK;
}

// inverse x transform that also leaves per-tile sums of P for the next plane means
// (pass-plan kernel); falls back to the plain transform (psum_valid = false)
cudaError_t bwd_with_sums(prj_plan* pl, double* P, cudaStream_t st, int accum, double* sq) {
    // capacity for the current tiling (x_rows may change it); allocated outside any capture
    // because the batched graphs run every case once before capturing
    const size_t need = (size_t)pl->g.ny * prj::bwd_tiles_per_plane(pl);
    if (pl->psum_elems < need) {
        dfree(pl->psum);
        pl->psum = nullptr;
        pl->device_bytes -= pl->psum_elems * sizeof(double);
        pl->psum_elems = 0;
        const cudaError_t e = cudaMalloc((void**)&pl->psum, need * sizeof(double));
        if (e != cudaSuccess) {
            pl->psum = nullptr;
            return e;
        }
        pl->psum_elems = need;
        pl->device_bytes += need * sizeof(double);
    }
    if (pl->psum) {
        const cudaError_t e = prj::launch_bwd_xd(pl, P, st, accum, sq, prj::YRange{}, pl->psum);
        if (e != cudaErrorNotSupported) {
            pl->psum_valid = (e == cudaSuccess);
            return e;
        }
    }
    pl->psum_valid = false;
    return prj::launch_bwd_xd(pl, P, st, accum, sq);
}

// FP32-storage solve with FP64 refinement: p = solve(b); repeat mixed_iters times
// { r = b - A p; p += solve(r) }.  The right-hand side is the divergence of
// (Uh, Vh, Wh) when Uh is given, else the incoming P.  b and r are scratch fields
// of nx nz ny doubles (the projection passes its still unused outputs U and V).
int run_mixed_core(prj_plan* pl, const double* Uh, const double* Vh, const double* Wh, const prj::StepScalars* sc,
                   double* b, double* r, double* P, cudaStream_t st) {
    int rc = ensure_mixed(pl);
    if (rc) return rc;
    struct KxsScope {
        prj_plan* pl;
        int saved;
        KxsScope(prj_plan* p) : pl(p), saved(p->kxs) { pl->kxs = pl->kxs_mixed; }
        ~KxsScope() { pl->kxs = saved; }
    } scope(pl);
    {
        StageTimer tm(pl, prj::kStFwdX, st);
        if (Uh)
            CK(prj::launch_fwd_xd(pl, prj::FwdSource::Divergence, nullptr, Uh, Vh, Wh, sc, st, b), "divergence + forward x");
        else
            CK(prj::launch_fwd_xd(pl, prj::FwdSource::Pressure, P, nullptr, nullptr, nullptr, nullptr, st, b), "forward x");
    }
    if ((rc = run_zsolve_mixed(pl, st))) return rc;
    {
        StageTimer tm(pl, prj::kStBwdX, st);
        CK(bwd_with_sums(pl, P, st, 0, nullptr), "inverse x");
    }
    for (int it = 1; it <= pl->mixed_iters; it++) {
        const bool last = (it == pl->mixed_iters);
        {
            StageTimer tm(pl, prj::kStResidual, st);
            if (pl->psum_valid)
                CK(prj::launch_plane_mean_partials(pl, pl->psum, prj::bwd_tiles_per_plane(pl), pl->pbar, st),
                   "plane means");
            else
                CK(prj::launch_plane_mean(pl, P, pl->pbar, st), "plane means");
        }
        {
            // the residual formed inside the forward x transform (no round trip of r through
            // HBM), or as its own kernel where the x length has no pass plan
            StageTimer tm(pl, prj::kStFwdX, st);
            const cudaError_t e = prj::launch_fwd_residual(pl, b, P, pl->pbar, st);
            if (e == cudaErrorNotSupported) {
                CK(prj::launch_residual(pl, b, P, pl->pbar, r, st), "residual");
                CK(prj::launch_fwd_xd(pl, prj::FwdSource::Pressure, r, nullptr, nullptr, nullptr, nullptr, st),
                   "forward x");
            } else {
                CK(e, "residual + forward x");
            }
        }
        if ((rc = run_zsolve_mixed(pl, st))) return rc;
        if (last) CK(cudaMemsetAsync(pl->stat_buf + 4, 0, 2 * sizeof(double), st), "norm slots");
        {
            StageTimer tm(pl, prj::kStBwdX, st);
            CK(bwd_with_sums(pl, P, st, 1, last ? pl->stat_buf + 4 : nullptr), "inverse x");
        }
    }
    return PRJ_OK;
}

int run_mixed_solve(prj_plan* pl, const double* Uh, const double* Vh, const double* Wh, double* U, double* V,
                    double* P, const prj::StepScalars& sc, cudaStream_t st) {
    return run_mixed_core(pl, Uh, Vh, Wh, &sc, U, V, P, st);
}

int mixed_supported(const prj_plan* pl) {
    if ((pl->zmode != 0 && pl->zmode != 3) || !pl->xd.ok)
        return fail(PRJ_ERR_UNSUPPORTED, "the mixed-precision path needs in-place plans for nx/2 and nz (radices 2, 3, 4, 5, 8)");
    return PRJ_OK;
}

// Poisson-only mixed solve: plan-owned scratch for b and r
int run_mixed_poisson(prj_plan* pl, double* P, cudaStream_t st) {
    int rc = mixed_supported(pl);
    if (rc) return rc;
    const size_t n = (size_t)pl->g.nx * pl->g.nz * pl->g.ny;
    if (!pl->mix_b) {
        CK(cudaMalloc((void**)&pl->mix_b, n * sizeof(double)), "cudaMalloc(mixed scratch)");
        pl->device_bytes += n * sizeof(double);
    }
    if (!pl->mix_r) {
        CK(cudaMalloc((void**)&pl->mix_r, n * sizeof(double)), "cudaMalloc(mixed scratch)");
        pl->device_bytes += n * sizeof(double);
    }
    return run_mixed_core(pl, nullptr, nullptr, nullptr, nullptr, pl->mix_b, pl->mix_r, P, st);
}

// z transforms + Thomas: three kernels (split) or one fused kernel
int run_zsolve(prj_plan* pl, cudaStream_t st) {
    if (pl->zmode == 3) {
        StageTimer tm(pl, prj::kStZSolve, st);
        const cudaError_t e = prj::launch_zline(pl, st);
        if (e != cudaErrorNotSupported) {
            CK(e, "z transform + Thomas (per-wavenumber kernel)");
            return PRJ_OK;
        }
    }
    if (pl->zmode == 0 || pl->zmode == 3) {
        {
            StageTimer tm(pl, prj::kStZfftFwd, st);
            CK(prj::launch_zfft(pl, -1, st), "z transform");
        }
        {
            StageTimer tm(pl, prj::kStThomas, st);
            CK(prj::launch_thomas(pl, st), "Thomas sweeps");
        }
        {
            StageTimer tm(pl, prj::kStZfftInv, st);
            CK(prj::launch_zfft(pl, +1, st), "inverse z transform");
        }
        return PRJ_OK;
    }
    StageTimer tm(pl, prj::kStZSolve, st);
    CK(prj::launch_zsolve(pl, st), "z transform + Thomas");
    return PRJ_OK;
}

int run_poisson(prj_plan* pl, double* d_P, cudaStream_t st) {
    {
        StageTimer tm(pl, prj::kStFwdX, st);
        CK(prj::launch_fwd_x(pl, prj::FwdSource::Pressure, d_P, nullptr, nullptr, nullptr, nullptr, st), "forward x");
    }
    {
        const int rz = run_zsolve(pl, st);
        if (rz) return rz;
    }
    {
        StageTimer tm(pl, prj::kStBwdX, st);
        CK(prj::launch_bwd_x(pl, d_P, st), "inverse x");
    }
    return PRJ_OK;
}

void release_events(prj_plan* pl) {
    for (auto& r : pl->rec) {
        cudaEventDestroy(r.t0);
        cudaEventDestroy(r.t1);
    }
    pl->rec.clear();
    for (auto e : pl->event_pool) cudaEventDestroy(e);
    pl->event_pool.clear();
}

int ensure_host_stage(prj_plan* pl, size_t elems) {
    if (pl->host_stage_elems >= elems) return PRJ_OK;
    dfree(pl->host_stage);
    pl->host_stage_elems = 0;
    CK(cudaMalloc((void**)&pl->host_stage, elems * sizeof(double)), "cudaMalloc(host staging)");
    pl->host_stage_elems = elems;
    return PRJ_OK;
}

// A captured batch: one CUDA graph, one branch (own stream during capture) per case.
struct BatchImpl {
    int device = 0;
    int ncases = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool persistent = false;   // one persistent kernel over a work queue (FP64 cases of the
    prj::BatchKernel bk;       // kernel's pass-plan lengths); else the per-case graph
    int graph_kernels = 0;     // kernel launches per replay of the graph
};

}  // namespace

struct prj_batch : BatchImpl {};

namespace {
void batch_release(prj_batch* b) {
    prj::batchk_free(&b->bk);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}
}  // namespace

int prj::record_error(int code, const char* msg) {
    g_last_error = msg;
    return code;
}

extern "C" {

const char* prj_last_error_string(void) { return g_last_error.c_str(); }

const char* prj_version(void) { return "prj_b200 0.1 (sm_100a)"; }

int prj_bands_from_yu(int ny, const double* yu, int mode, double* a, double* b, double* c, double* a00, double* b00,
                      double* c00) {
    if (ny < 2) return fail(PRJ_ERR_ARG, "ny=%d < 2", ny);
    if (!yu || !a || !b || !c || !a00 || !b00 || !c00) return fail(PRJ_ERR_ARG, "NULL argument");
    for (int i = 0; i < ny; i++)
        if (!(yu[i + 1] > yu[i])) return fail(PRJ_ERR_ARG, "yu must increase strictly (yu[%d] >= yu[%d])", i, i + 1);
    std::vector<double> ext((size_t)ny + 2);  // yp_ext, calc_bands.py:226-227
    ext[0] = yu[0];
    for (int i = 0; i < ny; i++) ext[i + 1] = (yu[i] + yu[i + 1]) / 2;
    ext[ny + 1] = yu[ny];
    if (mode == PRJ_BANDS_REFERENCE) {
        // mk_P_abc, calc_bands.py:181-201 (once plain, once is_dirich_first)
        std::vector<double> pad(ext);
        pad[0] = 2 * ext[0] - ext[1];
        pad[ny + 1] = 2 * ext[ny + 1] - ext[ny];
        for (int pass = 0; pass < 2; pass++) {
            double* A = pass ? a00 : a;
            double* B = pass ? b00 : b;
            double* C = pass ? c00 : c;
            for (int i = 0; i < ny; i++) {
                const double x0 = pad[i], x1 = pad[i + 1], x2 = pad[i + 2];
                const double dy = 0.5 * (x2 - x0);
                A[i] = 1.0 / ((x1 - x0) * dy);
                C[i] = 1.0 / ((x2 - x1) * dy);
                B[i] = -(A[i] + C[i]);
            }
            if (pass) B[0] -= A[0];
            else B[0] += A[0];
            B[ny - 1] += C[ny - 1];
            A[0] = 0.0;
            C[ny - 1] = 0.0;
        }
        return PRJ_OK;
    }
    if (mode == PRJ_BANDS_CONSISTENT) {
        const double* yp = ext.data() + 1;
        for (int k = 0; k < ny; k++) {
            const double idy = 1.0 / (yu[k + 1] - yu[k]);
            a[k] = (k > 0) ? idy / (yp[k] - yp[k - 1]) : 0.0;
            c[k] = (k < ny - 1) ? idy / (yp[k + 1] - yp[k]) : 0.0;
            b[k] = -(a[k] + c[k]);
            a00[k] = a[k];
            b00[k] = b[k];
            c00[k] = c[k];
        }
        const double ghost = 2 * yu[0] - yp[0];  // mirrored ghost, as yp_pad[0] of mk_P_abc
        b00[0] -= 2.0 * (1.0 / (yu[1] - yu[0])) / (yp[0] - ghost);
        return PRJ_OK;
    }
    return fail(PRJ_ERR_ARG, "unknown band mode %d", mode);
}

int prj_metrics_from_yu(int ny, const double* yu, double* inv_dy_p, double* dPdy_lo, double* dPdy_hi) {
    if (ny < 2) return fail(PRJ_ERR_ARG, "ny=%d < 2", ny);
    if (!yu || !inv_dy_p || !dPdy_lo || !dPdy_hi) return fail(PRJ_ERR_ARG, "NULL argument");
    for (int i = 0; i < ny; i++) {
        if (!(yu[i + 1] > yu[i])) return fail(PRJ_ERR_ARG, "yu must increase strictly (yu[%d] >= yu[%d])", i, i + 1);
        inv_dy_p[i] = 1. / (yu[i + 1] - yu[i]);
    }
    dPdy_lo[0] = 0.0;
    dPdy_hi[0] = 0.0;
    for (int i = 1; i < ny; i++) {
        const double dy = (yu[i] + yu[i + 1]) / 2 - (yu[i - 1] + yu[i]) / 2;
        dPdy_lo[i] = -1 / dy;
        dPdy_hi[i] = 1 / dy;
    }
    return PRJ_OK;
}

int prj_plan_create(int nx, int nz, int ny, double dx, double dz, const double* band_a, const double* band_b,
                    const double* band_c, const double* band_a00, const double* band_b00, const double* band_c00,
                    const double* inv_dy_p, const double* dPdy_lo, const double* dPdy_hi, unsigned flags, int device,
                    prj_plan** out) {
    if (!out) return fail(PRJ_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (nx < 1 || nx > 8192) return fail(PRJ_ERR_ARG, "nx=%d outside [1, 8192]", nx);
    if (nz < 1 || nz > 4094) return fail(PRJ_ERR_ARG, "nz=%d outside [1, 4094]", nz);
    if (ny < 2 || ny > 65536) return fail(PRJ_ERR_ARG, "ny=%d outside [2, 65536] (ny_glob < 2 is rejected as in the reference)", ny);
    if (!(dx > 0) || !(dz > 0) || !std::isfinite(dx) || !std::isfinite(dz))
        return fail(PRJ_ERR_ARG, "dx=%g, dz=%g must be finite and positive", dx, dz);
    if (!band_a || !band_b || !band_c || !band_a00 || !band_b00 || !band_c00)
        return fail(PRJ_ERR_ARG, "band pointer is NULL");
    const int nmet = (inv_dy_p != nullptr) + (dPdy_lo != nullptr) + (dPdy_hi != nullptr);
    if (nmet != 0 && nmet != 3) return fail(PRJ_ERR_ARG, "inv_dy_p, dPdy_lo, dPdy_hi must be all set or all NULL");
    if (flags != PRJ_FLAG_NONE) return fail(PRJ_ERR_ARG, "unknown flags 0x%x", flags);
    const double* bandv[6] = {band_a, band_b, band_c, band_a00, band_b00, band_c00};
    for (int i = 0; i < 6; i++)
        if (!finite_all(bandv[i], ny)) return fail(PRJ_ERR_ARG, "band array %d holds a non-finite value", i);
    if (nmet == 3 && (!finite_all(inv_dy_p, ny) || !finite_all(dPdy_lo, ny) || !finite_all(dPdy_hi, ny)))
        return fail(PRJ_ERR_ARG, "a 1-D metric holds a non-finite value");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(PRJ_ERR_CUDA, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(PRJ_ERR_ARG, "device %d outside [0, %d)", device, ndev);
    DeviceGuard dg(device);

    prj_plan* pl = new prj_plan();
    pl->device = device;
    pl->flags = flags;
    pl->has_metrics = (nmet == 3);
    prj::Geometry& g = pl->g;
    g.nx = nx; g.nz = nz; g.ny = ny; g.dx = dx; g.dz = dz;
    g.nxh = nx / 2 + 1;
    g.nzh = nz / 2 + 1;
    g.mzp = (g.nzh + 1) / 2 * 2;
    size_t bytes = 0;
    int rc = PRJ_OK;
    auto bail = [&](int code) {
        free_plan_buffers(pl);
        delete pl;
        return code;
    };
    if ((rc = make_rfft<double>(nx, &pl->fx64, &bytes))) return bail(rc);
    if ((rc = make_cfft<double>(nz, &pl->fz64.f, &pl->fz64.tw, &bytes))) return bail(rc);
    if ((rc = make_dif(pl->fx64.m, &pl->xd, &bytes))) return bail(rc);
    if ((rc = make_dif(nz, &pl->zd, &bytes))) return bail(rc);
    if (pl->zd.ok && (rc = make_slot_table(nz, &pl->kz_of_slot, &bytes))) return bail(rc);
    {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, pl->device) != cudaSuccess) sms = 0;
        pl->zmode = z_mode(pl->zd.ok && pl->kz_of_slot, sms > 0 && g.nxh >= 2 * sms);
    }
    // pass-plan kernels wherever the length has a plan; the Thomas ring for the
    // mixed-storage solve only (prj_tuning.thomas_ring changes it)
    pl->use_pass = true;
    pl->thomas_async = -1;
    pl->kxs = g.nxh;
    pl->tz_xd = prj::choose_tz_xd(pl->fx64.m, pl->fx64.even);
    pl->tz_xp = prj::choose_tz_xp(pl->fx64.m);

    // rows per CTA of the x kernels: fit two ping-pong buffers in ~100 KB
    {
        const size_t per_row = (size_t)2 * (pl->fx64.m + 1) * sizeof(double2);
        int tz = (int)((100 * 1024) / per_row);
        if (tz > 16) tz = 16;
        if (tz < 1) tz = 1;
        if (per_row * tz > 200 * 1024) return bail(fail(PRJ_ERR_UNSUPPORTED, "nx=%d too large for one CTA", nx));
        pl->tz_fwd = tz;
    }

    // wavenumber tables, poisson_solver_multigpu.f90:147-148
    const double const_pi = 4.0 * std::atan(1.0);
    const double inv_dx = 1.0 / dx, inv_dz = 1.0 / dz;
    std::vector<double> ax(g.nxh), az(g.nzh);
    for (int i = 0; i < g.nxh; i++) {
        const double s = std::sin(i * const_pi / nx);
        ax[i] = -4 * (inv_dx * inv_dx) * (s * s);
    }
    for (int j = 0; j < g.nzh; j++) {
        const double s = std::sin(j * const_pi / nz);
        az[j] = -4 * (inv_dz * inv_dz) * (s * s);
    }
    std::vector<double> bands((size_t)6 * ny);
    for (int i = 0; i < 6; i++) std::memcpy(&bands[(size_t)i * ny], bandv[i], sizeof(double) * ny);

    auto up = [&](double** d, const double* h, size_t n, const char* what) -> int {
        cudaError_t e = cudaMalloc((void**)d, n * sizeof(double));
        if (e != cudaSuccess) return cuda_fail(e, what);
        bytes += n * sizeof(double);
        e = cudaMemcpy(*d, h, n * sizeof(double), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(e, what);
        return PRJ_OK;
    };
    if ((rc = up(&pl->t.bands, bands.data(), bands.size(), "bands"))) return bail(rc);
    if ((rc = up(&pl->t.ax, ax.data(), ax.size(), "a_x"))) return bail(rc);
    if ((rc = up(&pl->t.az, az.data(), az.size(), "a_z"))) return bail(rc);
    if (pl->has_metrics) {
        if ((rc = up(&pl->t.inv_dy_p, inv_dy_p, ny, "inv_dy_p"))) return bail(rc);
        if ((rc = up(&pl->t.dpdy_lo, dPdy_lo, ny, "dPdy_lo"))) return bail(rc);
        if ((rc = up(&pl->t.dpdy_hi, dPdy_hi, ny, "dPdy_hi"))) return bail(rc);
    }
    const size_t spec_elems = (size_t)ny * g.nxh * nz;
    const size_t piv_elems = (size_t)ny * g.nxh * g.mzp;
    cudaError_t e;
    if ((e = cudaMalloc((void**)&pl->spec, spec_elems * sizeof(double2))) != cudaSuccess)
        return bail(cuda_fail(e, "cudaMalloc(spectrum)"));
    bytes += spec_elems * sizeof(double2);
    if ((e = cudaMalloc((void**)&pl->t.piv, piv_elems * sizeof(double))) != cudaSuccess)
        return bail(cuda_fail(e, "cudaMalloc(pivots)"));
    bytes += piv_elems * sizeof(double);
    if ((e = cudaMalloc((void**)&pl->t.pivc, piv_elems * sizeof(double))) != cudaSuccess)
        return bail(cuda_fail(e, "cudaMalloc(back-substitution factors)"));
    bytes += piv_elems * sizeof(double);
    if ((e = cudaMalloc((void**)&pl->stat_buf, 8 * sizeof(double))) != cudaSuccess)
        return bail(cuda_fail(e, "cudaMalloc(stats)"));
    bytes += 8 * sizeof(double);
    if ((e = cudaMemset(pl->stat_buf, 0, 8 * sizeof(double))) != cudaSuccess)
        return bail(cuda_fail(e, "cudaMemset(stats)"));
    if ((e = prj::launch_build_pivots(pl, 0)) != cudaSuccess) return bail(cuda_fail(e, "pivot table"));
    double mm[2] = {0, 0};
    if ((e = cudaMemcpy(mm, pl->stat_buf, sizeof(mm), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return bail(cuda_fail(e, "pivot table"));
    const double mp = mm[0];
    pl->min_pivot = mp;
    if (!(mp > 0) || !std::isfinite(mp))
        return bail(fail(PRJ_ERR_NUMERIC, "zero or non-finite Thomas pivot (min_abs_div_bacp = %g)", mp));
    if (!(mp >= prj::kDivRecipMinD) || !(mm[1] <= prj::kDivRecipMaxD))
        return bail(fail(PRJ_ERR_NUMERIC,
                         "Thomas pivots |D| in [%g, %g] leave the range [2^-40, 2^1000] of the forward sweeps' "
                         "correctly rounded division (a nearly singular wall-normal operator)",
                         mp, mm[1]));
    pl->device_bytes = bytes;
    *out = pl;
    return PRJ_OK;
}

int prj_plan_destroy(prj_plan* plan) {
    if (!plan) return PRJ_OK;
    DeviceGuard dg(plan->device);
    cudaDeviceSynchronize();
    release_events(plan);
    free_plan_buffers(plan);
    delete plan;
    return PRJ_OK;
}

int prj_plan_min_pivot(const prj_plan* plan, double* out) {
    if (!plan || !out) return fail(PRJ_ERR_ARG, "NULL argument");
    *out = plan->min_pivot;
    return PRJ_OK;
}

int prj_plan_check_error(prj_plan* plan, void* stream) {
    int rc = check_plan(plan);
    if (rc) return rc;
    DeviceGuard dg(plan->device);
    cudaStream_t st = (cudaStream_t)stream;
    int* word = reinterpret_cast<int*>(plan->stat_buf + prj::kStatErrSlot);
    int dev_err = 0;
    CK(cudaMemcpyAsync(&dev_err, word, sizeof(int), cudaMemcpyDeviceToHost, st), "error word copy");
    CK(cudaMemsetAsync(word, 0, sizeof(int), st), "error word reset");
    CK(cudaStreamSynchronize(st), "error word sync");
    if (dev_err) return fail(PRJ_ERR_TIMEOUT, "a bounded device-side wait gave up (code %d)", dev_err);
    return PRJ_OK;
}

int prj_plan_device_bytes(const prj_plan* plan, size_t* out) {
    if (!plan || !out) return fail(PRJ_ERR_ARG, "NULL argument");
    *out = plan->device_bytes + plan->host_stage_elems * sizeof(double);
    return PRJ_OK;
}

int prj_plan_enable_stage_timing(prj_plan* plan, int enable) {
    int rc = check_plan(plan);
    if (rc) return rc;
    plan->timing = enable != 0;
    return PRJ_OK;
}

int prj_plan_stage_times(prj_plan* plan, double* ms, int* launches, int max_stages, int* n_stages) {
    int rc = check_plan(plan);
    if (rc) return rc;
    if (!ms || !launches || max_stages <= 0) return fail(PRJ_ERR_ARG, "NULL or empty output");
    DeviceGuard dg(plan->device);
    for (int i = 0; i < max_stages; i++) { ms[i] = 0.0; launches[i] = 0; }
    int top = 0;
    cudaError_t err = cudaSuccess;
    for (auto& r : plan->rec) {
        float t = 0.f;
        cudaError_t e = cudaEventSynchronize(r.t1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&t, r.t0, r.t1);
        if (e != cudaSuccess && err == cudaSuccess) err = e;
        if (r.stage < max_stages) {
            ms[r.stage] += t;
            launches[r.stage] += 1;
            if (r.stage + 1 > top) top = r.stage + 1;
        }
        plan->event_pool.push_back(r.t0);
        plan->event_pool.push_back(r.t1);
    }
    plan->rec.clear();
    if (n_stages) *n_stages = top;
    if (err != cudaSuccess) return cuda_fail(err, "stage timing");
    return PRJ_OK;
}

const char* prj_stage_name(int stage) {
    switch (stage) {
    case prj::kStFwdX: return "k_fwd_x";
    case prj::kStZSolve: return "k_zsolve";
    case prj::kStBwdX: return "k_bwd_x";
    case prj::kStCorrect: return "k_correct";
    case prj::kStStats: return "k_stats";
    case prj::kStZfftFwd: return "k_zfft_fwd";
    case prj::kStThomas: return "k_thomas";
    case prj::kStZfftInv: return "k_zfft_inv";
    case prj::kStResidual: return "k_residual";
    case prj::kStVdRhs: return "k_vd_rhs";
    case prj::kStVdPrep: return "k_rho_prep";
    default: return "";
    }
}

int prj_poisson_fp64(prj_plan* plan, double* d_P, void* stream) {
    int rc = check_plan(plan);
    if (rc) return rc;
    if (!d_P) return fail(PRJ_ERR_ARG, "P is NULL");
    DeviceGuard dg(plan->device);
    return run_poisson(plan, d_P, (cudaStream_t)stream);
}

bool x_pass_active(const prj_plan* pl);

int prj_projection_step(prj_plan* plan, const double* d_Uh, const double* d_Vh, const double* d_Wh, double* d_U,
                        double* d_V, double* d_W, double* d_P, const prj_step_params* params, int mode,
                        prj_stats* stats, void* stream) {
    int rc = check_plan(plan);
    if (rc) return rc;
    if (!plan->has_metrics) return fail(PRJ_ERR_STATE, "plan was created without inv_dy_p / dPdy (Poisson-only)");
    if (!d_Uh || !d_Vh || !d_Wh || !d_U || !d_V || !d_W || !d_P || !params)
        return fail(PRJ_ERR_ARG, "NULL array or params");
    if (!(params->dt > 0) || !std::isfinite(params->dt)) return fail(PRJ_ERR_ARG, "dt=%g must be finite and positive", params->dt);
    if (mode != PRJ_MODE_FP64 && mode != PRJ_MODE_FP32_REFINE) return fail(PRJ_ERR_ARG, "unknown mode %d", mode);
    if (mode == PRJ_MODE_FP32_REFINE && (rc = mixed_supported(plan))) return rc;
    if (d_U == d_Uh || d_V == d_Vh || d_W == d_Wh || d_U == d_Vh || d_U == d_Wh || d_V == d_Uh || d_V == d_Wh)
        return fail(PRJ_ERR_ARG, "output velocity arrays must not alias the predictor arrays");
    DeviceGuard dg(plan->device);
    cudaStream_t st = (cudaStream_t)stream;
    prj::StepScalars sc{};
    sc.dt = params->dt;
    sc.inv_dt = 1.0 / params->dt;
    sc.wall[0] = params->wall_U_bot; sc.wall[1] = params->wall_V_bot; sc.wall[2] = params->wall_W_bot;
    sc.wall[3] = params->wall_U_top; sc.wall[4] = params->wall_V_top; sc.wall[5] = params->wall_W_top;
    if (mode == PRJ_MODE_FP32_REFINE) {
        const int rm = run_mixed_solve(plan, d_Uh, d_Vh, d_Wh, d_U, d_V, d_P, sc, st);
        if (rm) return rm;
    } else {
        {
            StageTimer tm(plan, prj::kStFwdX, st);
            CK(prj::launch_fwd_x(plan, prj::FwdSource::Divergence, nullptr, d_Uh, d_Vh, d_Wh, &sc, st), "divergence + forward x");
        }
        {
            const int rz = run_zsolve(plan, st);
            if (rz) return rz;
        }
        {
            StageTimer tm(plan, prj::kStBwdX, st);
            CK(prj::launch_bwd_x(plan, d_P, st), "inverse x");
        }
    }
    {
        StageTimer tm(plan, prj::kStCorrect, st);
        CK(prj::launch_correction(plan, d_P, d_Uh, d_Vh, d_Wh, d_U, d_V, d_W, sc, st), "correction");
    }
    if (stats || params->compute_stats) {
        {
            StageTimer tm(plan, prj::kStStats, st);
            CK(prj::launch_stats(plan, d_U, d_V, d_W, d_P, plan->stat_buf + 2, st), "stats");
        }
        double h[5] = {-1, -1, 0, 0, 0};
        CK(cudaMemcpyAsync(h, plan->stat_buf + 2, 5 * sizeof(double), cudaMemcpyDeviceToHost, st), "stats copy");
        CK(cudaStreamSynchronize(st), "stats sync");
        int dev_err = 0;
        std::memcpy(&dev_err, &h[prj::kStatErrSlot - 2], sizeof(int));
        if (dev_err) {  // reported once: the word is cleared for the next check
            cudaMemsetAsync(plan->stat_buf + prj::kStatErrSlot, 0, sizeof(int), st);
            return fail(PRJ_ERR_TIMEOUT, "a bounded device-side wait gave up (code %d)", dev_err);
        }
        if (stats) {
            stats->div_maxabs = h[0];
            stats->p_maxabs = h[1];
            stats->min_pivot = plan->min_pivot;
            stats->rho_min = 0.0;
            if (mode == PRJ_MODE_FP32_REFINE) {
                stats->refine_iters = plan->mixed_iters;
                stats->fp64_lines = plan->kxs_mixed * plan->g.nz;
                stats->last_update_rel = (h[3] > 0) ? std::sqrt(h[2] / h[3]) : 0.0;
            } else {
                stats->refine_iters = 0;
                stats->fp64_lines = plan->g.nxh * plan->g.nz;
                stats->last_update_rel = 0.0;
            }
        }
        if (!std::isfinite(h[0]) || !std::isfinite(h[1])) return fail(PRJ_ERR_NUMERIC, "NaN detected in the projection");
    }
    return PRJ_OK;
}

int prj_vd_metric_from_yu(int ny, const double* yu, double* inv_dy_p_pad) {
    if (ny < 2 || !yu || !inv_dy_p_pad) return fail(PRJ_ERR_ARG, "need ny >= 2 and non-NULL arrays");
    // yp_pad = [2 yu_0 - yp_0, yp_0 .. yp_{ny-1}, 2 yu_ny - yp_{ny-1}], calc_bands.py:273, :276
    std::vector<double> yp((size_t)ny + 2);
    for (int k = 0; k < ny; k++) yp[(size_t)k + 1] = (yu[k] + yu[k + 1]) / 2;
    yp[0] = 2 * yu[0] - yp[1];
    yp[(size_t)ny + 1] = 2 * yu[ny] - yp[(size_t)ny];
    for (int i = 0; i <= ny; i++) inv_dy_p_pad[i] = 1. / (yp[(size_t)i + 1] - yp[(size_t)i]);
    return PRJ_OK;
}

int prj_plan_set_vd_metric(prj_plan* plan, const double* inv_dy_p_pad) {
    int rc = check_plan(plan);
    if (rc) return rc;
    if (!inv_dy_p_pad) return fail(PRJ_ERR_ARG, "inv_dy_p_pad is NULL");
    for (int i = 0; i <= plan->g.ny; i++)
        if (!std::isfinite(inv_dy_p_pad[i])) return fail(PRJ_ERR_ARG, "inv_dy_p_pad[%d] is not finite", i);
    DeviceGuard dg(plan->device);
    const size_t bytes = (size_t)(plan->g.ny + 1) * sizeof(double);
    if (!plan->vd_pad) {
        CK(cudaMalloc((void**)&plan->vd_pad, bytes), "cudaMalloc(inv_dy_p_pad)");
        plan->device_bytes += bytes;
    }
    CK(cudaMemcpy(plan->vd_pad, inv_dy_p_pad, bytes, cudaMemcpyHostToDevice), "cudaMemcpy(inv_dy_p_pad)");
    return PRJ_OK;
}

int prj_projection_step_vd(prj_plan* plan, const double* d_Uh, const double* d_Vh, const double* d_Wh, double* d_U,
                           double* d_V, double* d_W, double* d_P, const prj_step_params* params,
                           const prj_vd_fields* vd, int mode, prj_stats* stats, void* stream) {
    int rc = check_plan(plan);
    if (rc) return rc;
    if (!plan->has_metrics) return fail(PRJ_ERR_STATE, "plan was created without inv_dy_p / dPdy (Poisson-only)");
    if (!plan->vd_pad) return fail(PRJ_ERR_STATE, "no inv_dy_p_pad: call prj_plan_set_vd_metric first");
    if (!d_Uh || !d_Vh || !d_Wh || !d_U || !d_V || !d_W || !d_P || !params || !vd)
        return fail(PRJ_ERR_ARG, "NULL array, params or fields");
    if (!vd->rho || !vd->P_now || !vd->P_old || !vd->div_now || !vd->P_next)
        return fail(PRJ_ERR_ARG, "NULL variable-density field");
    if (!(params->dt > 0) || !std::isfinite(params->dt)) return fail(PRJ_ERR_ARG, "dt=%g must be finite and positive", params->dt);
    if (mode != PRJ_MODE_FP64 && mode != PRJ_MODE_FP32_REFINE) return fail(PRJ_ERR_ARG, "unknown mode %d", mode);
    if (mode == PRJ_MODE_FP32_REFINE && (rc = mixed_supported(plan))) return rc;
    {
        const void* outs[5] = {d_U, d_V, d_W, d_P, vd->P_next};
        const void* ins[7] = {d_Uh, d_Vh, d_Wh, vd->rho, vd->P_now, vd->P_old, vd->div_now};
        for (const void* o : outs) {
            for (const void* in : ins)
                if (o == in) return fail(PRJ_ERR_ARG, "an output array aliases an input array");
        }
        for (int a = 0; a < 5; a++)
            for (int b = a + 1; b < 5; b++)
                if (outs[a] == outs[b]) return fail(PRJ_ERR_ARG, "two output arrays alias");
    }
    DeviceGuard dg(plan->device);
    cudaStream_t st = (cudaStream_t)stream;
    prj::StepScalars sc{};
    sc.dt = params->dt;
    sc.inv_dt = 1.0 / params->dt;
    sc.wall[0] = params->wall_U_bot; sc.wall[1] = params->wall_V_bot; sc.wall[2] = params->wall_W_bot;
    sc.wall[3] = params->wall_U_top; sc.wall[4] = params->wall_V_top; sc.wall[5] = params->wall_W_top;
    const prj::VdFields f{vd->rho, vd->P_now, vd->P_old, vd->div_now, vd->P_next};
    unsigned long long* slot = reinterpret_cast<unsigned long long*>(plan->stat_buf + prj::kStatRhoSlot);
    if (!plan->vd_ih) {
        const size_t nh = (size_t)(plan->g.nx + 2) * (plan->g.nz + 2) * (plan->g.ny + 2);
        CK(cudaMalloc((void**)&plan->vd_ih, nh * sizeof(double)), "cudaMalloc(0.5 / rho)");
        plan->device_bytes += nh * sizeof(double);
    }
    {
        StageTimer tm(plan, prj::kStVdPrep, st);
        CK(prj::launch_vd_prep(plan, vd->rho, plan->vd_ih, slot, st), "rho_min and 0.5 / rho");
    }
    {
        StageTimer tm(plan, prj::kStVdRhs, st);
        CK(prj::launch_vd_rhs(plan, d_Uh, d_Vh, d_Wh, f, sc, slot, d_P, st), "variable-density right-hand side");
    }
    if (mode == PRJ_MODE_FP32_REFINE) {
        if ((rc = run_mixed_poisson(plan, d_P, st))) return rc;
    } else if ((rc = run_poisson(plan, d_P, st))) {
        return rc;
    }
    {
        StageTimer tm(plan, prj::kStCorrect, st);
        CK(prj::launch_vd_correction(plan, d_P, d_Uh, d_Vh, d_Wh, f, sc, slot, d_U, d_V, d_W, st),
           "variable-density correction");
    }
    if (stats || params->compute_stats) {
        {
            StageTimer tm(plan, prj::kStStats, st);
            CK(prj::launch_stats(plan, d_U, d_V, d_W, d_P, plan->stat_buf + 2, st), "stats");
        }
        double h[6] = {-1, -1, 0, 0, 0, 0};
        CK(cudaMemcpyAsync(h, plan->stat_buf + 2, 6 * sizeof(double), cudaMemcpyDeviceToHost, st), "stats copy");
        CK(cudaStreamSynchronize(st), "stats sync");
        int dev_err = 0;
        std::memcpy(&dev_err, &h[prj::kStatErrSlot - 2], sizeof(int));
        if (dev_err) {  // reported once: the word is cleared for the next check
            cudaMemsetAsync(plan->stat_buf + prj::kStatErrSlot, 0, sizeof(int), st);
            return fail(PRJ_ERR_TIMEOUT, "a bounded device-side wait gave up (code %d)", dev_err);
        }
        unsigned long long ord = 0;
        std::memcpy(&ord, &h[prj::kStatRhoSlot - 2], sizeof(ord));
        const double rmin = prj::vd_rho_min_host(ord);
        if (stats) {
            stats->div_maxabs = h[0];
            stats->p_maxabs = h[1];
            stats->min_pivot = plan->min_pivot;
            stats->refine_iters = mode == PRJ_MODE_FP32_REFINE ? plan->mixed_iters : 0;
            stats->fp64_lines = (mode == PRJ_MODE_FP32_REFINE ? plan->kxs_mixed : plan->g.nxh) * plan->g.nz;
            stats->last_update_rel = (mode == PRJ_MODE_FP32_REFINE && h[3] > 0) ? std::sqrt(h[2] / h[3]) : 0.0;
            stats->rho_min = rmin;
        }
        if (!(rmin > 0)) return fail(PRJ_ERR_NUMERIC, "rho_min=%g must be positive", rmin);
        if (!std::isfinite(h[0]) || !std::isfinite(h[1])) return fail(PRJ_ERR_NUMERIC, "NaN detected in the projection");
    }
    return PRJ_OK;
}

int prj_poisson_fp64_host(prj_plan* plan, double* h_P) {
    int rc = check_plan(plan);
    if (rc) return rc;
    if (!h_P) return fail(PRJ_ERR_ARG, "P is NULL");
    DeviceGuard dg(plan->device);
    const size_t n = (size_t)plan->g.nx * plan->g.nz * plan->g.ny;
    if ((rc = ensure_host_stage(plan, n))) return rc;
    double* d = plan->host_stage;
    CK(cudaMemcpy(d, h_P, n * sizeof(double), cudaMemcpyHostToDevice), "copy P to device");
    if ((rc = run_poisson(plan, d, 0))) return rc;
    CK(cudaMemcpy(h_P, d, n * sizeof(double), cudaMemcpyDeviceToHost), "copy P to host");
    return PRJ_OK;
}

int prj_projection_step_host(prj_plan* plan, const double* h_Uh, const double* h_Vh, const double* h_Wh, double* h_U,
                             double* h_V, double* h_W, double* h_P, const prj_step_params* params, int mode,
                             prj_stats* stats) {
    int rc = check_plan(plan);
    if (rc) return rc;
    if (!h_Uh || !h_Vh || !h_Wh || !h_U || !h_V || !h_W || !h_P || !params) return fail(PRJ_ERR_ARG, "NULL argument");
    DeviceGuard dg(plan->device);
    const prj::Geometry& g = plan->g;
    const size_t nh = (size_t)(g.nx + 2) * (g.nz + 2) * (g.ny + 2);
    const size_t np = (size_t)g.nx * g.nz * g.ny;
    if ((rc = ensure_host_stage(plan, 6 * nh + np))) return rc;
    double* d = plan->host_stage;
    double *dUh = d, *dVh = d + nh, *dWh = d + 2 * nh, *dU = d + 3 * nh, *dV = d + 4 * nh, *dW = d + 5 * nh,
           *dP = d + 6 * nh;
    CK(cudaMemcpy(dUh, h_Uh, nh * sizeof(double), cudaMemcpyHostToDevice), "copy Uh");
    CK(cudaMemcpy(dVh, h_Vh, nh * sizeof(double), cudaMemcpyHostToDevice), "copy Vh");
    CK(cudaMemcpy(dWh, h_Wh, nh * sizeof(double), cudaMemcpyHostToDevice), "copy Wh");
    if ((rc = prj_projection_step(plan, dUh, dVh, dWh, dU, dV, dW, dP, params, mode, stats, 0))) return rc;
    CK(cudaMemcpy(h_U, dU, nh * sizeof(double), cudaMemcpyDeviceToHost), "copy U");
    CK(cudaMemcpy(h_V, dV, nh * sizeof(double), cudaMemcpyDeviceToHost), "copy V");
    CK(cudaMemcpy(h_W, dW, nh * sizeof(double), cudaMemcpyDeviceToHost), "copy W");
    CK(cudaMemcpy(h_P, dP, np * sizeof(double), cudaMemcpyDeviceToHost), "copy P");
    return PRJ_OK;
}

int prj_projection_step_host_async(prj_plan* plan, const double* h_Uh, const double* h_Vh, const double* h_Wh,
                                   double* h_U, double* h_V, double* h_W, double* h_P,
                                   const prj_step_params* params, int mode) {
    int rc = check_plan(plan);
    if (rc) return rc;
    if (!h_Uh || !h_Vh || !h_Wh || !h_U || !h_V || !h_W || !h_P || !params) return fail(PRJ_ERR_ARG, "NULL argument");
    DeviceGuard dg(plan->device);
    const prj::Geometry& g = plan->g;
    const size_t nh = (size_t)(g.nx + 2) * (g.nz + 2) * (g.ny + 2);
    const size_t np = (size_t)g.nx * g.nz * g.ny;
    const size_t elems = 6 * nh + np;
    if (plan->hp_elems < elems) {
        for (cudaStream_t hs : plan->hp_st)
            if (hs) CK(cudaStreamSynchronize(hs), "pipeline drain");
        for (double*& hb : plan->hp_stage) {
            dfree(hb);
            CK(cudaMalloc((void**)&hb, elems * sizeof(double)), "cudaMalloc(pipeline staging)");
        }
        plan->hp_elems = elems;
    }
    for (cudaStream_t& hs : plan->hp_st)
        if (!hs) CK(cudaStreamCreateWithFlags(&hs, cudaStreamNonBlocking), "pipeline stream");
    for (cudaEvent_t& he : plan->hp_ev)
        if (!he) CK(cudaEventCreateWithFlags(&he, cudaEventDisableTiming), "pipeline event");
    const int k = (int)(plan->hp_n & 1);
    cudaStream_t sin = plan->hp_st[0], scmp = plan->hp_st[1], sout = plan->hp_st[2];
    cudaEvent_t in_done = plan->hp_ev[k], cmp_done = plan->hp_ev[2 + k], out_done = plan->hp_ev[4 + k];
    double* d = plan->hp_stage[k];
    double *dUh = d, *dVh = d + nh, *dWh = d + 2 * nh, *dU = d + 3 * nh, *dV = d + 4 * nh, *dW = d + 5 * nh,
           *dP = d + 6 * nh;
    // copy-in: the slot's inputs are free once its previous solve is done
    CK(cudaStreamWaitEvent(sin, cmp_done, 0), "pipeline order");
    CK(cudaMemcpyAsync(dUh, h_Uh, nh * sizeof(double), cudaMemcpyHostToDevice, sin), "copy Uh");
    CK(cudaMemcpyAsync(dVh, h_Vh, nh * sizeof(double), cudaMemcpyHostToDevice, sin), "copy Vh");
    CK(cudaMemcpyAsync(dWh, h_Wh, nh * sizeof(double), cudaMemcpyHostToDevice, sin), "copy Wh");
    CK(cudaEventRecord(in_done, sin), "pipeline event");
    // solve: after the inputs, and after the slot's previous outputs were read out
    CK(cudaStreamWaitEvent(scmp, in_done, 0), "pipeline order");
    CK(cudaStreamWaitEvent(scmp, out_done, 0), "pipeline order");
    prj_step_params p = *params;
    p.compute_stats = 0;
    if ((rc = prj_projection_step(plan, dUh, dVh, dWh, dU, dV, dW, dP, &p, mode, nullptr, scmp))) return rc;
    CK(cudaEventRecord(cmp_done, scmp), "pipeline event");
    // copy-out
    CK(cudaStreamWaitEvent(sout, cmp_done, 0), "pipeline order");
    CK(cudaMemcpyAsync(h_U, dU, nh * sizeof(double), cudaMemcpyDeviceToHost, sout), "copy U");
    CK(cudaMemcpyAsync(h_V, dV, nh * sizeof(double), cudaMemcpyDeviceToHost, sout), "copy V");
    CK(cudaMemcpyAsync(h_W, dW, nh * sizeof(double), cudaMemcpyDeviceToHost, sout), "copy W");
    CK(cudaMemcpyAsync(h_P, dP, np * sizeof(double), cudaMemcpyDeviceToHost, sout), "copy P");
    CK(cudaEventRecord(out_done, sout), "pipeline event");
    plan->hp_n++;
    return PRJ_OK;
}

int prj_host_async_wait(prj_plan* plan) {
    int rc = check_plan(plan);
    if (rc) return rc;
    DeviceGuard dg(plan->device);
    for (cudaStream_t hs : plan->hp_st)
        if (hs) CK(cudaStreamSynchronize(hs), "pipeline wait");
    return PRJ_OK;
}

int prj_poisson_mixed(prj_plan* plan, double* d_P, void* stream) {
    int rc = check_plan(plan);
    if (rc) return rc;
    if (!d_P) return fail(PRJ_ERR_ARG, "P is NULL");
    DeviceGuard dg(plan->device);
    return run_mixed_poisson(plan, d_P, (cudaStream_t)stream);
}

// true when the x transforms run the pass-plan kernels (even nx, m = nx/2 with a plan)
bool x_pass_active(const prj_plan* pl) {
    int fac[8];
    return pl->use_pass && pl->fx64.even && pl->xd.ok && prj::pass_radices(pl->fx64.m, fac, 8) > 0;
}

int prj_plan_schedule(const prj_plan* plan, int mode, int* launches) {
    if (!plan || !launches) return fail(PRJ_ERR_ARG, "NULL argument");
    if (mode == PRJ_MODE_FP64) {
        const bool one_z = (plan->zmode == 1 || plan->zmode == 2) || (plan->zmode == 3 && prj::zline_supported(plan));
        *launches = one_z ? 4 : 6;
    } else {
        // forward x, z transforms of the FP64 and FP32 rows, one Thomas launch, inverse z of both,
        // inverse x; per refinement pass also the plane means and a norm reset, and the
        // residual where the forward x transform does not form it (no pass plan for nx/2);
        // then the correction
        const int solve = 1 + 2 + 1 + 2 + 1;
        *launches = solve + plan->mixed_iters * (solve + (x_pass_active(plan) ? 2 : 3)) + 1;
    }
    return PRJ_OK;
}

int prj_plan_get_tuning(const prj_plan* plan, prj_tuning* out) {
    if (!plan || !out) return fail(PRJ_ERR_ARG, "NULL argument");
    out->x_rows = x_pass_active(plan) ? plan->tz_xp : plan->tz_xd;
    out->z_rows = plan->zfft_rows;
    out->z_mode = plan->zmode;
    out->z_planes = plan->z_planes;
    out->z_stages = plan->z_stages;
    out->thomas_ring = plan->thomas_async;
    out->mixed_iters = plan->mixed_iters;
    out->mixed_tau = plan->mixed_tau;
    out->x_order = plan->x_order;
    out->z_order = plan->z_order;
    return PRJ_OK;
}

// rebuilds the in-place x or z transform tables in another radix order (z: with its slot
// table); the old tables are freed once the device is idle
int reorder_dif(prj_plan* pl, bool x_axis, int order) {
    const int n = x_axis ? pl->fx64.m : pl->g.nz;
    prj::DifFft fresh{};
    size_t bytes = 0;
    int* kz = nullptr;
    int rc = make_dif(n, &fresh, &bytes, order);
    if (!rc && !x_axis && fresh.ok) rc = make_slot_table(n, &kz, &bytes, order);
    if (rc || !fresh.ok) {
        dfree(fresh.tw);
        dfree(fresh.pos);
        dfree(kz);
        return rc ? rc : fail(PRJ_ERR_UNSUPPORTED, "no in-place plan of length %d in radix order %d", n, order);
    }
    cudaDeviceSynchronize();
    prj::DifFft& d = x_axis ? pl->xd : pl->zd;
    const size_t old = (size_t)prj::dif_twiddle_count(d.f) * sizeof(double2) + (size_t)n * sizeof(int) +
                       (x_axis ? 0 : (size_t)n * sizeof(int));
    dfree(d.tw);
    dfree(d.pos);
    d = fresh;
    if (!x_axis) {
        dfree(pl->kz_of_slot);
        pl->kz_of_slot = kz;
    }
    pl->device_bytes += bytes;
    pl->device_bytes -= std::min(old, pl->device_bytes);
    (x_axis ? pl->x_order : pl->z_order) = order;
    return PRJ_OK;
}

int prj_plan_set_tuning(prj_plan* plan, const prj_tuning* t) {
    int rc = check_plan(plan);
    if (rc) return rc;
    if (!t) return fail(PRJ_ERR_ARG, "NULL tuning");
    auto pow2 = [](int v) { return v >= 1 && v <= 16 && (v & (v - 1)) == 0; };
    if (!pow2(t->x_rows)) return fail(PRJ_ERR_ARG, "x_rows=%d must be a power of two in [1, 16]", t->x_rows);
    if (t->z_rows != 0 && !pow2(t->z_rows)) return fail(PRJ_ERR_ARG, "z_rows=%d must be 0 or a power of two in [1, 16]", t->z_rows);
    if (t->z_mode < 0 || t->z_mode > 3) return fail(PRJ_ERR_ARG, "z_mode=%d must be 0, 1, 2 or 3", t->z_mode);
    if ((t->z_mode == 0 || t->z_mode == 3) && !(plan->zd.ok && plan->kz_of_slot))
        return fail(PRJ_ERR_UNSUPPORTED, "no in-place z plan for nz=%d", plan->g.nz);
    if (t->z_planes < 0 || t->z_planes > 64) return fail(PRJ_ERR_ARG, "z_planes=%d must lie in [0, 64]", t->z_planes);
    if (t->z_stages != 0 && (t->z_stages < 2 || t->z_stages > (t->z_mode == 1 ? 8 : 4)))
        return fail(PRJ_ERR_ARG, "z_stages=%d must be 0 or in [2, %d]", t->z_stages, t->z_mode == 1 ? 8 : 4);
    if (t->thomas_ring < -1 || t->thomas_ring > 4) return fail(PRJ_ERR_ARG, "thomas_ring=%d must lie in [-1, 4]", t->thomas_ring);
    if (t->mixed_iters < 0 || t->mixed_iters > 8) return fail(PRJ_ERR_ARG, "mixed_iters=%d must lie in [0, 8]", t->mixed_iters);
    if (!(t->mixed_tau > 0.0 && t->mixed_tau < 1.0)) return fail(PRJ_ERR_ARG, "mixed_tau=%g must lie in (0, 1)", t->mixed_tau);
    const int nxo = std::max(1, prj::pass_orders(plan->fx64.m)), nzo = std::max(1, prj::pass_orders(plan->g.nz));
    if (t->x_order < 0 || t->x_order >= nxo)
        return fail(PRJ_ERR_ARG, "x_order=%d: length %d has %d compiled radix order(s)", t->x_order, plan->fx64.m, nxo);
    if (t->z_order < 0 || t->z_order >= nzo)
        return fail(PRJ_ERR_ARG, "z_order=%d: length %d has %d compiled radix order(s)", t->z_order, plan->g.nz, nzo);
    const int rs = plan->fx64.even ? plan->fx64.m + 1 : plan->fx64.m;
    if ((size_t)prj::padded_len(t->x_rows * rs, true) * sizeof(double2) + (size_t)plan->fx64.m * sizeof(int) > 200 * 1024)
        return fail(PRJ_ERR_ARG, "x_rows=%d does not fit shared memory for nx=%d", t->x_rows, plan->g.nx);
    if (t->z_rows && (size_t)prj::padded_len(t->z_rows * plan->g.nz, true) * sizeof(double2) > 200 * 1024)
        return fail(PRJ_ERR_ARG, "z_rows=%d does not fit shared memory for nz=%d", t->z_rows, plan->g.nz);
    DeviceGuard dg(plan->device);
    if (t->x_order != plan->x_order && plan->xd.ok && (rc = reorder_dif(plan, true, t->x_order))) return rc;
    if (t->z_order != plan->z_order && plan->zd.ok && (rc = reorder_dif(plan, false, t->z_order))) return rc;
    if (t->mixed_tau != plan->mixed_tau && (plan->spec32 || plan->kxs_mixed)) {
        // the FP64 row count follows mixed_tau: the mixed set-up runs again at the next mixed call
        cudaDeviceSynchronize();
        if (plan->spec32) {
            const size_t n32 = (size_t)(plan->g.nxh - plan->kxs_mixed) * plan->g.nz * plan->g.ny;
            dfree(plan->spec32);
            plan->spec32 = nullptr;
            plan->device_bytes -= n32 * sizeof(float2);
        }
        plan->kxs_mixed = 0;
    }
    plan->tz_xd = t->x_rows;
    plan->tz_xp = t->x_rows;
    plan->zfft_rows = t->z_rows;
    plan->zmode = t->z_mode;
    plan->z_planes = t->z_planes;
    plan->z_stages = t->z_stages;
    plan->thomas_async = t->thomas_ring;
    plan->mixed_iters = t->mixed_iters;
    plan->mixed_tau = t->mixed_tau;
    return PRJ_OK;
}

int prj_batch_create(prj_plan* const* plans, double* const* d_P, int ncases, int mode, prj_batch** out) {
    if (!out) return fail(PRJ_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!plans || !d_P || ncases < 1) return fail(PRJ_ERR_ARG, "need ncases >= 1 plans and arrays");
    const bool graph_form = (mode & PRJ_BATCH_GRAPH) != 0;
    mode &= ~PRJ_BATCH_GRAPH;
    if (mode != PRJ_MODE_FP64 && mode != PRJ_MODE_FP32_REFINE) return fail(PRJ_ERR_ARG, "unknown mode %d", mode);
    const int dev = plans[0] ? plans[0]->device : 0;
    for (int i = 0; i < ncases; i++) {
        int rc = check_plan(plans[i]);
        if (rc) return rc;
        if (!d_P[i]) return fail(PRJ_ERR_ARG, "array %d is NULL", i);
        if (plans[i]->device != dev) return fail(PRJ_ERR_ARG, "plans on different devices");
        for (int j = 0; j < i; j++)
            if (plans[j] == plans[i]) return fail(PRJ_ERR_ARG, "plan %d appears twice (a plan serves one solve at a time)", i);
        if (mode == PRJ_MODE_FP32_REFINE && (rc = mixed_supported(plans[i]))) return rc;
    }
    DeviceGuard dg(dev);
    bool persistent = (mode == PRJ_MODE_FP64) && !graph_form;
    // the persistent kernel reads P as 16-byte pairs (and copies it with 16-byte cp.async)
    for (int i = 0; i < ncases && persistent; i++)
        persistent = prj::batchk_supported(plans[i]) && ((uintptr_t)d_P[i] & 15u) == 0;
    if (persistent) {
        prj_batch* b = new prj_batch();
        b->device = dev;
        b->ncases = ncases;
        b->persistent = true;
        cudaError_t e = prj::batchk_build(plans, d_P, ncases, &b->bk);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e == cudaSuccess) {
            *out = b;
            return PRJ_OK;
        }
        batch_release(b);
        delete b;
        // a tensor map the driver refuses: the graph form instead
        if (e != cudaErrorNotSupported) return cuda_fail(e, "persistent batch kernel set-up");
    }
    // eager pass: lazy buffers, kernel attributes, and a check that every case runs
    std::vector<cudaStream_t> streams((size_t)ncases, nullptr);
    std::vector<cudaEvent_t> joins((size_t)ncases, nullptr);
    cudaStream_t s0 = nullptr;
    cudaEvent_t fork = nullptr;
    auto cleanup = [&]() {
        for (auto s_ : streams) if (s_) cudaStreamDestroy(s_);
        for (auto e_ : joins) if (e_) cudaEventDestroy(e_);
        if (fork) cudaEventDestroy(fork);
        if (s0) cudaStreamDestroy(s0);
    };
    auto bail = [&](int code) { cleanup(); return code; };
    int rc = PRJ_OK;
    std::vector<bool> timing((size_t)ncases);
    for (int i = 0; i < ncases; i++) {
        timing[i] = plans[i]->timing;
        plans[i]->timing = false;
        rc = (mode == PRJ_MODE_FP64) ? run_poisson(plans[i], d_P[i], 0) : run_mixed_poisson(plans[i], d_P[i], 0);
        if (rc) break;
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "batch warm-up");
    if (rc) {
        for (int i = 0; i < ncases; i++) plans[i]->timing = timing[i];
        return bail(rc);
    }
    prj_batch* b = new prj_batch();
    b->device = dev;
    b->ncases = ncases;
    e = cudaStreamCreateWithFlags(&s0, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
    for (int i = 0; i < ncases && e == cudaSuccess; i++) {
        e = cudaStreamCreateWithFlags(&streams[i], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&joins[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal);
    bool capturing = (e == cudaSuccess);
    if (e == cudaSuccess) e = cudaEventRecord(fork, s0);
    for (int i = 0; i < ncases && e == cudaSuccess && !rc; i++) {
        e = cudaStreamWaitEvent(streams[i], fork, 0);
        if (e != cudaSuccess) break;
        rc = (mode == PRJ_MODE_FP64) ? run_poisson(plans[i], d_P[i], streams[i])
                                     : run_mixed_poisson(plans[i], d_P[i], streams[i]);
        if (rc) break;
        e = cudaEventRecord(joins[i], streams[i]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s0, joins[i], 0);
    }
    if (capturing) {
        cudaError_t e2 = cudaStreamEndCapture(s0, &b->graph);
        if (e == cudaSuccess) e = e2;
    }
    for (int i = 0; i < ncases; i++) plans[i]->timing = timing[i];
    if (!rc && e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (!rc && e == cudaSuccess) {
        size_t nn = 0;
        if (cudaGraphGetNodes(b->graph, nullptr, &nn) == cudaSuccess && nn) {
            std::vector<cudaGraphNode_t> nodes(nn);
            cudaGraphGetNodes(b->graph, nodes.data(), &nn);
            for (cudaGraphNode_t nd : nodes) {
                cudaGraphNodeType t;
                if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) b->graph_kernels++;
            }
        }
    }
    if (rc || e != cudaSuccess) {
        if (!rc) rc = cuda_fail(e, "batch graph capture");
        batch_release(b);
        delete b;
        return bail(rc);
    }
    cleanup();
    *out = b;
    return PRJ_OK;
}

int prj_batch_launch(prj_batch* batch, void* stream) {
    if (!batch || (!batch->exec && !batch->persistent)) return fail(PRJ_ERR_ARG, "batch is NULL or empty");
    DeviceGuard dg(batch->device);
    if (batch->persistent) {
        CK(prj::batchk_launch(batch->bk, (cudaStream_t)stream), "persistent batch kernel");
        return PRJ_OK;
    }
    CK(cudaGraphLaunch(batch->exec, (cudaStream_t)stream), "batch graph launch");
    return PRJ_OK;
}

int prj_batch_info(const prj_batch* batch, int* persistent, int* kernels_per_launch, long long* work_items) {
    if (!batch) return fail(PRJ_ERR_ARG, "batch is NULL");
    if (persistent) *persistent = batch->persistent ? 1 : 0;
    if (kernels_per_launch) *kernels_per_launch = batch->persistent ? 1 : batch->graph_kernels;
    if (work_items) *work_items = batch->persistent ? batch->bk.nitems : 0;
    return PRJ_OK;
}

int prj_batch_check_error(prj_batch* batch, void* stream) {
    if (!batch) return fail(PRJ_ERR_ARG, "batch is NULL");
    if (!batch->persistent) return PRJ_OK;
    DeviceGuard dg(batch->device);
    cudaStream_t st = (cudaStream_t)stream;
    int* word = prj::batchk_err_word(batch->bk);
    int dev_err = 0;
    CK(cudaMemcpyAsync(&dev_err, word, sizeof(int), cudaMemcpyDeviceToHost, st), "batch error word");
    CK(cudaMemsetAsync(word, 0, sizeof(int), st), "batch error word");
    CK(cudaStreamSynchronize(st), "batch error word");
    if (dev_err) return fail(PRJ_ERR_TIMEOUT, "a bounded wait of the persistent batch kernel gave up (code %d)", dev_err);
    return PRJ_OK;
}

int prj_batch_destroy(prj_batch* batch) {
    if (!batch) return PRJ_OK;
    DeviceGuard dg(batch->device);
    batch_release(batch);
    delete batch;
    return PRJ_OK;
}

}  // extern "C"

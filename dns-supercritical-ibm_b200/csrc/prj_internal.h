// prj_internal.h -- plan layout and kernel launchers shared by the engine's
// translation units.  Not part of the public ABI (include/projection.h).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>

#include <vector>

#include "fft_device.cuh"
#include "fft_dif.cuh"

namespace prj {

// In-place DIF transform of one length (fft_dif.cuh): descriptor and device tables.
// `ok` is false when a radix has no hard-coded butterfly; the out-of-place
// Stockham kernels serve those lengths.
struct DifFft {
    bool ok = false;
    DifDev f{};
    double2* tw = nullptr;  // stage twiddles (forward sign)
    int* pos = nullptr;     // pos[k]: slot of index k after the transform
};

// One real-to-complex transform of length n along a contiguous axis, done as a
// complex FFT of length m (m = n/2 for even n, packed even/odd samples; m = n
// for odd n) plus a post-processing pass.  `nh` = n/2+1 spectral modes.
template <typename T>
struct RealFftPlan {
    int n = 0, m = 0, nh = 0;
    bool even = false;
    FftDev f{};                                  // complex FFT of length m
    typename C2<T>::t* tw = nullptr;             // stage twiddles (device)
    typename C2<T>::t* post = nullptr;           // exp(-2 pi i k / n), k = 0..m (device, even n only)
};

template <typename T>
struct ComplexFftPlan {
    FftDev f{};
    typename C2<T>::t* tw = nullptr;
};

// Spectral layout: X[y][kx][z] complex, kx in [0, nxh), z in [0, nz).
// Pivot table: D[y][kx][kzs], kzs in [0, mzp) covers the folded z wavenumber
// min(kz, nz - kz) = 0..nz/2 (padded to an even count).
struct Geometry {
    int nx, nz, ny;
    int nxh;      // nx/2 + 1
    int nzh;      // nz/2 + 1
    int mzp;      // nzh rounded up to a multiple of 2
    double dx, dz;
};

struct DeviceTables {
    double* bands = nullptr;     // a, b, c, a00, b00, c00 (6 ny)
    double* inv_dy_p = nullptr;  // ny
    double* dpdy_lo = nullptr;   // ny
    double* dpdy_hi = nullptr;   // ny
    double* ax = nullptr;        // nxh: -4/dx^2 sin^2(kx pi / nx)
    double* az = nullptr;        // nzh: -4/dz^2 sin^2(kzs pi / nz)
    double* piv = nullptr;       // D[y][kx][kzs]: Thomas pivots b + lambda - a c'
    double* pivc = nullptr;      // c'[y][kx][kzs] = c_y / D_y (the reference's poi_C, PSM:164-179), folded like D
};

}  // namespace prj

namespace prj {
// stage ids of the per-kernel timing record
enum Stage {
    kStFwdX = 0, kStZSolve = 1, kStBwdX = 2, kStCorrect = 3, kStStats = 4,
    kStZfftFwd = 5, kStThomas = 6, kStZfftInv = 7, kStResidual = 8, kStVdRhs = 9, kStVdPrep = 10, kNumStages = 12
};

struct StageRecord {
    int stage;
    cudaEvent_t t0, t1;
};
}  // namespace prj

struct prj_plan {
    int device = 0;
    bool timing = false;
    std::vector<prj::StageRecord> rec;       // events of the enabled timing window
    std::vector<cudaEvent_t> event_pool;     // reusable events
    double* host_stage = nullptr;            // device staging of the host-buffer entry points
    size_t host_stage_elems = 0;
    // pipelined host-buffer steps: two staging slots, copy-in / compute / copy-out streams
    double* hp_stage[2] = {nullptr, nullptr};
    size_t hp_elems = 0;
    cudaStream_t hp_st[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t hp_ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};  // in[2], cmp[2], out[2]
    long long hp_n = 0;
    unsigned flags = 0;
    bool has_metrics = false;
    prj::Geometry g{};
    prj::DeviceTables t{};
    prj::RealFftPlan<double> fx64;
    prj::ComplexFftPlan<double> fz64;
    double2* spec = nullptr;      // X[y][kx][z] complex FP64 (scratch of the solve)
    double* stat_buf = nullptr;   // device reduction slots
    double min_pivot = 0.0;
    size_t device_bytes = 0;
    int tz_fwd = 1;               // rows per CTA of the out-of-place x-transform kernels
    prj::DifFft xd;               // in-place transform of length fx64.m (x rows)
    prj::DifFft zd;               // in-place transform of length nz (z rows)
    int tz_xd = 1;                // rows per CTA of the in-place x-transform kernels
    int* kz_of_slot = nullptr;    // z wavenumber held by each slot of zd's output
    int kxs = 0;                  // spectral rows kx < kxs stored in FP64 (nxh on the FP64 path)
    int kxs_mixed = 0;            // FP64 row count of the mixed path
    int mixed_iters = 1;          // refinement iterations of the mixed path
    float2* spec32 = nullptr;     // FP32 spectral rows of the mixed path
    double* pbar = nullptr;       // per-plane means of P (ny) for the mixed-path residual
    double* psum = nullptr;       // per-CTA partial sums of P from the inverse x kernel (ny x tiles)
    size_t psum_elems = 0;
    bool psum_valid = false;      // psum holds the sums of the P last written by the inverse x kernel
    double* mix_b = nullptr;      // Poisson-only mixed solve: copy of the right-hand side
    double* mix_r = nullptr;      // Poisson-only mixed solve: residual
    int zfft_rows = 0;            // rows per CTA of the z-transform kernels (0: default rule)
    int zmode = 0;                // z direction: 0 split kernels, 1 fused pipelined, 2 unpipelined,
                                  // 3 one pass-plan kernel per x wavenumber (split where no plan)
    bool use_pass = true;         // compile-time pass-plan FFT kernels where the length has one
    int thomas_async = -1;        // Thomas lines streamed through a cp.async shared-memory ring:
                                  // -1 for the mixed storage only, 0 never, 1..4 always (ring shape)
    int tz_xp = 1;                // rows per CTA of the pass-plan x kernels
    double* vd_pad = nullptr;     // inv_dy_p_pad (ny+1) of the variable-density step
    double* vd_ih = nullptr;      // 0.5 / rho (halo'd) of the variable-density step (scratch)
    int x_order = 0;              // radix order of the in-place x transform (fft_pass.cuh PRJ_PASS_ALTS)
    int z_order = 0;              // radix order of the in-place z transform
    int z_planes = 0;             // planes per chunk of the per-wavenumber z kernels (0: their default)
    int z_stages = 0;             // stages of their copy rings (0: their default)
    double mixed_tau = 1e-3;      // FP64-row threshold of the mixed path
};

namespace prj {

// Kernel launchers (prj_kernels.cu).  All are asynchronous on `st`.
enum class FwdSource { Pressure, Divergence, Residual };

// a range of y planes [y0, y1) of one launch; y1 < 0 means up to ny
struct YRange {
    int y0 = 0, y1 = -1;
    YRange resolved(int ny) const { return YRange{y0, y1 < 0 ? ny : y1}; }
};

struct StepScalars {
    double dt, inv_dt;
    double wall[6];  // U_bot, V_bot, W_bot, U_top, V_top, W_top
};

cudaError_t launch_fwd_x(const prj_plan* pl, FwdSource src, const double* P, const double* Uh, const double* Vh,
                         const double* Wh, const StepScalars* sc, cudaStream_t st);
cudaError_t launch_zsolve(const prj_plan* pl, cudaStream_t st);
// divergence + forward x over a y range (the in-place x kernels)
inline cudaError_t launch_fwd_x_range(const prj_plan* pl, const double* Uh, const double* Vh, const double* Wh,
                                      const StepScalars* sc, cudaStream_t st, YRange yr);
cudaError_t launch_bwd_x(const prj_plan* pl, double* P, cudaStream_t st);
// kh: halo'd plane range [kh0, kh1) of 0 .. ny+1 (planes -1 .. ny); default all
cudaError_t launch_correction(const prj_plan* pl, const double* P, const double* Uh, const double* Vh,
                              const double* Wh, double* U, double* V, double* W, const StepScalars& sc,
                              cudaStream_t st, YRange kh = YRange{});
cudaError_t launch_build_pivots(const prj_plan* pl, cudaStream_t st);
cudaError_t launch_stats(const prj_plan* pl, const double* U, const double* V, const double* W, const double* P,
                         double* out2, cudaStream_t st);
// z transform + Thomas with bulk-copy prefetch (prj_zsolve.cu); cudaErrorNotSupported
// when the grid does not fit its shared-memory budget.  *err_word is raised if a
// bounded wait gives up.
cudaError_t launch_zsolve_pipelined(const prj_plan* pl, int* err_word, cudaStream_t st);
// z transform + Thomas + inverse z as one kernel per x wavenumber on the pass-plan
// butterflies (prj_zline.cu); cudaErrorNotSupported when nz has no pass plan
cudaError_t launch_zline(const prj_plan* pl, cudaStream_t st);
bool zline_supported(const prj_plan* pl);  // launch_zline would run (not fall back)

// x transforms with the in-place DIF FFT (prj_xfft.cu); used when pl->xd.ok
// bout: also store the source field (divergence) there; accum: P += result; sq: norms of
// the update and of the result (accum only)
cudaError_t launch_fwd_xd(const prj_plan* pl, FwdSource src, const double* P, const double* Uh, const double* Vh,
                          const double* Wh, const StepScalars* sc, cudaStream_t st, double* bout = nullptr,
                          YRange yr = YRange{});
// psum: per-CTA sums of the written P, [y][tile] (pass-plan kernel only; otherwise
// cudaErrorNotSupported and nothing launched)
cudaError_t launch_bwd_xd(const prj_plan* pl, double* P, cudaStream_t st, int accum = 0, double* sq = nullptr,
                          YRange yr = YRange{}, double* psum = nullptr);
int bwd_tiles_per_plane(const prj_plan* pl);
inline cudaError_t launch_fwd_x_range(const prj_plan* pl, const double* Uh, const double* Vh, const double* Wh,
                                      const StepScalars* sc, cudaStream_t st, YRange yr) {
    return launch_fwd_xd(pl, FwdSource::Divergence, nullptr, Uh, Vh, Wh, sc, st, nullptr, yr);
}
int choose_tz_xd(int m, bool even);
int choose_tz_xp(int m);                 // rows per CTA of the pass-plan x kernels
size_t pass_x_smem(int m, int tz);       // their shared memory

// z direction as separate kernels (prj_zsplit.cu); need pl->zd.ok and pl->kz_of_slot
cudaError_t launch_zfft(const prj_plan* pl, int dir, cudaStream_t st, YRange yr = YRange{});
cudaError_t launch_thomas(const prj_plan* pl, cudaStream_t st);
// Thomas sweeps of the lines kx0 .. kx0+rows-1 held in X as [y][kx - kx0][z] (FP64)
cudaError_t launch_thomas_rows(const prj_plan* pl, double2* X, int kx0, int rows, cudaStream_t st);
// mixed storage (FP64 rows kx < kxs in spec, FP32 rows in spec32)
cudaError_t launch_zfft_mixed(const prj_plan* pl, int dir, cudaStream_t st);
cudaError_t launch_thomas_mixed(const prj_plan* pl, cudaStream_t st);
// residual r = b - A p of the pinned operator and the per-plane means it needs (prj_mixed.cu)
cudaError_t launch_plane_mean(const prj_plan* pl, const double* P, double* pbar, cudaStream_t st);
// plane means from the inverse x kernel's partial sums ([ny][tiles])
cudaError_t launch_plane_mean_partials(const prj_plan* pl, const double* psum, int tiles, double* pbar,
                                       cudaStream_t st);
// forward x transform of the residual B - A P formed on the fly (the pass-plan kernel);
// cudaErrorNotSupported when the x length has no pass plan or an array is not 16-byte
// aligned (the caller then runs launch_residual and the forward x of its result)
cudaError_t launch_fwd_residual(const prj_plan* pl, const double* B, const double* P, const double* pbar,
                                cudaStream_t st);
cudaError_t launch_residual(const prj_plan* pl, const double* B, const double* P, const double* pbar, double* R,
                            cudaStream_t st);

// stat_buf slots: [0] min pivot (bits), [2] max|div u|, [3] max|P|, [6] device error word,
// [7] rho_min of the variable-density step (order-preserving integer image)
constexpr int kStatErrSlot = 6;
constexpr int kStatRhoSlot = 7;

// variable-density step (prj_vd.cu): halo'd fields supplied by the caller
struct VdFields {
    const double* rho;
    const double* P_now;
    const double* P_old;
    const double* div_now;
    double* P_next;
};
// rho_min and 0.5 / rho in one pass over rho
cudaError_t launch_vd_prep(const prj_plan* pl, const double* rho, double* ih, unsigned long long* slot,
                           cudaStream_t st);
cudaError_t launch_vd_rhs(const prj_plan* pl, const double* Uh, const double* Vh, const double* Wh, const VdFields& f,
                          const StepScalars& sc, const unsigned long long* slot, double* P, cudaStream_t st);
cudaError_t launch_vd_correction(const prj_plan* pl, const double* P, const double* Uh, const double* Vh,
                                 const double* Wh, const VdFields& f, const StepScalars& sc,
                                 const unsigned long long* slot, double* U, double* V, double* W, cudaStream_t st);
double vd_rho_min_host(unsigned long long o);

// Persistent batch kernel (prj_batchk.cu): FP64 solves of many plans from one work queue.
struct BatchKernel {
    void* d_cases = nullptr;   // per-case arguments
    void* d_segs = nullptr;    // runs of work items in execution order
    void* d_work = nullptr;    // item counter, per-case stage counters, error word
    size_t work_bytes = 0;     // bytes of d_work reset before every launch (all but the error word)
    size_t smem = 0;
    int grid = 0, nseg = 0, ncases = 0;
    long long nitems = 0;      // work items (runs of up to 16 tiles)
    long long ntiles = 0;      // tiles over all cases and stages
};
bool batchk_supported(const prj_plan* pl);   // the plan's lengths are among the kernel's pass plans
cudaError_t batchk_build(prj_plan* const* plans, double* const* d_P, int ncases, BatchKernel* out);
cudaError_t batchk_launch(const BatchKernel& k, cudaStream_t st);
int* batchk_err_word(const BatchKernel& k);
void batchk_free(BatchKernel* k);

// Sets the calling thread's prj_last_error_string() message and returns code.
int record_error(int code, const char* msg);

}  // namespace prj

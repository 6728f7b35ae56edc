// prj_dist.cu -- one FP64 Poisson solve spread over several GPUs (ranks).
//
// The reference spreads a solve over MPI ranks with pencil transposes
// (poisson_solver_multigpu.f90:328-554, diezDecomp's tr_poi_xy / tr_poi_yx): the
// transforms run where whole x- and z-rows are local, the Thomas sweeps where whole
// y-lines are.  Here rank r owns the y planes [y0, y1) for the transforms and the x
// wavenumbers [kx0, kx1) for the Thomas lines; the host exchanges the spectrum between
// the two ownerships with an all-to-all (torch.distributed, NCCL between GPUs).  The
// stages are the single-GPU kernels on plane and line subsets, so the assembled result
// equals the single-GPU split-kernel solve bit for bit.
//
// Layouts (complex FP64):
//   the plan's spectrum X[y][kx][z] (global y), of which a rank uses its planes;
//   the exchange blocks, q-major: [q][y - y0][kx - kxb[q]][z] for the destinations
//   q = 0 .. R-1 with x-wavenumber ranges [kxb[q], kxb[q+1]);
//   the line buffer [y][kx - kx0][z] over all ny planes: the blocks received from the
//   ranks in rank order, whose y ranges ascend and tile [0, ny).
#include <cstdio>

#include "../../include/projection.h"
#include "fft_host.h"
#include "prj_internal.h"

using prj::record_error;

namespace {

int dist_check(const prj_plan* pl, int y0, int y1) {
    if (!pl || !pl->spec) return record_error(PRJ_ERR_ARG, "prj_dist: NULL plan or plan without buffers");
    if (y0 < 0 || y1 > pl->g.ny || y0 > y1) return record_error(PRJ_ERR_ARG, "prj_dist: plane range outside [0, ny)");
    int fac[8];
    if (!pl->use_pass || !pl->zd.ok || !pl->kz_of_slot || prj::pass_radices(pl->g.nz, fac, 8) <= 0)
        return record_error(PRJ_ERR_UNSUPPORTED, "prj_dist: needs a z length with a compile-time pass plan");
    if (!pl->xd.ok)
        return record_error(PRJ_ERR_UNSUPPORTED, "prj_dist: needs an x length of radices 2, 3, 4, 5, 6, 8");
    return PRJ_OK;
}

int dist_bounds(const prj_plan* pl, const int* kxb, int R) {
    if (!kxb || R < 1) return record_error(PRJ_ERR_ARG, "prj_dist: NULL or empty x-wavenumber bounds");
    if (kxb[0] != 0 || kxb[R] != pl->g.nxh) return record_error(PRJ_ERR_ARG, "prj_dist: bounds must span [0, nx/2+1)");
    for (int q = 0; q < R; q++)
        if (kxb[q + 1] < kxb[q]) return record_error(PRJ_ERR_ARG, "prj_dist: bounds must not decrease");
    return PRJ_OK;
}

struct OnPlanDevice {
    int prev = -1;
    explicit OnPlanDevice(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~OnPlanDevice() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

int cuda_rc(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return PRJ_OK;
    char buf[256];
    snprintf(buf, sizeof(buf), "prj_dist: %s: %s", what, cudaGetErrorString(e));
    return record_error(PRJ_ERR_CUDA, buf);
}

// block copies between the plan's planes [y0, y1) and the q-major exchange blocks
int move_blocks(prj_plan* pl, int y0, int y1, const int* kxb, int R, double2* blocks, bool to_blocks,
                cudaStream_t st) {
    const size_t nz = (size_t)pl->g.nz, nh = (size_t)pl->g.nxh, rows = (size_t)(y1 - y0);
    const size_t pitch = nh * nz * sizeof(double2);
    size_t off = 0;
    for (int q = 0; q < R; q++) {
        const size_t w = (size_t)(kxb[q + 1] - kxb[q]) * nz;  // elements per plane in block q
        if (w && rows) {
            double2* sp = pl->spec + ((size_t)y0 * nh + (size_t)kxb[q]) * nz;
            const cudaError_t e =
                to_blocks ? cudaMemcpy2DAsync(blocks + off, w * sizeof(double2), sp, pitch, w * sizeof(double2), rows,
                                              cudaMemcpyDeviceToDevice, st)
                          : cudaMemcpy2DAsync(sp, pitch, blocks + off, w * sizeof(double2), w * sizeof(double2), rows,
                                              cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) return cuda_rc(e, "block copy");
        }
        off += w * rows;
    }
    return PRJ_OK;
}

prj::StepScalars scalars(const prj_step_params* params) {
    prj::StepScalars sc{};
    sc.dt = params->dt;
    sc.inv_dt = 1.0 / params->dt;
    sc.wall[0] = params->wall_U_bot; sc.wall[1] = params->wall_V_bot; sc.wall[2] = params->wall_W_bot;
    sc.wall[3] = params->wall_U_top; sc.wall[4] = params->wall_V_top; sc.wall[5] = params->wall_W_top;
    return sc;
}

int step_check(const prj_plan* pl, const prj_step_params* params) {
    if (!pl->has_metrics) return record_error(PRJ_ERR_STATE, "prj_dist: plan was created without inv_dy_p / dPdy");
    if (!params || !(params->dt > 0)) return record_error(PRJ_ERR_ARG, "prj_dist: NULL params or dt <= 0");
    return PRJ_OK;
}

}  // namespace

extern "C" {

int prj_dist_divergence(prj_plan* plan, const double* d_Uh_loc, const double* d_Vh_loc, const double* d_Wh_loc,
                        int y0, int y1, const prj_step_params* params, void* stream) {
    int rc = dist_check(plan, y0, y1);
    if (rc || (rc = step_check(plan, params))) return rc;
    if (y1 == y0) return PRJ_OK;
    if (!d_Uh_loc || !d_Vh_loc || !d_Wh_loc) return record_error(PRJ_ERR_ARG, "prj_dist_divergence: NULL field");
    OnPlanDevice od(plan->device);
    cudaStream_t st = (cudaStream_t)stream;
    const prj::StepScalars sc = scalars(params);
    // the local halo'd arrays start at halo'd plane y0 (global plane y0 - 1)
    const ptrdiff_t shift = (ptrdiff_t)y0 * (plan->g.nx + 2) * (plan->g.nz + 2);
    const prj::YRange yr{y0, y1};
    if ((rc = cuda_rc(prj::launch_fwd_x_range(plan, d_Uh_loc - shift, d_Vh_loc - shift, d_Wh_loc - shift, &sc, st, yr),
                      "divergence + forward x")))
        return rc;
    return cuda_rc(prj::launch_zfft(plan, -1, st, yr), "forward z");
}

int prj_dist_correct(prj_plan* plan, const double* d_P_ext, const double* d_Uh_loc, const double* d_Vh_loc,
                     const double* d_Wh_loc, double* d_U_loc, double* d_V_loc, double* d_W_loc, int y0, int y1,
                     const prj_step_params* params, void* stream) {
    int rc = dist_check(plan, y0, y1);
    if (rc || (rc = step_check(plan, params))) return rc;
    if (y1 == y0) return PRJ_OK;
    if (!d_P_ext || !d_Uh_loc || !d_Vh_loc || !d_Wh_loc || !d_U_loc || !d_V_loc || !d_W_loc)
        return record_error(PRJ_ERR_ARG, "prj_dist_correct: NULL array");
    OnPlanDevice od(plan->device);
    const prj::StepScalars sc = scalars(params);
    const ptrdiff_t shift = (ptrdiff_t)y0 * (plan->g.nx + 2) * (plan->g.nz + 2);
    // d_P_ext holds planes y0-1 .. y1-1 of P
    const double* Pg = d_P_ext - (ptrdiff_t)(y0 - 1) * plan->g.nz * plan->g.nx;
    // halo'd planes y0+1 .. y1 (global planes y0 .. y1-1), plus the wall planes at the ends
    const prj::YRange kh{y0 == 0 ? 0 : y0 + 1, y1 == plan->g.ny ? plan->g.ny + 2 : y1 + 1};
    return cuda_rc(prj::launch_correction(plan, Pg, d_Uh_loc - shift, d_Vh_loc - shift, d_Wh_loc - shift,
                                          d_U_loc - shift, d_V_loc - shift, d_W_loc - shift, sc, (cudaStream_t)stream,
                                          kh),
                   "correction");
}

int prj_dist_forward(prj_plan* plan, const double* d_P_local, int y0, int y1, void* stream) {
    int rc = dist_check(plan, y0, y1);
    if (rc) return rc;
    if (!d_P_local && y1 > y0) return record_error(PRJ_ERR_ARG, "prj_dist_forward: P is NULL");
    if (y1 == y0) return PRJ_OK;
    OnPlanDevice od(plan->device);
    cudaStream_t st = (cudaStream_t)stream;
    // the x kernels address P by global plane: shift the local array by y0 planes
    const double* Pg = d_P_local - (ptrdiff_t)y0 * plan->g.nz * plan->g.nx;
    const prj::YRange yr{y0, y1};
    if ((rc = cuda_rc(prj::launch_fwd_xd(plan, prj::FwdSource::Pressure, Pg, nullptr, nullptr, nullptr, nullptr, st,
                                         nullptr, yr), "forward x")))
        return rc;
    return cuda_rc(prj::launch_zfft(plan, -1, st, yr), "forward z");
}

int prj_dist_pack(prj_plan* plan, int y0, int y1, const int* kx_bounds, int nranks, double* d_send, void* stream) {
    int rc = dist_check(plan, y0, y1);
    if (rc || (rc = dist_bounds(plan, kx_bounds, nranks))) return rc;
    if (!d_send && y1 > y0) return record_error(PRJ_ERR_ARG, "prj_dist_pack: send buffer is NULL");
    OnPlanDevice od(plan->device);
    return move_blocks(plan, y0, y1, kx_bounds, nranks, reinterpret_cast<double2*>(d_send), true,
                       (cudaStream_t)stream);
}

int prj_dist_thomas(prj_plan* plan, double* d_lines, int kx0, int kx1, void* stream) {
    int rc = dist_check(plan, 0, plan ? plan->g.ny : 0);
    if (rc) return rc;
    if (kx0 < 0 || kx1 > plan->g.nxh || kx0 > kx1) return record_error(PRJ_ERR_ARG, "prj_dist_thomas: bad x-wavenumber range");
    if (kx1 == kx0) return PRJ_OK;
    if (!d_lines) return record_error(PRJ_ERR_ARG, "prj_dist_thomas: line buffer is NULL");
    OnPlanDevice od(plan->device);
    return cuda_rc(prj::launch_thomas_rows(plan, reinterpret_cast<double2*>(d_lines), kx0, kx1 - kx0,
                                           (cudaStream_t)stream),
                   "Thomas sweeps");
}

int prj_dist_unpack(prj_plan* plan, int y0, int y1, const int* kx_bounds, int nranks, const double* d_recv,
                    void* stream) {
    int rc = dist_check(plan, y0, y1);
    if (rc || (rc = dist_bounds(plan, kx_bounds, nranks))) return rc;
    if (!d_recv && y1 > y0) return record_error(PRJ_ERR_ARG, "prj_dist_unpack: receive buffer is NULL");
    OnPlanDevice od(plan->device);
    return move_blocks(plan, y0, y1, kx_bounds, nranks, reinterpret_cast<double2*>(const_cast<double*>(d_recv)), false,
                       (cudaStream_t)stream);
}

int prj_dist_inverse(prj_plan* plan, double* d_P_local, int y0, int y1, void* stream) {
    int rc = dist_check(plan, y0, y1);
    if (rc) return rc;
    if (!d_P_local && y1 > y0) return record_error(PRJ_ERR_ARG, "prj_dist_inverse: P is NULL");
    if (y1 == y0) return PRJ_OK;
    OnPlanDevice od(plan->device);
    cudaStream_t st = (cudaStream_t)stream;
    const prj::YRange yr{y0, y1};
    if ((rc = cuda_rc(prj::launch_zfft(plan, +1, st, yr), "inverse z"))) return rc;
    double* Pg = d_P_local - (ptrdiff_t)y0 * plan->g.nz * plan->g.nx;
    return cuda_rc(prj::launch_bwd_xd(plan, Pg, st, 0, nullptr, yr), "inverse x");
}

}  // extern "C"

// prj_ibm.cu -- immersed-boundary forcing of the predictor ahead of the projection.
//
// Rough-wall runs force u_hat, v_hat, w_hat before the divergence is formed
// (mod_cfd_subroutines.f90:411-426):
//   * ibm_part_2 (src/ibm_setup/mod_cfd_ibm.f90:47-131): every (x, z) column has a
//     bottom index and a top index per component; the column's cells 0..bot take
//     the bottom wall value, top..ny-1 (v: top..ny, the top wall face) the top one;
//   * the interpolated forcing points of diezdecomp_ibm_exec on one rank
//     (src/diezdecomp_api_ibm.f90:374-424): A[pos_i] = c1_i A[s1_i] + c2_i A[s2_i] + c0_i,
//     with every source read before any point is written, then copies
//     A[dst_j] = A[src_j] (the forced values' periodic images).
// Both run in place on the halo'd fields.  k_rough_force takes one thread per
// column (x fastest, so each plane's writes are coalesced) and touches only the
// rough layers; the interpolation is a gather into scratch followed by a scatter.
#include "../../include/projection.h"
#include "prj_internal.h"

namespace prj {

namespace {

__global__ void k_rough_force(int nx, int nz, int ny, double* __restrict__ F, const int* __restrict__ bot,
                              const int* __restrict__ top, int kmax, double vbot, double vtop) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nx * nz) return;
    const int i = c % nx, j = c / nx;
    const size_t hrow = (size_t)nx + 2, hplane = hrow * (size_t)(nz + 2);
    double* col = F + (size_t)(i + 1) + hrow * (size_t)(j + 1) + hplane;  // (i, j, k = 0)
    const int kb = min(bot[c], kmax);
    for (int k = 0; k <= kb; k++) col[(size_t)k * hplane] = vbot;
    for (int k = max(top[c], 0); k <= kmax; k++) col[(size_t)k * hplane] = vtop;
}

// every position is checked against the array length; an out-of-range one is
// skipped and counted in *bad (the host turns it into an error)
__device__ __forceinline__ bool inside(long long p, long long len, unsigned* bad) {
    if (p >= 0 && p < len) return true;
    atomicAdd(bad, 1u);
    return false;
}

__global__ void k_ibm_gather(int n, long long len, const double* __restrict__ A, const long long* __restrict__ s1,
                             const long long* __restrict__ s2, double* __restrict__ g, unsigned* bad) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    g[t] = inside(s1[t], len, bad) ? A[s1[t]] : 0.0;
    g[(size_t)n + t] = inside(s2[t], len, bad) ? A[s2[t]] : 0.0;
}

__global__ void k_ibm_apply(int n, long long len, double* __restrict__ A, const long long* __restrict__ pos,
                            const double* __restrict__ c0, const double* __restrict__ c1,
                            const double* __restrict__ c2, const double* __restrict__ g, unsigned* bad) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n || !inside(pos[t], len, bad)) return;
    // cw12(1,i)*buffer(pos_b(1,i)) + cw12(2,i)*buffer(pos_b(2,i)) + cw12(0,i)
    A[pos[t]] = __dadd_rn(__dadd_rn(__dmul_rn(c1[t], g[t]), __dmul_rn(c2[t], g[(size_t)n + t])), c0[t]);
}

__global__ void k_ibm_copy(int n, long long len, double* __restrict__ A, const long long* __restrict__ dst,
                           const long long* __restrict__ src, unsigned* bad) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n && inside(dst[t], len, bad) && inside(src[t], len, bad)) A[dst[t]] = A[src[t]];
}

}  // namespace

}  // namespace prj

using prj::record_error;

extern "C" {

int prj_rough_force(int nx, int nz, int ny, double* d_Uh, double* d_Vh, double* d_Wh, const prj_rough_inds* inds,
                    const prj_step_params* walls, void* stream) {
    if (nx < 1 || nz < 1 || ny < 1 || !d_Uh || !d_Vh || !d_Wh || !inds || !walls)
        return record_error(PRJ_ERR_ARG, "prj_rough_force: bad grid or NULL argument");
    if (!inds->U_bot || !inds->U_top || !inds->V_bot || !inds->V_top || !inds->W_bot || !inds->W_top)
        return record_error(PRJ_ERR_ARG, "prj_rough_force: NULL index array");
    cudaStream_t st = (cudaStream_t)stream;
    const int cols = nx * nz;
    const unsigned grid = (unsigned)((cols + 255) / 256);
    // kmax: last cell of the top range (ny-1 for cell-centred u, w; ny for the v face)
    prj::k_rough_force<<<grid, 256, 0, st>>>(nx, nz, ny, d_Uh, inds->U_bot, inds->U_top, ny - 1, walls->wall_U_bot,
                                             walls->wall_U_top);
    prj::k_rough_force<<<grid, 256, 0, st>>>(nx, nz, ny, d_Wh, inds->W_bot, inds->W_top, ny - 1, walls->wall_W_bot,
                                             walls->wall_W_top);
    prj::k_rough_force<<<grid, 256, 0, st>>>(nx, nz, ny, d_Vh, inds->V_bot, inds->V_top, ny, walls->wall_V_bot,
                                             walls->wall_V_top);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return record_error(PRJ_ERR_CUDA, cudaGetErrorString(e));
    return PRJ_OK;
}

int prj_ibm_interp(double* d_A, long long len, int n, const long long* d_pos, const long long* d_src1,
                   const long long* d_src2, const double* d_c0, const double* d_c1, const double* d_c2, int ncopy,
                   const long long* d_dst, const long long* d_src, double* d_scratch, void* stream) {
    if (!d_A || len < 1 || n < 0 || ncopy < 0 || !d_scratch) return record_error(PRJ_ERR_ARG, "prj_ibm_interp: bad arguments");
    if (n > 0 && (!d_pos || !d_src1 || !d_src2 || !d_c0 || !d_c1 || !d_c2))
        return record_error(PRJ_ERR_ARG, "prj_ibm_interp: NULL point array");
    if (ncopy > 0 && (!d_dst || !d_src)) return record_error(PRJ_ERR_ARG, "prj_ibm_interp: NULL copy array");
    cudaStream_t st = (cudaStream_t)stream;
    unsigned* bad = reinterpret_cast<unsigned*>(d_scratch + 2 * (size_t)n);
    cudaError_t e = cudaMemsetAsync(bad, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return record_error(PRJ_ERR_CUDA, cudaGetErrorString(e));
    if (n > 0) {
        const unsigned grid = (unsigned)((n + 255) / 256);
        prj::k_ibm_gather<<<grid, 256, 0, st>>>(n, len, d_A, d_src1, d_src2, d_scratch, bad);
        prj::k_ibm_apply<<<grid, 256, 0, st>>>(n, len, d_A, d_pos, d_c0, d_c1, d_c2, d_scratch, bad);
    }
    if (ncopy > 0)
        prj::k_ibm_copy<<<(unsigned)((ncopy + 255) / 256), 256, 0, st>>>(ncopy, len, d_A, d_dst, d_src, bad);
    unsigned h_bad = 0;
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(&h_bad, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return record_error(PRJ_ERR_CUDA, cudaGetErrorString(e));
    if (h_bad) return record_error(PRJ_ERR_ARG, "prj_ibm_interp: forcing position outside the array (skipped)");
    return PRJ_OK;
}

}  // extern "C"

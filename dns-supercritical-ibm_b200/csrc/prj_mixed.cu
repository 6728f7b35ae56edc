// prj_mixed.cu -- FP64 residual of the pinned Poisson operator, for the
// mixed-precision path (FP32 spectral storage + FP64 iterative refinement).
//
// The spectral solve inverts, exactly, the operator
//   (A p)(i,j,k) = (p(i+1) - 2 p(i) + p(i-1)) / dx^2        (x periodic)
//                + (p(j+1) - 2 p(j) + p(j-1)) / dz^2        (z periodic)
//                + a_k p(k-1) + b_k p(k) + c_k p(k+1)       (a_0 = c_{ny-1} = 0)
//                + (a00_k - a_k) pm(k-1) + (b00_k - b_k) pm(k) + (c00_k - c_k) pm(k+1)
// where pm(k) is the (x, z) mean of plane k: the kx = kz = 0 mode uses the
// pinned bands (poisson_solver_multigpu.f90:167-175), i.e. the Neumann problem
// with the gauge of the reference.  The x/z stencils are the ones whose
// eigenvalues are a_x, a_z (PSM:147-148).  k_residual forms r = b - A p in FP64 (the
// refinement's forward x transform forms it on the fly instead where the x length has a
// pass plan: fwd_xp_tile's residual source, xfft_tiles.cuh).
#include "prj_internal.h"
#include "residual.cuh"

namespace prj {

namespace {

// pm[k] = mean over (x, z) of plane k (one CTA per plane, fixed reduction order)
__global__ void __launch_bounds__(256) k_plane_mean(int nx, int nz, const double* __restrict__ P, double* pm) {
    const int k = blockIdx.x;
    const size_t n = (size_t)nx * nz;
    const double* p = P + (size_t)k * n;
    double s = 0.0;
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) s += p[i];
    __shared__ double red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) pm[k] = red[0] / (double)n;
}

// pm[k] = (sum of the inverse x kernel's tile sums of plane k, in tile order) / (nx nz)
__global__ void k_plane_mean_partials(int ny, int tiles, double inv_n, const double* __restrict__ ps, double* pm) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ny) return;
    double s = 0.0;
    for (int t = 0; t < tiles; t++) s += ps[(size_t)k * tiles + t];
    pm[k] = s * inv_n;
}

struct ResArgs {
    int nx, nz, ny;
    double idx2, idz2;
    const double* bands;  // a, b, c, a00, b00, c00
    const double* B;
    const double* P;
    const double* pm;
    double* R;
};

// one CTA per x-row (j, k)
__global__ void __launch_bounds__(128) k_residual(const ResArgs a) {
    const int nx = a.nx, nz = a.nz, ny = a.ny;
    const int k = blockIdx.x, j = blockIdx.y;
    const int jp = j + 1 == nz ? 0 : j + 1, jm = j == 0 ? nz - 1 : j - 1;
    const size_t row = ((size_t)k * nz + j) * nx;
    const double* p0 = a.P + row;
    const double* pjp = a.P + ((size_t)k * nz + jp) * nx;
    const double* pjm = a.P + ((size_t)k * nz + jm) * nx;
    const double* pkm = k > 0 ? a.P + ((size_t)(k - 1) * nz + j) * nx : p0;
    const double* pkp = k < ny - 1 ? a.P + ((size_t)(k + 1) * nz + j) * nx : p0;
    const double* bd = a.bands;
    const double ak = bd[k], bk = bd[ny + k], ck = bd[2 * ny + k];
    const double pin = residual_pin(bd, a.pm, ny, k);  // pinned-mode correction of the plane
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        const int ip = i + 1 == nx ? 0 : i + 1, im = i == 0 ? nx - 1 : i - 1;
        a.R[row + i] = residual_at(a.B[row + i], p0[i], p0[ip], p0[im], pjp[i], pjm[i], pkm[i], pkp[i], k > 0,
                                   k < ny - 1, a.idx2, a.idz2, ak, bk, ck, pin);
    }
}

}  // namespace

cudaError_t launch_plane_mean(const prj_plan* pl, const double* P, double* pbar, cudaStream_t st) {
    k_plane_mean<<<pl->g.ny, 256, 0, st>>>(pl->g.nx, pl->g.nz, P, pbar);
    return cudaGetLastError();
}

cudaError_t launch_plane_mean_partials(const prj_plan* pl, const double* psum, int tiles, double* pbar,
                                       cudaStream_t st) {
    const int ny = pl->g.ny;
    k_plane_mean_partials<<<(ny + 127) / 128, 128, 0, st>>>(ny, tiles, 1.0 / ((double)pl->g.nx * pl->g.nz), psum,
                                                          pbar);
    return cudaGetLastError();
}

cudaError_t launch_residual(const prj_plan* pl, const double* B, const double* P, const double* pbar, double* R,
                            cudaStream_t st) {
    const Geometry& g = pl->g;
    ResArgs a{};
    a.nx = g.nx; a.nz = g.nz; a.ny = g.ny;
    a.idx2 = 1.0 / (g.dx * g.dx);
    a.idz2 = 1.0 / (g.dz * g.dz);
    a.bands = pl->t.bands;
    a.B = B; a.P = P; a.pm = pbar; a.R = R;
    k_residual<<<dim3((unsigned)g.ny, (unsigned)g.nz), 128, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace prj

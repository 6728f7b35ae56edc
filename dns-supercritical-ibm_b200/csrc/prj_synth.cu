// prj_synth.cu -- synthetic channel predictor fields on the device (benchmarks, tests,
// and the served requests that bring a seed instead of a field).
//
// u_hat = 1.5 (1 - (y_p - 1)^2) + sigma n_u, v_hat = sigma n_v, w_hat = sigma n_w on the
// interior of the halo'd arrays, v_hat = 0 on the bottom wall face (k = 0): the channel
// predictor of the projection workload (a Poiseuille profile plus noise), written in one
// pass.  The normals n are a deterministic function of (seed, field, point): a
// splitmix64 hash of the counter gives two 32-bit uniforms, and one Box-Muller step in
// single precision turns them into one standard normal, stored as a double.  So a seed
// names a field exactly, and the generation costs about one write of the three fields.
// Halos are not written (the projection reads no halo of its inputs).
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/projection.h"
#include "prj_internal.h"

namespace prj {
namespace {

__device__ __forceinline__ unsigned long long synth_mix(unsigned long long z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// standard normal of counter c under key `seed`
__device__ __forceinline__ double synth_normal(unsigned long long seed, unsigned long long c) {
    const unsigned long long h = synth_mix(seed ^ synth_mix(c));
    const float u1 = ((unsigned)(h >> 40) + 0.5f) * 5.9604645e-8f;              // (0, 1), 24 bits
    const float u2 = (float)(unsigned)(h & 0xffffffu) * 5.9604645e-8f;           // [0, 1)
    const float r = sqrtf(-2.0f * __logf(u1));
    return (double)(r * __cosf(6.2831853f * u2));
}

__global__ void k_synth_predictor(int nx, int nz, int ny, const double* __restrict__ yp, unsigned long long seed,
                                  double sigma, double* Uh, double* Vh, double* Wh) {
    const unsigned long long n = (unsigned long long)nx * nz * ny;
    for (unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (unsigned long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % nx);
        const unsigned long long r = t / nx;
        const int j = (int)(r % nz);
        const int k = (int)(r / nz);
        const size_t h = (size_t)(i + 1) + (size_t)(nx + 2) * ((size_t)(j + 1) + (size_t)(nz + 2) * (size_t)(k + 1));
        const double d = yp[k] - 1.0;
        Uh[h] = 1.5 * (1.0 - d * d) + sigma * synth_normal(seed, 3 * t);
        Vh[h] = (k == 0) ? 0.0 : sigma * synth_normal(seed, 3 * t + 1);
        Wh[h] = sigma * synth_normal(seed, 3 * t + 2);
    }
}

}  // namespace
}  // namespace prj

extern "C" int prj_synth_channel_predictor(int nx, int nz, int ny, const double* d_yp, unsigned long long seed,
                                           double sigma, double* d_Uh, double* d_Vh, double* d_Wh, void* stream) {
    if (nx < 1 || nz < 1 || ny < 1 || !d_yp || !d_Uh || !d_Vh || !d_Wh)
        return prj::record_error(PRJ_ERR_ARG, "prj_synth_channel_predictor: bad size or NULL array");
    const unsigned long long n = (unsigned long long)nx * nz * ny;
    const int blocks = (int)((n + 255) / 256 < 148ull * 32 ? (n + 255) / 256 : 148ull * 32);
    prj::k_synth_predictor<<<blocks, 256, 0, (cudaStream_t)stream>>>(nx, nz, ny, d_yp, seed, sigma, d_Uh, d_Vh, d_Wh);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return prj::record_error(PRJ_ERR_CUDA, cudaGetErrorString(e));
    return PRJ_OK;
}

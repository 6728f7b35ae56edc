// prj_synth.cu -- synthetic channel predictor fields on the device (benchmarks, tests,
// and the served requests that bring a seed instead of a field).
//
// u_hat = 1.5 (1 - (y_p - 1)^2) + sigma n_u, v_hat = sigma n_v, w_hat = sigma n_w on the
// interior of the halo'd arrays, v_hat = 0 on the bottom wall face (k = 0): the channel
// predictor of the projection workload (a Poiseuille profile plus noise), written in one
// pass.  The normals n are a deterministic function of (seed, field, point): a
// splitmix64 hash of the counter gives two 32-bit uniforms, and one Box-Muller step in
// single precision turns them into one standard normal, stored as a double.  Every double
// operation is rounded on its own, so a seed names a field exactly.  One CTA per (y, z)
// row: the hashes and the Box-Muller step, not the writes, set its time (about 1.05 ms at
// 768x384x384, where the three fields' 2.75 GB alone would take 0.43 ms).
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

// one CTA per (y, z) row of the interior (row r = k nz + j, found once per CTA), threads
// along x: no per-point division, and point t = r nx + i keeps the counter of the field's
// linear interior index, so a seed names the same field whatever the launch shape
__global__ void k_synth_predictor(int nx, int nz, int ny, const double* __restrict__ yp, unsigned long long seed,
                                  double sigma, double* Uh, double* Vh, double* Wh) {
    const unsigned r = blockIdx.x;
    const int j = (int)(r % (unsigned)nz), k = (int)(r / (unsigned)nz);
    const double d = yp[k] - 1.0;
    const size_t h0 = (size_t)1 + (size_t)(nx + 2) * ((size_t)(j + 1) + (size_t)(nz + 2) * (size_t)(k + 1));
    const unsigned long long t0 = (unsigned long long)r * (unsigned long long)nx;
    // every operation rounded on its own (no contraction), so the field is fixed by the seed
    const double mean = __dmul_rn(1.5, __dsub_rn(1.0, __dmul_rn(d, d)));
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        const unsigned long long t = t0 + (unsigned long long)i;
        const size_t h = h0 + (size_t)i;
        Uh[h] = __dadd_rn(mean, __dmul_rn(sigma, synth_normal(seed, 3 * t)));
        Vh[h] = (k == 0) ? 0.0 : __dmul_rn(sigma, synth_normal(seed, 3 * t + 1));
        Wh[h] = __dmul_rn(sigma, synth_normal(seed, 3 * t + 2));
    }
}

}  // namespace
}  // namespace prj

extern "C" int prj_synth_channel_predictor(int nx, int nz, int ny, const double* d_yp, unsigned long long seed,
                                           double sigma, double* d_Uh, double* d_Vh, double* d_Wh, void* stream) {
    if (nx < 1 || nz < 1 || ny < 1 || !d_yp || !d_Uh || !d_Vh || !d_Wh)
        return prj::record_error(PRJ_ERR_ARG, "prj_synth_channel_predictor: bad size or NULL array");
    const unsigned long long rows = (unsigned long long)nz * ny;
    if (rows > 0x7fffffffull) return prj::record_error(PRJ_ERR_ARG, "prj_synth_channel_predictor: too many rows");
    const int threads = nx >= 256 ? 256 : (nx + 31) / 32 * 32;
    prj::k_synth_predictor<<<(unsigned)rows, threads, 0, (cudaStream_t)stream>>>(nx, nz, ny, d_yp, seed, sigma, d_Uh,
                                                                                 d_Vh, d_Wh);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return prj::record_error(PRJ_ERR_CUDA, cudaGetErrorString(e));
    return PRJ_OK;
}

// residual.cuh -- r = b - A p of the pinned discrete operator at one point, shared by the
// residual kernel (prj_mixed.cu) and the forward x tile that forms it on the fly
// (xfft_tiles.cuh), so both give the same bits.  A is stated in prj_mixed.cu's header:
// the x/z second differences, the wall-normal bands a, b, c of plane k, and the
// pinned-mode correction `pin` of the plane means pm.  Round-to-nearest intrinsics fix
// the operation order.
#pragma once
#include <cuda_runtime.h>

namespace prj {

// (b00_k - b_k) pm(k) + (a00_k - a_k) pm(k-1) + (c00_k - c_k) pm(k+1), the same for a whole plane
__device__ __forceinline__ double residual_pin(const double* bands, const double* pm, int ny, int k) {
    const double ak = bands[k], bk = bands[ny + k], ck = bands[2 * ny + k];
    const double a0 = bands[3 * ny + k], b0 = bands[4 * ny + k], c0 = bands[5 * ny + k];
    double pin = __dmul_rn(__dsub_rn(b0, bk), pm[k]);
    if (k > 0) pin = __dadd_rn(pin, __dmul_rn(__dsub_rn(a0, ak), pm[k - 1]));
    if (k < ny - 1) pin = __dadd_rn(pin, __dmul_rn(__dsub_rn(c0, ck), pm[k + 1]));
    return pin;
}

// b - A p at a point with value pc, x neighbours pxp / pxm, z neighbours pjp / pjm and wall-normal
// neighbours pkm / pkp (used where has_km / has_kp)
__device__ __forceinline__ double residual_at(double b, double pc, double pxp, double pxm, double pjp, double pjm,
                                              double pkm, double pkp, bool has_km, bool has_kp, double idx2,
                                              double idz2, double ak, double bk, double ck, double pin) {
    const double lx = __dadd_rn(__dsub_rn(pxp, __dmul_rn(2.0, pc)), pxm);
    const double lz = __dadd_rn(__dsub_rn(pjp, __dmul_rn(2.0, pc)), pjm);
    double ap = __dadd_rn(__dadd_rn(__dmul_rn(lx, idx2), __dmul_rn(lz, idz2)), __dmul_rn(bk, pc));
    if (has_km) ap = __dadd_rn(ap, __dmul_rn(ak, pkm));
    if (has_kp) ap = __dadd_rn(ap, __dmul_rn(ck, pkp));
    return __dsub_rn(b, __dadd_rn(ap, pin));
}

}  // namespace prj

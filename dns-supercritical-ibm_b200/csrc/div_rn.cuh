// div_rn.cuh -- correctly rounded division by a divisor whose reciprocal is known.
//
// Markstein's final correction step (P. Markstein, "IA-64 and Elementary Functions",
// Prentice Hall 2000; also M. Cornea, J. Harrison, P. T. P. Tang, "Scientific Computing
// on Itanium-based Systems", Intel Press 2002): with y = RN(1/D), the product
// q = RN(u y) is within one ulp of u / D, the residual r = u - D q is exact in one fused
// multiply-add, and RN(q + r y) is the correctly rounded quotient RN(u / D), for
// operands and quotients inside the normal range (the window below).  When r is zero q is already the exact
// quotient and is returned as it is: that also keeps the sign of a zero numerator
// (q = +-0 * y has the sign of u / D, while +0 * y + q could turn -0 into +0).
// y comes from __drcp_rn; when it is formed off a recurrence's critical path (D does
// not depend on the previous step), the dependent work per step is one multiply, two
// fused multiply-adds and a select.
//
// The correction step is exact only while u, D and q stay inside the normal range with
// room to spare: y = RN(1/D) must be normal, u - D q must be representable (it is about
// 2^-53 |u|, so u must lie well above the subnormal range) and q must neither overflow
// nor underflow.  Outside the window |u| in [2^-960, 2^1020] (or u = 0), |D| and |q| in
// [2^-1000, 2^1000] -- subnormal, huge, infinite or NaN operands, a zero divisor -- the
// quotient is taken from __ddiv_rn instead, so the result is RN(u / D) for every pair of
// doubles.  The window tests are integer compares on the exponent fields; the D test does
// not depend on the recurrence, and the q test runs beside the residual's multiply-add.
// prj_selftest_division compares the function with __ddiv_rn bit for bit on random
// pairs in and around the window (subnormals, infinities, NaNs and zeros included).
#pragma once

namespace prj {

// lo <= unbiased exponent of x <= hi (subnormals and zeros count as -1023, infinities
// and NaNs as 1024)
__device__ __forceinline__ bool exp_within(double x, int lo, int hi) {
    const int e = (int)((unsigned long long)__double_as_longlong(x) >> 52 & 0x7ffull) - 1023;
    return (unsigned)(e - lo) <= (unsigned)(hi - lo);
}

__device__ __forceinline__ double div_by_recip(double u, double D, double y) {
    const double q = __dmul_rn(u, y);
    const double r = __fma_rn(-D, q, u);
    const bool in_window =
        exp_within(D, -1000, 1000) && (u == 0.0 || (exp_within(u, -960, 1020) && exp_within(q, -1000, 1000)));
    if (!in_window) return __ddiv_rn(u, D);
    return r == 0.0 ? q : __fma_rn(r, y, q);
}

}  // namespace prj

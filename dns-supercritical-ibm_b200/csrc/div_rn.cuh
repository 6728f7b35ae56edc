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
// The correction step is exact only while the operands and the quotient stay inside the
// normal range with room to spare: y = RN(1/D) must be normal, u - D q must be
// representable (it is about 2^-53 |u|, so u must lie well above the subnormal range)
// and q must neither overflow nor underflow.  The divisors here are Thomas pivots, and
// plan creation checks that every pivot satisfies 2^-40 <= |D| <= 2^1000
// (PRJ_ERR_NUMERIC otherwise).  With D in that range, |q| in [2^-900, 2^1000) implies
// |u| >= 2^-941, so all three conditions hold; the function tests only the quotient's
// exponent (its high word: a mask, a subtraction and a compare) and takes the quotient
// from __ddiv_rn outside that window, unless u = 0 (then q = +-0 is exact).  So for every
// u -- zeros, subnormals, infinities and NaNs included -- and every D in the pivot range,
// the result is RN(u / D).  prj_selftest_division compares it with __ddiv_rn bit for
// bit on random pairs of that domain, with the window's edges weighted.
#pragma once

namespace prj {

// smallest and largest |D| for which div_by_recip is correctly rounded for every u
constexpr double kDivRecipMinD = 0x1p-40;
constexpr double kDivRecipMaxD = 0x1p1000;

__device__ __forceinline__ double div_by_recip(double u, double D, double y) {
    const double q = __dmul_rn(u, y);
    const double r = __fma_rn(-D, q, u);
    // 2^-900 <= |q| < 2^1000: the biased exponent of q in [123, 2023)
    const unsigned hq = (unsigned)__double2hiint(q) & 0x7fffffffu;
    const bool q_in = hq - 0x07B00000u < 0x7E700000u - 0x07B00000u;
    if (!q_in && u != 0.0) return __ddiv_rn(u, D);
    return r == 0.0 ? q : __fma_rn(r, y, q);
}

}  // namespace prj

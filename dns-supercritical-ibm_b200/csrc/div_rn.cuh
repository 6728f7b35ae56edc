// div_rn.cuh -- correctly rounded division by a divisor whose reciprocal is known.
//
// Markstein's final correction step (P. Markstein, "IA-64 and Elementary Functions",
// Prentice Hall 2000; also M. Cornea, J. Harrison, P. T. P. Tang, "Scientific Computing
// on Itanium-based Systems", Intel Press 2002): with y = RN(1/D), the product
// q = RN(u y) is within one ulp of u / D, the residual r = u - D q is exact in one fused
// multiply-add, and RN(q + r y) is the correctly rounded quotient RN(u / D), for
// operands and quotients in the normal range.  When r is zero q is already the exact
// quotient and is returned as it is: that also keeps the sign of a zero numerator
// (q = +-0 * y has the sign of u / D, while +0 * y + q could turn -0 into +0).
// y comes from __drcp_rn; when it is formed off a recurrence's critical path (D does
// not depend on the previous step), the dependent work per step is one multiply, two
// fused multiply-adds and a select.  prj_selftest_division compares it with __ddiv_rn
// bit for bit, signed zero numerators and negative divisors included.  The divisors here
// are Thomas pivots, which plan creation requires to be nonzero and finite (a zero D would
// give NaN where IEEE division gives an infinity; the step's NaN check reports either).
#pragma once

namespace prj {

__device__ __forceinline__ double div_by_recip(double u, double D, double y) {
    const double q = __dmul_rn(u, y);
    const double r = __fma_rn(-D, q, u);
    return r == 0.0 ? q : __fma_rn(r, y, q);
}

}  // namespace prj

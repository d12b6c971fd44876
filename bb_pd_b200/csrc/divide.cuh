// Correctly rounded double division by a shared divisor, after P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000 processor",
// IBM J. Res. Dev. 34(1), 1990 (the reciprocal and quotient correction
// theorems), as also presented in Cornea, Harrison & Tang, "Scientific
// Computing on Itanium-based Systems", 2002, ch. 8.
//
//   recip_rn(b):  y0 = hardware reciprocal approximation (rcp.approx.ftz.f64),
//                 Newton-Raphson y <- y + y (1 - b y) until within one ulp, then
//                 one more correction step, which yields RN(1/b) for every b
//                 whose significand is not all ones (those are reported).
//   quot_rn(a, b, y):  with y = RN(1/b): q0 = RN(a y), r = a - q0 b (exact by
//                 fused multiply-add), q = RN(q0 + r y) = RN(a / b).
//
// Preconditions (no underflow or overflow in any step): b and a / b normal and
// well inside the exponent range, a not -0. The kernels use these only when
// every coordinate is +0 or of magnitude in [2^-100, 2^100] and L0 lies in the
// same range; outside it they fall back to IEEE division. bbpd_selftest_division
// compares both against IEEE `/` bit for bit on the device.
#pragma once

namespace bbpd {

__device__ __forceinline__ double rcp_approx(double b)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
    return y;
}

// RN(1/b) for normal positive b in [2^-200, 2^200]; ok = false when the low
// 32 bits of the significand are all ones, which includes the all-ones
// significand (the one case the final step does not cover).
__device__ __forceinline__ double recip_rn(double b, bool &ok)
{
    double y = rcp_approx(b);
    double e = __fma_rn(-b, y, 1.0);
    y = __fma_rn(y, e, y);
    e = __fma_rn(-b, y, 1.0);
    y = __fma_rn(y, e, y);
    e = __fma_rn(-b, y, 1.0);
    y = __fma_rn(y, e, y);
    ok = __double2loint(b) != -1;
    return y;
}

// RN(a / b) given y = RN(1/b), for a = +0 or |a / b| normal (see
// preconditions). An exact q0 leaves r = +0 and q0 unchanged.
__device__ __forceinline__ double quot_rn(double a, double b, double y)
{
    const double q0 = __dmul_rn(a, y);
    const double r = __fma_rn(-q0, b, a);
    return __fma_rn(r, y, q0);
}

}  // namespace bbpd

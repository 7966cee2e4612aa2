// fast_math.cuh -- the models' means (exp(xb) and the logistic probability
// 1 / (1 + exp(-xb))) in FP64 for the batched solver, with about half the
// FP64 operations of exp() followed by an IEEE division: on B200 the FP64
// pipe, not memory, bounds the gradient sums of an 8-fit group.
//
// exp: the table-driven method of P. T. P. Tang, "Table-driven
// implementation of the exponential function in IEEE floating-point
// arithmetic", ACM TOMS 15(2):144-157, 1989.  x = (64 k + j) ln2/64 + r with
// |r| <= ln2/128; exp(x) = 2^k * 2^(j/64) * exp(r), 2^(j/64) from a table
// (hi + lo, exp_table.h) and exp(r) - 1 by its Taylor polynomial to degree
// 6 (truncation below 4e-18 relative).  Arguments beyond +-708 (overflow,
// gradual underflow) and NaN take the library exp.
// Reciprocal: a single-precision seed refined by two Newton-Raphson steps
// r <- r + r (1 - d r) in FP64 (quadratic convergence: 2^-23 -> 2^-92
// before the final rounding).
// Both are within a few units in the last place of the correctly rounded
// values, as the library's exp and division are; tests/test_fast_math_gpu.py
// bounds them against an extended-precision reference.
#pragma once
#include "exp_table.h"

namespace cyc {

__device__ __forceinline__ double exp_table(double x) {
    if (!(fabs(x) <= 708.0)) return exp(x);
    const double n = rint(x * kInvLn2By64);
    const double r = fma(-n, kLn2By64Lo, fma(-n, kLn2By64Hi, x));
    const int ni = (int)n;
    const int j = ni & 63;
    const int k = (ni - j) / 64;
    const double p = fma(r * r,
                         fma(r, fma(r, fma(r, fma(r, 1.0 / 720.0, 1.0 / 120.0), 1.0 / 24.0), 1.0 / 6.0), 0.5), r);
    const double th = __ldg(kExp2Hi + j), tl = __ldg(kExp2Lo + j);
    const double m = th + fma(th, p, tl);
    return m * __longlong_as_double((long long)(k + 1023) << 52);
}

// 1 / d for d in [1, 2^127)
__device__ __forceinline__ double rcp_newton(double d) {
    double r = (double)__frcp_rn((float)d);
    double t = fma(-d, r, 1.0);
    r = fma(r, t, r);
    t = fma(-d, r, 1.0);
    return fma(r, t, r);
}

// 1 / (1 + exp(-v)); below -40, 1 + exp(-v) rounds to exp(-v) in FP64, so
// the probability is exp(v)
__device__ __forceinline__ double logistic_mean(double v) {
    if (v < -40.0) return exp_table(v);
    return rcp_newton(1.0 + exp_table(-v));
}

}  // namespace cyc

// Exponential and natural logarithm of the Spalart-Allmaras source term,
// written out so that the CPU restatement (oracle/) and the GPU kernels
// compute the same numbers: the host and device libraries' exp and log may
// differ in the last bit, which would break the bit-for-bit comparison of the
// two.  Both are textbook constructions, accurate to a few ulp (not correctly
// rounded); they are compiled without FMA contraction on both sides.
//
//  log x: x = m 2^e with m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s) with
//         s = (m-1)/(m+1), |s| <= 0.1716, by the odd power series of atanh to
//         s^23; log x = e ln2 + log m.
//  exp x: x = k ln2 + r, |r| <= ln2/2, by Cody-Waite reduction with ln2 split
//         into a 21-bit head (k*head exact) and a tail; exp r by its Taylor
//         series to r^14/14!; then scaled by 2^k.
//
// The integer powers of the reference (Fortran x**3 and x**6) are pinned to
// x3 = (x*x)*x and x6 = x3*x3.
#pragma once
#include <cmath>

#if defined(__CUDACC__)
#define FLITE_HD __host__ __device__ __forceinline__
#else
#define FLITE_HD inline
#endif

namespace flite_pm {

constexpr double kLn2Head = 0.6931467056274414;      // ln2 with its low 32 bits cleared
constexpr double kLn2Tail = 4.7493250390316726e-07;  // ln2 - head
constexpr double kInvLn2 = 1.4426950408889634;
constexpr double kSqrtHalf = 0.7071067811865476;

FLITE_HD double pm_log(double x) {
    if (!(x > 0.0)) return x == 0.0 ? -INFINITY : NAN;
    if (x == INFINITY) return x;
    int e = 0;
    double m = frexp(x, &e);  // x = m 2^e, m in [0.5, 1)
    if (m < kSqrtHalf) {
        m = 2.0 * m;
        e = e - 1;
    }
    const double s = (m - 1.0) / (m + 1.0);
    const double s2 = s * s;
    // 1 + s2/3 + s2^2/5 + ... + s2^11/23 (Horner)
    double p = 0.043478260869565216;  // 1/23
    p = 0.047619047619047616 + s2 * p;
    p = 0.05263157894736842 + s2 * p;
    p = 0.058823529411764705 + s2 * p;
    p = 0.06666666666666667 + s2 * p;
    p = 0.07692307692307693 + s2 * p;
    p = 0.09090909090909091 + s2 * p;
    p = 0.1111111111111111 + s2 * p;
    p = 0.14285714285714285 + s2 * p;
    p = 0.2 + s2 * p;
    p = 0.3333333333333333 + s2 * p;
    p = 1.0 + s2 * p;
    const double lm = 2.0 * s * p;
    const double de = (double)e;
    return (de * kLn2Head + lm) + de * kLn2Tail;
}

FLITE_HD double pm_exp(double x) {
    if (x != x) return x;
    if (x > 709.0) return INFINITY;
    if (x < -745.0) return 0.0;
    const double kd = nearbyint(x * kInvLn2);
    const int k = (int)kd;
    const double r = (x - kd * kLn2Head) - kd * kLn2Tail;
    // sum r^n/n!, n = 0..14 (Horner)
    double p = 1.1470745597729725e-11;
    p = 1.6059043836821613e-10 + r * p;
    p = 2.08767569878681e-09 + r * p;
    p = 2.505210838544172e-08 + r * p;
    p = 2.755731922398589e-07 + r * p;
    p = 2.7557319223985893e-06 + r * p;
    p = 2.48015873015873e-05 + r * p;
    p = 0.0001984126984126984 + r * p;
    p = 0.001388888888888889 + r * p;
    p = 0.008333333333333333 + r * p;
    p = 0.041666666666666664 + r * p;
    p = 0.16666666666666666 + r * p;
    p = 0.5 + r * p;
    p = 1.0 + r * p;
    p = 1.0 + r * p;
    return ldexp(p, k);
}

FLITE_HD double pm_cube(double x) { return (x * x) * x; }
FLITE_HD double pm_pow6(double x) {
    const double x3 = (x * x) * x;
    return x3 * x3;
}

}  // namespace flite_pm

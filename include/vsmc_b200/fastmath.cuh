// fastmath.cuh -- table-driven FP64 natural logarithm and exponential for
// the SMC step's device code (sm_100a).
//
// The methods are P. T. P. Tang's table-driven algorithms ("Table-driven
// implementation of the exponential function in IEEE floating-point
// arithmetic", ACM TOMS 15(2), 1989; "Table-driven implementation of the
// logarithm function in IEEE floating-point arithmetic", ACM TOMS 16(4),
// 1990), with a reciprocal table for the logarithm's reduction and Taylor
// polynomials for the reduced arguments; the tables (fastmath_tables.cuh)
// are generated at 60 digits by gen_fastmath_tables.py.  The final sum is
// assembled in double-double, so the results are within 0.5 ulp plus a
// small fraction of an ulp of the exact values (nearly always the
// correctly rounded double, as glibc's log and exp are) in about half the
// instructions of the general-purpose library functions.  Every operation
// is an explicit _rn intrinsic: nvcc contracts nothing here.
//
// fm_log(x): x = 2^k m, m in [sqrt(1/2), sqrt(2)); F = round(256 m) / 256,
// c = 1/F rounded; log x = k ln2 - log c + log1p(m c - 1) with |m c - 1| <=
// 2^-8.5, m c - 1 exact as a double-double.
// fm_exp(x): n = round(256 x / ln2), r = x - n ln2/256 (|r| <= 2^-9.5, as a
// double-double); exp x = 2^(n div 256) 2^((n mod 256)/256) exp(r).
#pragma once

#include <cstdint>

#include "fastmath_tables.cuh"

namespace vsmc_b200 {
namespace fm {

// s + e = a + b exactly (Knuth's two-sum).
__device__ __forceinline__ void two_sum(double a, double b, double &s,
                                        double &e)
{
    s = __dadd_rn(a, b);
    const double bb = __dadd_rn(s, -a);
    e = __dadd_rn(__dadd_rn(a, -__dadd_rn(s, -bb)), __dadd_rn(b, -bb));
}

// s + e = a + b exactly when a == 0 or |a| >= |b| (Dekker's fast two-sum).
__device__ __forceinline__ void fast_two_sum(double a, double b, double &s,
                                             double &e)
{
    s = __dadd_rn(a, b);
    e = __dadd_rn(b, -__dadd_rn(s, -a));
}

__device__ __forceinline__ double fm_log(double x)
{
    int hx = __double2hiint(x);
    int lx = __double2loint(x);
    int kadj = 0;
    if (hx < 0x00100000 || hx >= 0x7ff00000) {
        // zero, negative, subnormal, infinite or NaN
        if (x != x || x == INFINITY)
            return __dadd_rn(x, x);
        if (x == 0.0)
            return -INFINITY;
        if (x < 0.0)
            return __longlong_as_double(0x7ff8000000000000ll);
        x = __dmul_rn(x, 0x1p54); // subnormal: exact scaling
        hx = __double2hiint(x);
        lx = __double2loint(x);
        kadj = -54;
    }
    int k = ((hx >> 20) & 0x7ff) - 1023 + kadj;
    int hm = (hx & 0x000fffff) | 0x3ff00000; // m in [1, 2)
    if (hm > 0x3ff6a09e) {                   // m > about sqrt(2): m / 2
        hm -= 0x00100000;
        ++k;
    }
    const double m = __hiloint2double(hm, lx);
    // j = round(256 m) - kLogJ0 by the 1.5 * 2^52 rounding constant
    const int j = __double2loint(__fma_rn(m, 256.0, 0x1.8p52)) - kLogJ0;
    const double c = __ldg(&kLogTab[j][0]);
    const double lhi = __ldg(&kLogTab[j][1]);
    const double llo = __ldg(&kLogTab[j][2]);
    // r = m c - 1 = rh + rl exactly: p = m c rounded, pe its error, p - 1
    // exact (p is within 2^-8 of 1)
    const double p = __dmul_rn(m, c);
    const double pe = __fma_rn(m, c, -p);
    double rh, rl;
    fast_two_sum(__dadd_rn(p, -1.0), pe, rh, rl);
    // log1p(r) - r = -r^2/2 + r^3 (1/3 - r/4 + r^2/5 - r^3/6 + r^4/7)
    const double r2 = __dmul_rn(rh, rh);
    double q = __fma_rn(rh, 1.0 / 7.0, -1.0 / 6.0);
    q = __fma_rn(rh, q, 1.0 / 5.0);
    q = __fma_rn(rh, q, -1.0 / 4.0);
    q = __fma_rn(rh, q, 1.0 / 3.0);
    const double tail = __fma_rn(__dmul_rn(r2, rh), q, __dmul_rn(-0.5, r2));
    // k ln2 + (-log c) + r, then the low-order parts
    const double kd = (double)k;
    double s1, e1, s2, e2;
    two_sum(__dmul_rn(kd, kLn2Hi), lhi, s1, e1); // k * kLn2Hi is exact
    two_sum(s1, rh, s2, e2);
    double lo = __dadd_rn(tail, rl);
    lo = __dadd_rn(lo, llo);
    lo = __fma_rn(kd, kLn2Lo, lo);
    lo = __dadd_rn(lo, __dadd_rn(e1, e2));
    return __dadd_rn(s2, lo);
}

// 2^(n mod 256 / 256) exp(r) for x = n ln2/256 + r, and k = floor(n / 256)
// (|x| <= 746).
__device__ __forceinline__ double fm_exp_core(double x, int &k)
{
    // n = round(256 x / ln 2); its double nd is exact
    const double t = __fma_rn(x, kExpInv, 0x1.8p52);
    const int n = __double2loint(t);
    const double nd = __dadd_rn(t, -0x1.8p52);
    // r = x - n ln2/256 = rh + rl
    const double r0 = __fma_rn(-nd, kExpCHi, x);
    const double rh = __fma_rn(-nd, kExpCLo, r0);
    const double rl = __fma_rn(-nd, kExpCLo, __dadd_rn(r0, -rh));
    // exp(r) - 1 = rh + rl + rh^2 (1/2 + rh/6 + rh^2/24 + rh^3/120)
    double q = __fma_rn(rh, 1.0 / 120.0, 1.0 / 24.0);
    q = __fma_rn(rh, q, 1.0 / 6.0);
    q = __fma_rn(rh, q, 0.5);
    const double pm = __dadd_rn(rh, __fma_rn(__dmul_rn(rh, rh), q, rl));
    const int jt = n & (kExpN - 1);
    const double th = __ldg(&kExpTab[jt][0]);
    const double tl = __ldg(&kExpTab[jt][1]);
    k = n >> 8; // floor(n / 256)
    // 2^(j/256) exp(r) = th + (th pm + tl (1 + pm))
    return __dadd_rn(th, __fma_rn(th, pm, __fma_rn(tl, pm, tl)));
}

// The edges of the range: overflow, underflow, subnormal results, NaN.
static __device__ __noinline__ double fm_exp_edge(double x)
{
    if (x != x)
        return __dadd_rn(x, x);
    if (x > 709.782712893384)
        return INFINITY;
    if (x < -745.1332191019412)
        return 0.0;
    int k;
    const double v = fm_exp_core(x, k);
    if (k > 0) // v 2^(k-1) 2
        return __dmul_rn(
            __dmul_rn(v, __hiloint2double((k - 1 + 1023) << 20, 0)), 2.0);
    if (k >= -1022)
        return __dmul_rn(v, __hiloint2double((k + 1023) << 20, 0));
    // subnormal results: exact scaling into the normal range, then one
    // rounding
    return __dmul_rn(
        __dmul_rn(v, __hiloint2double((k + 1000 + 1023) << 20, 0)),
        0x1p-1000);
}

__device__ __forceinline__ double fm_exp(double x)
{
    if (!(fabs(x) <= 708.0))
        return fm_exp_edge(x);
    int k;
    const double v = fm_exp_core(x, k); // k in [-1022, 1021]
    return __dmul_rn(v, __hiloint2double((k + 1023) << 20, 0));
}

} // namespace fm
} // namespace vsmc_b200

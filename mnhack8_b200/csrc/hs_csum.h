// hs_csum.h -- compensated FP64 accumulation, host and device.
//
// The error-free transformations of T. Ogita, S. M. Rump and S. Oishi,
// "Accurate sum and dot product", SIAM J. Sci. Comput. 26(6), 2005:
//   TwoSum(a, b)     = (s, e) with s = fl(a + b) and s + e = a + b exactly
//                      (Knuth's branch-free form, 6 operations);
//   TwoProduct(a, b) = (p, e) with p = fl(a * b) and p + e = a * b exactly
//                      (one rounded product and one fused multiply-add);
//   Dot2: the running sum is kept as hi + lo; each term's rounding errors
//   (of the product and of the addition) are collected in lo, so the result
//   is as accurate as if it had been computed in twice the working precision
//   and then rounded.
// Merging two partial sums (hi1, lo1) + (hi2, lo2) = TwoSum(hi1, hi2) with
// lo = (lo1 + lo2) + e is symmetric in its operands, bit for bit, so xor
// butterflies over lanes give every lane the same value.
//
// Every operation is spelled out rounded to nearest (intrinsics on the
// device; the host build uses -ffp-contract=off), so the same inputs give the
// same bits on either side.
#pragma once

#if defined(__CUDACC__)
#define HS_HD __host__ __device__ __forceinline__
#else
#define HS_HD inline
#endif

#include <cmath>

namespace hs {

HS_HD double cs_add(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
HS_HD double cs_sub(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
HS_HD double cs_mul(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
HS_HD double cs_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}

struct CSum {
    double hi, lo;
};

HS_HD void two_sum(double a, double b, double& s, double& e) {
    s = cs_add(a, b);
    const double bb = cs_sub(s, a);
    e = cs_add(cs_sub(a, cs_sub(s, bb)), cs_sub(b, bb));
}
// c += x
HS_HD void csum_add(CSum& c, double x) {
    double s, e;
    two_sum(c.hi, x, s, e);
    c.hi = s;
    c.lo = cs_add(c.lo, e);
}
// c += a * b (Dot2 step)
HS_HD void csum_fma(CSum& c, double a, double b) {
    const double p = cs_mul(a, b);
    const double pe = cs_fma(a, b, -p);
    double s, e;
    two_sum(c.hi, p, s, e);
    c.hi = s;
    c.lo = cs_add(c.lo, cs_add(e, pe));
}
// a += b (two partial sums)
HS_HD void csum_merge(CSum& a, const CSum& b) {
    double s, e;
    two_sum(a.hi, b.hi, s, e);
    a.hi = s;
    a.lo = cs_add(cs_add(a.lo, b.lo), e);
}
HS_HD double csum_value(const CSum& c) { return cs_add(c.hi, c.lo); }

}  // namespace hs

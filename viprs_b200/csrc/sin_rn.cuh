// sin_rn.cuh -- sin(x) rounded to nearest, for the Lanczos weights of the
// affine and mapim interpolators (host and device).
//
// viprs evaluates its Lanczos2/3 weights with the platform sin (glibc on
// Linux), which rounds to nearest for all but a vanishing fraction of
// arguments.  This version is built from published methods only:
//   * Cody-Waite range reduction (Cody & Waite, "Software Manual for the
//     Elementary Functions", 1980): x = k pi/2 + r with pi/2 split into three
//     doubles, the products k * part formed exactly with fma;
//   * Taylor series of sin(r) and cos(r), |r| <= pi/4 (plus rounding), the
//     four leading terms in double-double arithmetic (Dekker 1971: TwoSum,
//     TwoProduct by fma), the tail in double;
//   * the result rounded once from the double-double sum.
// The relative error before that rounding is below 2^-75, so the result is
// the correctly rounded sin(x) unless sin(x) lies within 2^-75 of the midpoint
// of two doubles.  The constants are exact rationals (Machin's formula for pi,
// 1/n!) split into doubles by gen_sin_consts.py beside this file.
//
// Valid for |x| <= 2^20 (the interpolators pass |x| <= 3 pi); this file is
// compiled without floating-point contraction (fma appears only where written).
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define VIPRS_SIN_HD __host__ __device__ __forceinline__
// the entry point stays one out-of-line copy in device code: the samplers
// select their kernel at run time, so an inlined copy per weight would swell
// every sampler whether it evaluates a Lanczos weight or not
#define VIPRS_SIN_ENTRY static __host__ __device__ __noinline__
#else
#define VIPRS_SIN_HD inline
#define VIPRS_SIN_ENTRY static inline
#endif

namespace viprs {
namespace sinrn {

struct DD {
    double hi, lo;
};

// s + e == a + b exactly (Knuth's TwoSum)
VIPRS_SIN_HD DD two_sum(double a, double b) {
    const double s = a + b;
    const double bb = s - a;
    const double e = (a - (s - bb)) + (b - bb);
    return {s, e};
}

// s + e == a + b exactly, for |a| >= |b| (Dekker's FastTwoSum)
VIPRS_SIN_HD DD fast_two_sum(double a, double b) {
    const double s = a + b;
    return {s, b - (s - a)};
}

// p + e == a * b exactly
VIPRS_SIN_HD DD two_prod(double a, double b) {
    const double p = a * b;
    return {p, fma(a, b, -p)};
}

VIPRS_SIN_HD DD dd_add(DD a, DD b) {
    DD s = two_sum(a.hi, b.hi);
    const DD t = two_sum(a.lo, b.lo);
    s.lo += t.hi;
    s = fast_two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return fast_two_sum(s.hi, s.lo);
}

VIPRS_SIN_HD DD dd_mul(DD a, DD b) {
    DD p = two_prod(a.hi, b.hi);
    p.lo += a.hi * b.lo + a.lo * b.hi;
    return fast_two_sum(p.hi, p.lo);
}

// sin(r) = r + r^3 (a0 + a1 r^2 + ...), a_k = (-1)^(k+1) / (2k+3)!
VIPRS_SIN_HD DD sin_series(DD r) {
    const DD r2 = dd_mul(r, r);
    const double z = r2.hi;
    double t = 0x1.71b8ef6dcf572p-66;           // a9
    t = t * z + -0x1.2f49b46814157p-57;         // a8
    t = t * z + 0x1.952c77030ad4ap-49;          // a7
    t = t * z + -0x1.ae7f3e733b81fp-41;         // a6
    t = t * z + 0x1.6124613a86d09p-33;          // a5
    t = t * z + -0x1.ae64567f544e4p-26;         // a4
    DD s{t, 0.0};
    s = dd_add(dd_mul(s, r2), DD{0x1.71de3a556c734p-19, -0x1.c154f8ddc6c00p-73});   // a3
    s = dd_add(dd_mul(s, r2), DD{-0x1.a01a01a01a01ap-13, -0x1.a01a01a01a01ap-73});  // a2
    s = dd_add(dd_mul(s, r2), DD{0x1.1111111111111p-7, 0x1.1111111111111p-63});     // a1
    s = dd_add(dd_mul(s, r2), DD{-0x1.5555555555555p-3, -0x1.5555555555555p-57});   // a0
    return dd_add(r, dd_mul(dd_mul(r2, r), s));
}

// cos(r) = 1 + r^2 (b0 + b1 r^2 + ...), b_k = (-1)^(k+1) / (2k+2)!
VIPRS_SIN_HD DD cos_series(DD r) {
    const DD r2 = dd_mul(r, r);
    const double z = r2.hi;
    double t = -0x1.0ce396db7f853p-70;          // b10
    t = t * z + 0x1.e542ba4020225p-62;          // b9
    t = t * z + -0x1.6827863b97d97p-53;         // b8
    t = t * z + 0x1.ae7f3e733b81fp-45;          // b7
    t = t * z + -0x1.93974a8c07c9dp-37;         // b6
    t = t * z + 0x1.1eed8eff8d898p-29;          // b5
    t = t * z + -0x1.27e4fb7789f5cp-22;         // b4
    DD s{t, 0.0};
    s = dd_add(dd_mul(s, r2), DD{0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-76});    // b3
    s = dd_add(dd_mul(s, r2), DD{-0x1.6c16c16c16c17p-10, 0x1.f49f49f49f49fp-65});   // b2
    s = dd_add(dd_mul(s, r2), DD{0x1.5555555555555p-5, 0x1.5555555555555p-59});     // b1
    s = dd_add(dd_mul(s, r2), DD{-0.5, 0.0});                                       // b0
    return dd_add(DD{1.0, 0.0}, dd_mul(r2, s));
}

// sin(x) rounded to nearest (see the file comment), |x| <= 2^20.
VIPRS_SIN_ENTRY double sin_rn(double x) {
    if (!(fabs(x) >= 0x1p-26)) return x;  // |x| < 2^-26 (and NaN): sin(x) rounds to x
    const double pio2_1 = 0x1.921fb54442d18p+0, pio2_2 = 0x1.1a62633145c07p-54, pio2_3 = -0x1.f1976b7ed8fbcp-110;
    const double k = rint(x * 0x1.45f306dc9c883p-1);  // nearest multiple of pi/2
    // r = x - k pi/2 in double-double
    const DD p1 = two_prod(k, pio2_1);
    DD r = two_sum(x, -p1.hi);
    r = dd_add(r, DD{-p1.lo, 0.0});
    const DD p2 = two_prod(k, pio2_2);
    r = dd_add(r, DD{-p2.hi, -p2.lo});
    r = dd_add(r, DD{-(k * pio2_3), 0.0});
    const int q = int(static_cast<long long>(k) & 3);
    const DD v = (q & 1) ? cos_series(r) : sin_series(r);
    return (q & 2) ? -v.hi : v.hi;
}

}  // namespace sinrn
}  // namespace viprs

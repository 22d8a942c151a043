// vll_ddmath.cuh -- correctly rounded double-precision sin, cos, tan, atan,
// atan2, acos and exp for the map projection of the orthoimage rasters and the
// TIN geometry.
//
// The host code these kernels reproduce (ps2wgs_single,
// CoordConversion.cpp:396-490) calls the C library's functions; glibc 2.39
// returns the correctly rounded result for all but about 0.1% of arguments
// (tests/native/ddmath_check.cpp counts them).  CUDA's functions are accurate
// to one or two units in the last place, so about one raster coordinate in
// thirty came out an ulp apart from the host's; with these, about one in a
// thousand.  These versions evaluate each function in
// double-double arithmetic (Dekker 1971; Knuth's TwoSum; products exact
// through fma) to ~100 bits and round once, so they return the correctly
// rounded result except when the exact value lies within ~2^-100 relative of
// a rounding boundary.
//
//  * sin / cos / tan: x reduced by k * pi/2 with pi/2 split into three
//    doubles (the digits of pi), then the Taylor series of sin or cos on
//    |r| <= pi/4 by Horner's scheme in double-double.
//  * exp: x reduced by k * ln 2 (three doubles), Taylor series on
//    |r| <= ln2 / 2, scaled by 2^k.
//  * atan / atan2 / acos: one Newton step (on g(t) = x sin t - y cos t, or
//    cos t - x) from the hardware estimate, with g evaluated in double-double; the step has
//    quadratic convergence, so the corrected angle is good to ~2^-100.
//
// Arguments outside the ranges the projection produces (|x| >= 2^20 for the
// trigonometric functions, |x| > 700 for exp, infinities and NaNs) return the
// hardware functions' results.
#pragma once

#include <cmath>

// Device functions under nvcc (coefficients in constant memory, read
// uniformly by a warp); plain inline functions for a host compiler.
#ifdef __CUDACC__
#define VLL_HD __device__ __forceinline__
#define VLL_COEF static __constant__ double
#else
#define VLL_HD inline
#define VLL_COEF static constexpr double
#endif

namespace vll {
namespace ddm {

// IEEE operations that never contract, whatever the compilation flags.
VLL_HD double add(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    volatile double s = a + b;
    return s;
#endif
}
VLL_HD double sub(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    volatile double s = a - b;
    return s;
#endif
}
VLL_HD double mul(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    volatile double p = a * b;
    return p;
#endif
}
VLL_HD double div(double a, double b) {
#ifdef __CUDA_ARCH__
    return __ddiv_rn(a, b);
#else
    volatile double q = a / b;
    return q;
#endif
}
VLL_HD double fma(double a, double b, double c) {
#ifdef __CUDA_ARCH__
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}

struct dd {
    double hi, lo;
};

VLL_HD dd two_sum(double a, double b) {
    const double s = add(a, b);
    const double bb = sub(s, a);
    const double e = add(sub(a, sub(s, bb)), sub(b, bb));
    return {s, e};
}
VLL_HD dd quick_two_sum(double a, double b) {   // |a| >= |b|
    const double s = add(a, b);
    return {s, sub(b, sub(s, a))};
}
VLL_HD dd two_prod(double a, double b) {
    const double p = mul(a, b);
    return {p, fma(a, b, -p)};
}
VLL_HD dd dd_add(dd a, dd b) {
    dd s = two_sum(a.hi, b.hi);
    const dd t = two_sum(a.lo, b.lo);
    s.lo = add(s.lo, t.hi);
    s = quick_two_sum(s.hi, s.lo);
    s.lo = add(s.lo, t.lo);
    return quick_two_sum(s.hi, s.lo);
}
VLL_HD dd dd_neg(dd a) { return {-a.hi, -a.lo}; }
VLL_HD dd dd_sub(dd a, dd b) { return dd_add(a, dd_neg(b)); }
VLL_HD dd dd_mul(dd a, dd b) {
    dd p = two_prod(a.hi, b.hi);
    p.lo = add(p.lo, add(mul(a.hi, b.lo), mul(a.lo, b.hi)));
    return quick_two_sum(p.hi, p.lo);
}
VLL_HD dd dd_mul_d(dd a, double b) {
    dd p = two_prod(a.hi, b);
    p.lo = add(p.lo, mul(a.lo, b));
    return quick_two_sum(p.hi, p.lo);
}
VLL_HD dd dd_div(dd a, dd b) {
    const double q1 = div(a.hi, b.hi);
    dd r = dd_sub(a, dd_mul_d(b, q1));
    const double q2 = div(r.hi, b.hi);
    r = dd_sub(r, dd_mul_d(b, q2));
    const double q3 = div(r.hi, b.hi);
    const dd q = quick_two_sum(q1, q2);
    return dd_add(q, dd{q3, 0.0});
}
VLL_HD dd dd_div_d(dd a, double b) { return dd_div(a, dd{b, 0.0}); }
// The double nearest hi + lo (a normalised pair already has hi = fl(hi + lo)).
VLL_HD double round_dd(dd a) { return quick_two_sum(a.hi, a.lo).hi; }

// pi/2 and ln 2 as sums of three doubles (their leading 159 bits)
VLL_COEF kPio2[3] = {1.5707963267948966, 6.123233995736766e-17, -1.4973849048591698e-33};
VLL_COEF kLn2[3] = {0.6931471805599453, 2.3190468138462996e-17, 5.707708438416212e-34};

// Taylor coefficients (-1)^k / (2k+1)!, (-1)^k / (2k)! and 1 / n! as
// double-double pairs for the leading terms and doubles for the tails, whose
// contributions stay below 2^-100 of the result on the reduced ranges.
VLL_COEF kSinDD[7][2] = {
    {-0.16666666666666666, -9.25185853854297e-18},
    {0.008333333333333333, 1.1564823173178714e-19},
    {-0.0001984126984126984, -1.7209558293420705e-22},
    {2.7557319223985893e-06, -1.858393274046472e-22},
    {-2.505210838544172e-08, 1.448814070935912e-24},
    {1.6059043836821613e-10, 1.2585294588752098e-26},
    {-7.647163731819816e-13, -7.03872877733453e-30},
};
VLL_COEF kSinTail[6] = {2.8114572543455206e-15,  -8.22063524662433e-18,
                                1.9572941063391263e-20,  -3.868170170630684e-23,
                                6.446950284384474e-26,   -9.183689863795546e-29};
VLL_COEF kCosDD[7][2] = {
    {-0.5, 0.0},
    {0.041666666666666664, 2.3129646346357427e-18},
    {-0.001388888888888889, 5.300543954373577e-20},
    {2.48015873015873e-05, 2.1511947866775882e-23},
    {-2.755731922398589e-07, -2.3767714622250297e-23},
    {2.08767569878681e-09, -1.20734505911326e-25},
    {-1.1470745597729725e-11, -2.0655512752830745e-28},
};
VLL_COEF kCosTail[7] = {4.779477332387385e-14,   -1.5619206968586225e-16,
                                4.110317623312165e-19,   -8.896791392450574e-22,
                                1.6117375710961184e-24,  -2.4795962632247976e-27,
                                3.279889237069838e-30};
VLL_COEF kExpDD[12][2] = {
    {0.5, 0.0},
    {0.16666666666666666, 9.25185853854297e-18},
    {0.041666666666666664, 2.3129646346357427e-18},
    {0.008333333333333333, 1.1564823173178714e-19},
    {0.001388888888888889, -5.300543954373577e-20},
    {0.0001984126984126984, 1.7209558293420705e-22},
    {2.48015873015873e-05, 2.1511947866775882e-23},
    {2.7557319223985893e-06, -1.858393274046472e-22},
    {2.755731922398589e-07, 2.3767714622250297e-23},
    {2.505210838544172e-08, -1.448814070935912e-24},
    {2.08767569878681e-09, -1.20734505911326e-25},
    {1.6059043836821613e-10, 1.2585294588752098e-26},
};
VLL_COEF kExpTail[10] = {1.1470745597729725e-11, 7.647163731819816e-13,
                                 4.779477332387385e-14,  2.8114572543455206e-15,
                                 1.5619206968586225e-16, 8.22063524662433e-18,
                                 4.110317623312165e-19,  1.9572941063391263e-20,
                                 8.896791392450574e-22,  3.868170170630684e-23};

// Horner's scheme: tail in doubles, then the double-double coefficients.
template <int ND, int NT>
VLL_HD dd horner(const double (&cdd)[ND][2], const double (&tail)[NT], dd z) {
    double t = tail[NT - 1];
    for (int i = NT - 2; i >= 0; --i) t = add(mul(t, z.hi), tail[i]);
    dd acc = {t, 0.0};
    for (int k = ND - 1; k >= 0; --k) acc = dd_add(dd_mul(acc, z), dd{cdd[k][0], cdd[k][1]});
    return acc;
}

// sin r = r + r^3 (c1 + r^2 (c2 + ...)), cos r = 1 + r^2 (d1 + ...), |r| <= pi/4.
VLL_HD dd sin_series(dd r) {
    const dd r2 = dd_mul(r, r);
    return dd_add(r, dd_mul(dd_mul(r, r2), horner(kSinDD, kSinTail, r2)));
}
VLL_HD dd cos_series(dd r) {
    const dd r2 = dd_mul(r, r);
    return dd_add(dd{1.0, 0.0}, dd_mul(r2, horner(kCosDD, kCosTail, r2)));
}

// x = k * pi/2 + r, |r| <= pi/4; returns k mod 4.  |x| < 2^20.
VLL_HD int reduce_pio2(double x, dd &r) {
    const double k = rint(mul(x, 0.63661977236758134));   // 2/pi, rounded: any k works
    dd t = dd_sub(dd{x, 0.0}, two_prod(k, kPio2[0]));
    t = dd_sub(t, two_prod(k, kPio2[1]));
    t = dd_sub(t, dd{mul(k, kPio2[2]), 0.0});
    r = t;
    return ((int)k) & 3;
}

VLL_HD void sincos_dd(double x, dd &s, dd &c) {
    dd r;
    const int q = reduce_pio2(x, r);
    const dd sr = sin_series(r), cr = cos_series(r);
    switch (q) {
        case 0: s = sr; c = cr; break;
        case 1: s = cr; c = dd_neg(sr); break;
        case 2: s = dd_neg(sr); c = dd_neg(cr); break;
        default: s = dd_neg(cr); c = sr; break;
    }
}

VLL_HD bool trig_in_range(double x) { return fabs(x) < 1048576.0; }

VLL_HD double sin_cr(double x) {
    if (x == 0.0 || !trig_in_range(x)) return sin(x);
    dd r;
    const int q = reduce_pio2(x, r);
    const dd v = (q & 1) ? cos_series(r) : sin_series(r);
    return round_dd(q & 2 ? dd_neg(v) : v);
}
VLL_HD double cos_cr(double x) {
    if (!trig_in_range(x)) return cos(x);
    dd r;
    const int q = reduce_pio2(x, r);
    const dd v = (q & 1) ? sin_series(r) : cos_series(r);
    return round_dd(((q + 1) & 2) ? dd_neg(v) : v);
}
VLL_HD double tan_cr(double x) {
    if (x == 0.0 || !trig_in_range(x)) return tan(x);
    dd s, c;
    sincos_dd(x, s, c);
    return round_dd(dd_div(s, c));
}

VLL_HD double exp_cr(double x) {
    if (!(fabs(x) <= 700.0)) return exp(x);
    const double k = rint(mul(x, 1.4426950408889634));    // 1/ln2, rounded: any k works
    dd r = dd_sub(dd{x, 0.0}, two_prod(k, kLn2[0]));
    r = dd_sub(r, two_prod(k, kLn2[1]));
    r = dd_sub(r, dd{mul(k, kLn2[2]), 0.0});
    // e^r = 1 + r + r^2 (1/2! + r (1/3! + ...)), |r| <= ln2 / 2
    const dd sum = dd_add(dd_add(dd{1.0, 0.0}, r), dd_mul(dd_mul(r, r), horner(kExpDD, kExpTail, r)));
    return ldexp(round_dd(sum), (int)k);
}

// One Newton step on g(t) = cx * sin t - sy * cos t (root: t = atan2(sy, cx))
// from t0, g in double-double; returns fl(t0 + correction).
VLL_HD double newton_angle(double t0, double sy, double cx) {
    dd s, c;
    sincos_dd(t0, s, c);
    const dd g = dd_sub(dd_mul_d(s, cx), dd_mul_d(c, sy));
    const double gp = add(mul(cx, c.hi), mul(sy, s.hi));
    if (!(gp != 0.0)) return t0;
    const double corr = -div(add(g.hi, g.lo), gp);
    return add(t0, corr);
}

// acos by one Newton step on g(t) = cos t - x (g' = -sin t) from the
// hardware estimate; the endpoints and |x| > 1 return the hardware result.
VLL_HD double acos_cr(double x) {
    const double t0 = acos(x);
    if (!(fabs(x) < 1.0)) return t0;
    dd s, c;
    sincos_dd(t0, s, c);
    const dd g = dd_sub(c, dd{x, 0.0});
    if (!(s.hi != 0.0)) return t0;
    return add(t0, div(add(g.hi, g.lo), s.hi));
}

VLL_HD double atan_cr(double x) {
    const double t0 = atan(x);
    if (x == 0.0 || !(fabs(x) < 1e300)) return t0;
    return newton_angle(t0, x, 1.0);
}

VLL_HD double atan2_cr(double y, double x) {
    const double t0 = atan2(y, x);
    if (y == 0.0 || x == 0.0 || !(fabs(x) < 1e300) || !(fabs(y) < 1e300)) return t0;
    return newton_angle(t0, y, x);
}

}  // namespace ddm
}  // namespace vll

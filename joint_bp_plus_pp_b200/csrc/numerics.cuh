// Double-precision natural logarithm evaluated in double-double arithmetic and rounded once
// to the nearest double, for the |LLR| keys that order the OSD columns (the reference uses
// std::log, jointbp_ets.cpp:2484-2492).
//
// Method (textbook argument reduction + series): x = 2^k * m with m in [sqrt(1/2), sqrt(2)),
// log(x) = k*ln2 + 2*atanh(f), f = (m - 1) / (m + 1), |f| <= 0.1716, and
// atanh(f) = f * sum_{i>=0} f^(2i) / (2i + 1).  Everything after the exact reduction is
// carried as an unevaluated sum hi + lo (Dekker / Knuth two-sum, two-product via fma), so the
// result before the final rounding is accurate to about 2^-100 relative, and the rounded
// value is the correctly rounded logarithm except for inputs within ~2^-100 of a rounding
// midpoint.  ln2 is used as the double-double pair (hi, lo) of its exact value.
#pragma once

namespace jbp {

struct dd {
    double hi, lo;
};

__device__ __forceinline__ dd two_sum(double a, double b) {
    const double s = __dadd_rn(a, b);
    const double bb = __dsub_rn(s, a);
    const double e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
    return {s, e};
}

__device__ __forceinline__ dd quick_two_sum(double a, double b) {
    const double s = __dadd_rn(a, b);
    return {s, __dsub_rn(b, __dsub_rn(s, a))};
}

__device__ __forceinline__ dd two_prod(double a, double b) {
    const double p = __dmul_rn(a, b);
    return {p, __fma_rn(a, b, -p)};
}

__device__ __forceinline__ dd dd_add(dd a, dd b) {
    dd s = two_sum(a.hi, b.hi);
    dd t = two_sum(a.lo, b.lo);
    s.lo = __dadd_rn(s.lo, t.hi);
    s = quick_two_sum(s.hi, s.lo);
    s.lo = __dadd_rn(s.lo, t.lo);
    return quick_two_sum(s.hi, s.lo);
}

__device__ __forceinline__ dd dd_mul(dd a, dd b) {
    dd p = two_prod(a.hi, b.hi);
    p.lo = __dadd_rn(p.lo, __dadd_rn(__dmul_rn(a.hi, b.lo), __dmul_rn(a.lo, b.hi)));
    return quick_two_sum(p.hi, p.lo);
}

__device__ __forceinline__ dd dd_div(dd a, dd b) {
    // long division: q1 = a/b, r = a - q1*b, q2 = r/b, r -= q2*b, q3 = r/b
    const double q1 = __ddiv_rn(a.hi, b.hi);
    dd r = dd_add(a, dd_mul({-q1, 0.0}, b));
    const double q2 = __ddiv_rn(r.hi, b.hi);
    r = dd_add(r, dd_mul({-q2, 0.0}, b));
    const double q3 = __ddiv_rn(r.hi, b.hi);
    dd q = quick_two_sum(q1, q2);
    return dd_add(q, {q3, 0.0});
}

// Natural logarithm of a positive normal double, correctly rounded up to the caveat above.
__device__ inline double log_dd(double x) {
    int k = 0;
    double m = frexp(x, &k);  // x = m * 2^k, m in [0.5, 1)
    if (m < 0.70710678118654752440) {
        m = __dmul_rn(m, 2.0);
        k -= 1;
    }
    // f = (m - 1) / (m + 1); m - 1 is exact (Sterbenz), m + 1 as a double-double
    const dd num = {__dsub_rn(m, 1.0), 0.0};
    const dd den = two_sum(m, 1.0);
    const dd f = dd_div(num, den);
    const dd f2 = dd_mul(f, f);
    // atanh(f)/f = sum f^(2i) / (2i+1), Horner from the highest term; 24 terms reach 2^-120
    dd s = {1.0 / 49.0, 0.0};
    for (int i = 23; i >= 0; --i) {
        const dd c = dd_div({1.0, 0.0}, {static_cast<double>(2 * i + 1), 0.0});
        s = dd_add(c, dd_mul(s, f2));
    }
    dd l = dd_mul(dd_mul({2.0, 0.0}, f), s);
    const dd ln2 = {0x1.62e42fefa39efp-1, 0x1.abc9e3b39803fp-56};
    l = dd_add(dd_mul({static_cast<double>(k), 0.0}, ln2), l);
    return __dadd_rn(l.hi, l.lo);
}

}  // namespace jbp

// Double-double arithmetic (an unevaluated sum hi + lo of two doubles, ~106
// significand bits) from the error-free transformations of Knuth (TwoSum),
// Dekker (FastTwoSum) and the FMA product error; the "sloppy" addition of
// Bailey's QD library.
#pragma once

namespace fmlb {

struct dd {
    double hi, lo;
};

// a + b = s + e exactly
__device__ __forceinline__ void two_sum(double a, double b, double &s, double &e) {
    s = __dadd_rn(a, b);
    const double bb = __dsub_rn(s, a);
    e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}

// a + b = s + e exactly, for |a| >= |b|
__device__ __forceinline__ void fast_two_sum(double a, double b, double &s, double &e) {
    s = __dadd_rn(a, b);
    e = __dsub_rn(b, __dsub_rn(s, a));
}

__device__ __forceinline__ dd dd_add(dd a, dd b) {
    double s, e;
    two_sum(a.hi, b.hi, s, e);
    e = __dadd_rn(e, __dadd_rn(a.lo, b.lo));
    dd r;
    fast_two_sum(s, e, r.hi, r.lo);
    return r;
}

__device__ __forceinline__ dd dd_add_d(dd a, double b) {
    double s, e;
    two_sum(a.hi, b, s, e);
    e = __dadd_rn(e, a.lo);
    dd r;
    fast_two_sum(s, e, r.hi, r.lo);
    return r;
}

// a * (x.hi + x.lo) for a double a, accurate to ~2^-104 relative
__device__ __forceinline__ dd dd_mul_d(dd x, double a) {
    const double p = __dmul_rn(a, x.hi);
    double e = __fma_rn(a, x.hi, -p);
    e = __fma_rn(a, x.lo, e);
    dd r;
    fast_two_sum(p, e, r.hi, r.lo);
    return r;
}

__device__ __forceinline__ dd dd_neg(dd a) { return dd{-a.hi, -a.lo}; }

}  // namespace fmlb

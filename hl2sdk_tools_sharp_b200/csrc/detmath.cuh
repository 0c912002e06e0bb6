// detmath.cuh -- correctly rounded single-precision arcsine and power on
// the device: the reference's DetMathF.Asin and DetMathF.Pow
// (MapFormats/Numerics/DetMathF.cs:141-164, 265-292), which return the
// float nearest the exact value.
//
// Both start from CUDA's double-precision function, whose result lies
// within a few units of the last double place; rounded to float it is the
// correct answer unless it lies next to the midpoint between two floats.
// There the midpoint m decides, by an exact-enough test in double-double
// arithmetic: asin x > m exactly when x > sin m (sin m by its Taylor
// series), and x^y > m, for an integer exponent, exactly when the
// double-double power exceeds m.  A case neither test settles (a
// non-integer exponent next to a midpoint, or a tie the double-double
// value cannot split) returns the plain rounding and is counted in *open.
#pragma once

#include <cuda_runtime.h>

namespace vrad {

// Double-double arithmetic (error-free transformations with explicit
// rounding), used only to settle an arcsine that lies next to a rounding
// boundary of float.
struct DD {
    double hi, lo;
};
__device__ __forceinline__ DD two_sum(double a, double b) {
    const double s = __dadd_rn(a, b);
    const double bb = __dsub_rn(s, a);
    const double e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
    return {s, e};
}
__device__ __forceinline__ DD quick_two_sum(double a, double b) {
    const double s = __dadd_rn(a, b);
    return {s, __dsub_rn(b, __dsub_rn(s, a))};
}
__device__ __forceinline__ DD dd_mul(DD a, DD b) {
    const double p = __dmul_rn(a.hi, b.hi);
    double e = __fma_rn(a.hi, b.hi, -p);
    e = __dadd_rn(e, __dadd_rn(__dmul_rn(a.hi, b.lo), __dmul_rn(a.lo, b.hi)));
    return quick_two_sum(p, e);
}
__device__ __forceinline__ DD dd_sub_from_one(DD a) {  // 1 - a
    DD s = two_sum(1.0, -a.hi);
    return quick_two_sum(s.hi, __dsub_rn(s.lo, a.lo));
}
__device__ __forceinline__ DD dd_div_d(DD a, double b) {
    const double q1 = __ddiv_rn(a.hi, b);
    const double p = __dmul_rn(q1, b);
    const double e = __fma_rn(q1, b, -p);
    const double r = __dadd_rn(__dsub_rn(__dsub_rn(a.hi, p), e), a.lo);
    return quick_two_sum(q1, __ddiv_rn(r, b));
}
// sin m for |m| <= pi/2 by its Taylor series in Horner form,
// m (1 - m^2/(2*3) (1 - m^2/(4*5) (1 - ...))), 18 terms, in double-double.
__device__ inline DD dd_sin(double m) {
    const DD mm = {m, 0.0};
    const DD m2 = dd_mul(mm, mm);
    DD t = {1.0, 0.0};
    for (int k = 18; k >= 1; k--) t = dd_sub_from_one(dd_div_d(dd_mul(m2, t), (double)(2 * k) * (double)(2 * k + 1)));
    return dd_mul(mm, t);
}

// DetMathF.Asin: the correctly rounded float arcsine.  The double arcsine
// (within a few units of the last double place) rounds to the right float
// unless it lies next to the midpoint between two floats; there the
// midpoint m decides, as asin x > m exactly when x > sin m, with sin m in
// double-double.  `open` counts ties not even that settles (none expected).
__device__ inline float asin_cr(float x, unsigned long long *open) {
    if (x == 0.0f || isnan(x)) return x;
    if (!(fabsf(x) <= 1.0f)) return __int_as_float(0x7fc00000);
    const double r = asin((double)x);
    const float f = __double2float_rn(r);
    if ((double)f == r) return f;
    const float g = r > (double)f ? nextafterf(f, INFINITY) : nextafterf(f, -INFINITY);
    const double mid = __dmul_rn(__dadd_rn((double)f, (double)g), 0.5);
    const double ulp = ldexp(1.0, ilogb(r) - 52);
    if (fabs(__dsub_rn(r, mid)) > 8.0 * ulp) return f;
    const DD s = dd_sin(mid);
    const double d = __dsub_rn(__dsub_rn((double)x, s.hi), s.lo);
    const float lo = fminf(f, g), hi = fmaxf(f, g);
    if (d == 0.0) {
        atomicAdd(open, 1ull);
        return f;
    }
    return d > 0.0 ? hi : lo;
}

// x^y for a float base and exponent, correctly rounded to float.
__device__ inline DD dd_pow_int(double x, int n) {
    DD result = {1.0, 0.0}, base = {x, 0.0};
    while (n > 0) {
        if (n & 1) result = dd_mul(result, base);
        base = dd_mul(base, base);
        n >>= 1;
    }
    return result;
}

__device__ inline float pow_cr(float x, float y, unsigned long long *open) {
    const double r = pow((double)x, (double)y);
    const float f = __double2float_rn(r);
    if (!isfinite(r) || r == 0.0 || (double)f == r) return f;
    const double ar = fabs(r);
    const float af = fabsf(f);
    const float g = ar > (double)af ? nextafterf(af, INFINITY) : nextafterf(af, 0.0f);
    const double mid = __dmul_rn(__dadd_rn((double)af, (double)g), 0.5);
    const double ulp = ldexp(1.0, ilogb(ar) - 52);
    if (fabs(__dsub_rn(ar, mid)) > 8.0 * ulp) return f;
    const float ay = fabsf(y);
    if (ay == floorf(ay) && ay >= 1.0f && ay <= 64.0f) {
        DD p = dd_pow_int(fabs((double)x), (int)ay);
        if (y < 0.0f) {
            // 1 / p: compare 1 with mid * p instead.
            const DD mp = dd_mul({mid, 0.0}, p);
            const double d = __dsub_rn(__dsub_rn(1.0, mp.hi), mp.lo);  // > 0: x^y > mid
            if (d != 0.0) {
                const float mag = d > 0.0 ? fmaxf(af, g) : fminf(af, g);
                return f < 0.0f ? -mag : mag;
            }
        } else {
            const double d = __dadd_rn(__dsub_rn(p.hi, mid), p.lo);  // > 0: x^y > mid
            if (d != 0.0) {
                const float mag = d > 0.0 ? fmaxf(af, g) : fminf(af, g);
                return f < 0.0f ? -mag : mag;
            }
        }
    }
    atomicAdd(open, 1ull);
    return f;
}

}  // namespace vrad

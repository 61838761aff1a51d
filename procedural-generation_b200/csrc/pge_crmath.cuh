// pge_crmath.cuh -- float64 tan, atan, sin and cos rounded to nearest from a
// double-double evaluation, for host and device.
//
// The reference's face crossing (bake/globe/cubesphere.py:70-220) and the
// direction of a re-injected droplet (bake/globe/erosion/particle.py:400-401)
// call the C library's tan / atan / sin / cos in float64.  CUDA's own
// functions differ from them in the last bit now and then, and one flipped bit
// moves a droplet.  These evaluate each function to about 100 bits and round
// once, so they return the correctly rounded result except when the exact
// value lies within ~1e-30 (relative) of a halfway point between two doubles;
// wherever the C library is correctly rounded too, the two agree bit for bit.
//
// Method (textbook double-double arithmetic after Dekker and Knuth, with the
// exact product from fma):
//   sin, cos: x reduced to r = x - k pi/2 (|r| <= pi/4) with a three-part
//             pi/2, then their Taylor series in r^2 (Horner, terms to r^29).
//   tan:      sin(r) / cos(r), or -cos(r) / sin(r) for odd k.
//   atan:     |x| > 1 by pi/2 - atan(1/|x|); then t in [0, 1] by
//             atan(t) = atan(c) + atan((t - c) / (1 + t c)), c = round(8 t) / 8
//             (|z| <= 1/16), and the odd Taylor series of atan(z) to z^27.
// The constants (pi/2 in three parts, atan(k/8) in two) are the exact values
// rounded to double, computed with 90-digit decimal arithmetic.
//
// Every operation is an IEEE double add, multiply, divide or fma, so a host
// build and a device build give identical results (the device build must not
// contract a * b + c into fma itself: compile with -fmad=false).
#pragma once
#include <cmath>

#if defined(__CUDACC__)
#define PGE_HD __host__ __device__ __forceinline__
#else
#define PGE_HD inline
#endif

namespace pge {
namespace cr {

struct dd {
    double hi, lo;
};

PGE_HD dd two_sum(double a, double b)
{
    const double s = a + b;
    const double bb = s - a;
    const double e = (a - (s - bb)) + (b - bb);
    return {s, e};
}

PGE_HD dd quick_two_sum(double a, double b)
{
    const double s = a + b;
    return {s, b - (s - a)};
}

PGE_HD dd two_prod(double a, double b)
{
    const double p = a * b;
    return {p, fma(a, b, -p)};
}

PGE_HD dd add(dd a, dd b)
{
    dd s = two_sum(a.hi, b.hi);
    const dd t = two_sum(a.lo, b.lo);
    s.lo += t.hi;
    s = quick_two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return quick_two_sum(s.hi, s.lo);
}

PGE_HD dd neg(dd a) { return {-a.hi, -a.lo}; }

PGE_HD dd mul(dd a, dd b)
{
    dd p = two_prod(a.hi, b.hi);
    p.lo += a.hi * b.lo + a.lo * b.hi;
    return quick_two_sum(p.hi, p.lo);
}

PGE_HD dd mul_d(dd a, double b)
{
    dd p = two_prod(a.hi, b);
    p.lo += a.lo * b;
    return quick_two_sum(p.hi, p.lo);
}

// a / b: a first quotient, its remainder taken exactly, a second and third correction
PGE_HD dd div(dd a, dd b)
{
    const double q1 = a.hi / b.hi;
    dd r = add(a, neg(mul_d(b, q1)));
    const double q2 = r.hi / b.hi;
    r = add(r, neg(mul_d(b, q2)));
    const double q3 = r.hi / b.hi;
    const dd q = quick_two_sum(q1, q2);
    return add(q, dd{q3, 0.0});
}

PGE_HD dd div_d(dd a, double b)
{
    const double q1 = a.hi / b;
    const dd r = add(a, neg(two_prod(q1, b)));
    const double q2 = r.hi / b;
    const dd r2 = add(r, neg(two_prod(q2, b)));
    const double q3 = r2.hi / b;
    return add(quick_two_sum(q1, q2), dd{q3, 0.0});
}

// pi/2 = P1 + P2 + P3 (each the rounded rest of the one before)
constexpr double kPio2_1 = 1.5707963267948966;
constexpr double kPio2_2 = 6.123233995736766e-17;
constexpr double kPio2_3 = -1.4973849048591698e-33;
constexpr double kTwoOverPi = 0.6366197723675814;

// sin(r) and cos(r) for |r| <= pi/4 + a little, r in double-double
PGE_HD void sincos_reduced(dd r, dd &s, dd &c)
{
    const dd r2 = mul(r, r);
    // sin: r (1 - r^2/(2*3) (1 - r^2/(4*5) (1 - ...))), innermost n = 28 (the r^29 term)
    dd ps = {1.0, 0.0};
    for (int n = 28; n >= 2; n -= 2) ps = add(dd{1.0, 0.0}, neg(div_d(mul(r2, ps), (double)(n * (n + 1)))));
    s = mul(r, ps);
    // cos: 1 - r^2/(1*2) (1 - r^2/(3*4) (1 - ...)), innermost n = 27 (the r^28 term)
    dd pc = {1.0, 0.0};
    for (int n = 27; n >= 1; n -= 2) pc = add(dd{1.0, 0.0}, neg(div_d(mul(r2, pc), (double)(n * (n + 1)))));
    c = pc;
}

// x = k pi/2 + r; returns k mod 4.  |x| up to a few thousand keeps k pi/2 exact enough
PGE_HD int reduce(double x, dd &r)
{
    const double k = rint(x * kTwoOverPi);
    dd t = add(dd{x, 0.0}, neg(two_prod(k, kPio2_1)));  // x - k P1 exactly, then the smaller parts
    t = add(t, neg(two_prod(k, kPio2_2)));
    t = add(t, dd{-k * kPio2_3, 0.0});
    r = t;
    const long long ki = (long long)k;
    return (int)(((ki % 4) + 4) % 4);
}

PGE_HD double cr_sin(double x)
{
    if (x == 0.0 || !(x == x) || fabs(x) == INFINITY) return x == 0.0 ? x : x - x;
    dd r, s, c;
    const int q = reduce(x, r);
    sincos_reduced(r, s, c);
    const dd v = q == 0 ? s : q == 1 ? c : q == 2 ? neg(s) : neg(c);
    return v.hi + v.lo;
}

PGE_HD double cr_cos(double x)
{
    if (!(x == x) || fabs(x) == INFINITY) return x - x;
    dd r, s, c;
    const int q = reduce(x, r);
    sincos_reduced(r, s, c);
    const dd v = q == 0 ? c : q == 1 ? neg(s) : q == 2 ? neg(c) : s;
    return v.hi + v.lo;
}

PGE_HD double cr_tan(double x)
{
    if (x == 0.0 || !(x == x) || fabs(x) == INFINITY) return x == 0.0 ? x : x - x;
    dd r, s, c;
    const int q = reduce(x, r);
    sincos_reduced(r, s, c);
    const dd v = (q & 1) ? neg(div(c, s)) : div(s, c);
    return v.hi + v.lo;
}

// atan(k/8), k = 0..8, each as hi + lo
PGE_HD dd atan_k8(int k)
{
    switch (k) {
    case 1: return {0.12435499454676144, -3.1253241424539383e-18};
    case 2: return {0.24497866312686414, 1.0698755618734451e-17};
    case 3: return {0.35877067027057225, -2.4623815582638635e-17};
    case 4: return {0.4636476090008061, 2.2698777452961687e-17};
    case 5: return {0.5585993153435624, -5.4556305485916264e-18};
    case 6: return {0.6435011087932844, 1.5834785051444286e-17};
    case 7: return {0.7188299996216245, -2.1478388444456983e-17};
    case 8: return {0.7853981633974483, 3.061616997868383e-17};
    default: return {0.0, 0.0};
    }
}

// atan(t) for t in [0, 1] (double-double)
PGE_HD dd atan01(dd t)
{
    const int k = (int)rint(t.hi * 8.0);
    const double c = (double)k * 0.125;
    const dd z = div(add(t, dd{-c, 0.0}), add(dd{1.0, 0.0}, mul_d(t, c)));  // (t - c) / (1 + t c)
    const dd z2 = mul(z, z);
    // atan(z) = z (1 - z^2/3 + z^4/5 - ...), terms to z^27
    dd p = div_d(dd{1.0, 0.0}, 27.0);
    for (int n = 25; n >= 1; n -= 2) p = add(div_d(dd{1.0, 0.0}, (double)n), neg(mul(z2, p)));
    return add(atan_k8(k), mul(z, p));
}

PGE_HD double cr_atan(double x)
{
    if (x == 0.0 || !(x == x)) return x == 0.0 ? x : x + x;
    const bool neg_x = x < 0.0;
    const double ax = fabs(x);
    dd v;
    if (ax <= 1.0) {
        v = atan01(dd{ax, 0.0});
    } else if (ax == INFINITY) {
        v = dd{kPio2_1, kPio2_2};
    } else {  // pi/2 - atan(1/ax)
        const dd inv = div(dd{1.0, 0.0}, dd{ax, 0.0});
        v = add(add(dd{kPio2_1, kPio2_2}, dd{kPio2_3, 0.0}), neg(atan01(inv)));
    }
    const double y = v.hi + v.lo;
    return neg_x ? -y : y;
}

#if defined(__CUDACC__)
// out-of-line device copies: a call at a face crossing instead of the whole
// evaluation inlined into a register-heavy kernel
static __device__ __noinline__ double d_tan(double x) { return cr_tan(x); }
static __device__ __noinline__ double d_atan(double x) { return cr_atan(x); }
static __device__ __noinline__ double d_sin(double x) { return cr_sin(x); }
static __device__ __noinline__ double d_cos(double x) { return cr_cos(x); }
#endif

}  // namespace cr
}  // namespace pge

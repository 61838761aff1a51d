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
// exact product from fma; table-driven argument reduction):
//   sin, cos: x reduced to r = x - k pi/2 (|r| <= pi/4) with a three-part
//             pi/2, then r = j/32 + t (|t| <= 1/64) and the angle sums with
//             tabulated sin(j/32), cos(j/32); sin(t), cos(t) by their series,
//             the leading terms in double-double, the rest in double.
//   tan:      sin(r) / cos(r), or -cos(r) / sin(r) for odd k.
//   atan:     |x| > 1 by pi/2 - atan(1/|x|); then t in [0, 1] by
//             atan(t) = atan(k/64) + atan((t - k/64) / (1 + t k/64)), |z| <= 1/128,
//             and atan(z)'s odd series.
// The error before the final rounding stays below about 2^-100 of the result.
// The constants (pi/2 in three parts, the tables, the series' leading
// coefficients) are exact values rounded to double pairs, computed with
// 100-digit decimal arithmetic (gen_crmath_tables.py).
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

// the constants (pge_crmath_tables.inc, made by gen_crmath_tables.py): constant memory on the device,
// plain arrays on the host; PGE_CR_TAB names the copy the code being compiled reads
namespace host_tab {
#define PGE_CR_QUAL static const
#include "pge_crmath_tables.inc"
#undef PGE_CR_QUAL
}  // namespace host_tab
#if defined(__CUDACC__)
namespace dev_tab {
#define PGE_CR_QUAL static __constant__ const
#include "pge_crmath_tables.inc"
#undef PGE_CR_QUAL
}  // namespace dev_tab
#endif
#if defined(__CUDA_ARCH__)
#define PGE_CR_TAB dev_tab
#else
#define PGE_CR_TAB host_tab
#endif

PGE_HD dd pair(const double *v) { return {v[0], v[1]}; }

// sin(t) and cos(t) for |t| <= 1/64 (and a little), t double-double: the series' leading terms in
// double-double, the terms from t^7 (sin) and t^8 (cos) on, below 2^-47 of the result, in double
PGE_HD void sincos_small(dd t, dd &s, dd &c)
{
    const dd t2 = mul(t, t);
    const double x = t2.hi;
    const double ps = -1.0 / 5040.0 + x * (1.0 / 362880.0 + x * (-1.0 / 39916800.0 + x * (1.0 / 6227020800.0)));
    const dd sa = add(pair(PGE_CR_TAB::kInv5f), mul_d(t2, ps));  // 1/5! + t^2 (...)
    const dd sb = add(neg(pair(PGE_CR_TAB::kInv3f)), mul(t2, sa));  // -1/3! + t^2 (...)
    s = add(t, mul(mul(t, t2), sb));
    const double pc = 1.0 / 40320.0 + x * (-1.0 / 3628800.0 + x * (1.0 / 479001600.0));
    const dd ca = add(neg(pair(PGE_CR_TAB::kInv6f)), mul_d(t2, pc));  // -1/6! + t^2 (...)
    const dd cb = add(pair(PGE_CR_TAB::kInv4f), mul(t2, ca));
    const dd cc = add(neg(pair(PGE_CR_TAB::kInv2f)), mul(t2, cb));
    c = add(dd{1.0, 0.0}, mul(t2, cc));
}

// sin(r) and cos(r) for |r| <= pi/4 + a little: r = j/32 + t, the angle sums with the tabulated
// sin(j/32), cos(j/32)
PGE_HD void sincos_reduced(dd r, dd &s, dd &c)
{
    const int j = (int)rint(r.hi * 32.0);
    const int aj = j < 0 ? -j : j;
    const dd t = add(r, dd{-(double)j * 0.03125, 0.0});  // j/32 is exact
    dd st, ct;
    sincos_small(t, st, ct);
    dd sj = pair(PGE_CR_TAB::kSinJ[aj]);
    if (j < 0) sj = neg(sj);
    const dd cj = pair(PGE_CR_TAB::kCosJ[aj]);
    s = add(mul(sj, ct), mul(cj, st));
    c = add(mul(cj, ct), neg(mul(sj, st)));
}

// x = k pi/2 + r; returns k mod 4.  |x| up to a few thousand keeps k pi/2 exact enough
PGE_HD int reduce(double x, dd &r)
{
    const double k = rint(x * 0.6366197723675814);  // x * 2/pi, any rounding of it will do
    dd t = add(dd{x, 0.0}, neg(two_prod(k, PGE_CR_TAB::kPio2[0])));  // x - k P1 exactly, then the smaller parts
    t = add(t, neg(two_prod(k, PGE_CR_TAB::kPio2[1])));
    t = add(t, dd{-k * PGE_CR_TAB::kPio2[2], 0.0});
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

// atan(t) for t in [0, 1] (double-double): t = k/64 + ..., atan(t) = atan(k/64) + atan(z),
// z = (t - k/64) / (1 + t k/64), |z| <= 1/128; atan(z)'s terms to z^7 in double-double, from z^9 on in double
PGE_HD dd atan01(dd t)
{
    const int k = (int)rint(t.hi * 64.0);
    const double c = (double)k * 0.015625;
    const dd z = div(add(t, dd{-c, 0.0}), add(dd{1.0, 0.0}, mul_d(t, c)));
    const dd z2 = mul(z, z);
    const double x = z2.hi;
    const double pa = 1.0 / 9.0 + x * (-1.0 / 11.0 + x * (1.0 / 13.0 + x * (-1.0 / 15.0)));
    const dd a7 = add(neg(pair(PGE_CR_TAB::kInv7)), mul_d(z2, pa));  // -1/7 + z^2 (...)
    const dd a5 = add(pair(PGE_CR_TAB::kInv5), mul(z2, a7));
    const dd a3 = add(neg(pair(PGE_CR_TAB::kInv3)), mul(z2, a5));
    return add(pair(PGE_CR_TAB::kAtanK[k]), add(z, mul(mul(z, z2), a3)));
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
        v = dd{PGE_CR_TAB::kPio2[0], PGE_CR_TAB::kPio2[1]};
    } else {  // pi/2 - atan(1/ax)
        const dd inv = div(dd{1.0, 0.0}, dd{ax, 0.0});
        v = add(add(dd{PGE_CR_TAB::kPio2[0], PGE_CR_TAB::kPio2[1]}, dd{PGE_CR_TAB::kPio2[2], 0.0}), neg(atan01(inv)));
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

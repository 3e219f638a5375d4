// cplx.cuh -- ComplexF64 arithmetic on the parts, shared by complex.cu and cplxj.cu.
//
// Julia's Complex arithmetic written out, every operation rounded separately (no fused
// multiply-adds): (a+bi)(c+di) = (ac - bd) + (ad + bc)i; complex x real scales both parts;
// division is Baudin & Smith's robust algorithm (the one Julia's Base uses for ComplexF64,
// without its rescaling near overflow and underflow).  The CPU oracle writes the same
// operations in the same order.
#pragma once
#include "common.cuh"

namespace lhl {

struct dc {
    double re, im;
};

__device__ __forceinline__ dc cmul(dc a, dc b)
{
    return {dsub(dmul(a.re, b.re), dmul(a.im, b.im)), dadd(dmul(a.re, b.im), dmul(a.im, b.re))};
}
__device__ __forceinline__ dc csub(dc a, dc b) { return {dsub(a.re, b.re), dsub(a.im, b.im)}; }
__device__ __forceinline__ dc cadd(dc a, dc b) { return {dadd(a.re, b.re), dadd(a.im, b.im)}; }
__device__ __forceinline__ dc cscale(dc a, double s) { return {dmul(a.re, s), dmul(a.im, s)}; }
// tau * h with a real or a complex h (G = sigma I + tau H on a real or a complex reduction)
__device__ __forceinline__ dc tmul(dc a, double h) { return cscale(a, h); }
__device__ __forceinline__ dc tmul(dc a, dc h) { return cmul(a, h); }
__device__ __forceinline__ double cmag(dc a) { return dadd(fabs(a.re), fabs(a.im)); }
__device__ __forceinline__ bool ciszero(dc a) { return a.re == 0.0 && a.im == 0.0; }

__device__ __forceinline__ double cdiv2(double a, double b, double c, double d, double r, double t)
{
    if (r != 0.0) {
        const double br = dmul(b, r);
        return br != 0.0 ? dmul(dadd(a, br), t) : dadd(dmul(a, t), dmul(dmul(b, t), r));
    }
    return dmul(dadd(a, dmul(d, __ddiv_rn(b, c))), t);
}

// Baudin & Smith, "A robust complex division in Scilab" (2012).
__device__ __forceinline__ dc cdiv(dc x, dc y)
{
    const double a = x.re, b = x.im, c = y.re, d = y.im;
    if (fabs(d) <= fabs(c)) {
        const double r = __ddiv_rn(d, c), t = __ddiv_rn(1.0, dadd(c, dmul(d, r)));
        return {cdiv2(a, b, c, d, r, t), cdiv2(b, -a, c, d, r, t)};
    }
    const double r = __ddiv_rn(c, d), t = __ddiv_rn(1.0, dadd(d, dmul(c, r)));
    return {cdiv2(b, a, d, c, r, t), -cdiv2(a, -b, d, c, r, t)};
}

// |z| = hypot(re, im), the modulus the reference's abs(::Complex) returns (pivot search
// F:470-477 and balancing norms F:310-311 of a complex J).  Borges, "An improved algorithm
// for hypot(a, b)" (arXiv:1904.09481, 2019): the square root of a fused x^2 + y^2, then one
// correction step computed with fused multiply-adds; operands are first scaled by a power of
// two when they are very large or very small, so the steps are exact in scale.  IEEE square
// root and division; the oracle computes the same steps with C's fma, sqrt and /.
__device__ __forceinline__ double cabs_h(dc z)
{
    const double ax = fabs(z.re), ay = fabs(z.im);
    if (isinf(ax) || isinf(ay)) return __longlong_as_double(0x7ff0000000000000ll);
    if (isnan(ax) || isnan(ay)) return dadd(ax, ay);
    double x = fmax(ax, ay), y = fmin(ax, ay);
    if (y == 0.0) return x;
    double s = 1.0;
    if (x > 0x1p+500) { x = dmul(x, 0x1p-600); y = dmul(y, 0x1p-600); s = 0x1p+600; }
    else if (x < 0x1p-500) { x = dmul(x, 0x1p+600); y = dmul(y, 0x1p+600); s = 0x1p-600; }
    double h = __dsqrt_rn(dfma(x, x, dmul(y, y)));
    const double h2 = dmul(h, h), x2 = dmul(x, x);
    const double c = dsub(dadd(dfma(-y, y, dsub(h2, x2)), dfma(h, h, -h2)), dfma(x, x, -x2));
    h = dsub(h, __ddiv_rn(c, dmul(2.0, h)));
    return dmul(h, s);
}

}  // namespace lhl

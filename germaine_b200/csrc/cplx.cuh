// Complex helpers for the sm_100a kernels.
//
// Two families:
//  * rn_*  -- every product and sum rounded separately with the IEEE _rn
//    intrinsics (no FMA contraction).  The assembly kernel uses these to
//    reproduce, bit for bit, the roundings of the reference's C99 complex
//    arithmetic as compiled by gcc for x86-64 (no FMA in the baseline ISA):
//    complex*complex = (ac - bd, ad + bc), real*complex = component-wise.
//  * fast complex (cmul, cfma_sub, ...) for the numerical factorisation and
//    substitution, where FMA contraction is wanted.
#pragma once
#include <cuda_runtime.h>

namespace gm {

// ---- exact-rounding complex float / double ----
__device__ __forceinline__ float2 rn_cf(float re, float im) { return make_float2(re, im); }
__device__ __forceinline__ double2 rn_up(float2 a) { return make_double2((double)a.x, (double)a.y); }
__device__ __forceinline__ float2 rn_down(double2 a) {
    return make_float2(__double2float_rn(a.x), __double2float_rn(a.y));
}
__device__ __forceinline__ float2 rn_scale(float s, float2 a) {
    return make_float2(__fmul_rn(s, a.x), __fmul_rn(s, a.y));
}
__device__ __forceinline__ double2 rn_scale(double s, double2 a) {
    return make_double2(__dmul_rn(s, a.x), __dmul_rn(s, a.y));
}
__device__ __forceinline__ float2 rn_add(float2 a, float2 b) {
    return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
}
__device__ __forceinline__ float2 rn_sub(float2 a, float2 b) {
    return make_float2(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y));
}
__device__ __forceinline__ double2 rn_add(double2 a, double2 b) {
    return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}
__device__ __forceinline__ double2 rn_sub(double2 a, double2 b) {
    return make_double2(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y));
}
__device__ __forceinline__ float2 rn_mul(float2 a, float2 b) {
    return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                       __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ double2 rn_mul(double2 a, double2 b) {
    return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                        __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float2 rn_neg(float2 a) { return make_float2(-a.x, -a.y); }

// real float divided by complex float, rounded the way gcc's complex-float
// division rounds on x86-64: Smith's (1962) algorithm evaluated in double
// precision with a zero imaginary numerator, then rounded to float.
__device__ __forceinline__ float2 rn_real_div_cf(float a_f, float2 w) {
    const double a = a_f, b = 0.0, c = w.x, d = w.y;
    double re, im;
    if (fabs(c) >= fabs(d)) {
        const double r = __ddiv_rn(d, c);
        const double den = __dadd_rn(c, __dmul_rn(d, r));
        re = __ddiv_rn(__dadd_rn(a, __dmul_rn(b, r)), den);
        im = __ddiv_rn(__dsub_rn(b, __dmul_rn(a, r)), den);
    } else {
        const double r = __ddiv_rn(c, d);
        const double den = __dadd_rn(__dmul_rn(c, r), d);
        re = __ddiv_rn(__dadd_rn(__dmul_rn(a, r), b), den);
        im = __ddiv_rn(__dsub_rn(__dmul_rn(b, r), a), den);
    }
    return make_float2(__double2float_rn(re), __double2float_rn(im));
}

// ---- numerical complex arithmetic (FMA allowed) ----
template <class R> struct cplx_t;
template <> struct cplx_t<double> { using type = double2; };
template <> struct cplx_t<float> { using type = float2; };
template <class R> using cplx = typename cplx_t<R>::type;

__device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
template <class C> __device__ __forceinline__ C czero();
template <> __device__ __forceinline__ double2 czero<double2>() { return make_double2(0.0, 0.0); }
template <> __device__ __forceinline__ float2 czero<float2>() { return make_float2(0.f, 0.f); }

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return mk(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return mk(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return mk(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return mk(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return mk(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return mk(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// acc -= a*b
__device__ __forceinline__ void cfms(double2 &acc, double2 a, double2 b) {
    acc.x = fma(-a.x, b.x, acc.x); acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(-a.x, b.y, acc.y); acc.y = fma(-a.y, b.x, acc.y);
}
__device__ __forceinline__ void cfms(float2 &acc, float2 a, float2 b) {
    acc.x = fmaf(-a.x, b.x, acc.x); acc.x = fmaf(a.y, b.y, acc.x);
    acc.y = fmaf(-a.x, b.y, acc.y); acc.y = fmaf(-a.y, b.x, acc.y);
}
// acc += a*b
__device__ __forceinline__ void cfma(double2 &acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, acc.x); acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y); acc.y = fma(a.y, b.x, acc.y);
}
__device__ __forceinline__ void cfma(float2 &acc, float2 a, float2 b) {
    acc.x = fmaf(a.x, b.x, acc.x); acc.x = fmaf(-a.y, b.y, acc.x);
    acc.y = fmaf(a.x, b.y, acc.y); acc.y = fmaf(a.y, b.x, acc.y);
}
__device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ float cabs2(float2 a) { return a.x * a.x + a.y * a.y; }
// 1/a (straightforward; pivots here are far from over/underflow)
__device__ __forceinline__ double2 crcp(double2 a) {
    const double d = 1.0 / (a.x * a.x + a.y * a.y);
    return mk(a.x * d, -a.y * d);
}
__device__ __forceinline__ float2 crcp(float2 a) {
    const float d = 1.0f / (a.x * a.x + a.y * a.y);
    return mk(a.x * d, -a.y * d);
}
template <class C> __device__ __forceinline__ C cconv(double2 a);
template <> __device__ __forceinline__ double2 cconv<double2>(double2 a) { return a; }
template <> __device__ __forceinline__ float2 cconv<float2>(double2 a) { return mk((float)a.x, (float)a.y); }
__device__ __forceinline__ double2 cto_d(double2 a) { return a; }
__device__ __forceinline__ double2 cto_d(float2 a) { return mk((double)a.x, (double)a.y); }

}  // namespace gm

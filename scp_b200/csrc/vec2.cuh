// vec2.cuh -- a pair of fp32 values computed with the sm_100 packed FP32
// instructions (__ffma2_rn, __fadd2_rn, __fmul2_rn): one instruction does the
// arithmetic of two lattice sites.
#pragma once
#include <cuda_runtime.h>

#include "trig.cuh"

namespace scp {

struct V2 {
    float2 v;
    __device__ __forceinline__ V2() {}
    __device__ __forceinline__ V2(float2 a) : v(a) {}
    __device__ __forceinline__ V2(float a, float b) { v.x = a; v.y = b; }
    __device__ __forceinline__ explicit V2(float s) { v.x = s; v.y = s; }
};

__device__ __forceinline__ V2 operator+(V2 a, V2 b) { return V2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ V2 operator*(V2 a, V2 b) { return V2(__fmul2_rn(a.v, b.v)); }
// a - b as b*(-1) + a: one rounding, like a scalar subtraction
__device__ __forceinline__ V2 operator-(V2 a, V2 b) { return V2(__ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v)); }
__device__ __forceinline__ V2 operator-(V2 a) { return V2(-a.v.x, -a.v.y); }
__device__ __forceinline__ V2 fma2(V2 a, V2 b, V2 c) { return V2(__ffma2_rn(a.v, b.v, c.v)); }

// exact pair sums: s + e = a + b in each lane (Knuth two-sum)
__device__ __forceinline__ void two_sum2(V2 a, V2 b, V2 *s, V2 *e) {
    const V2 t = a + b;
    const V2 bb = t - a;
    *e = (a - (t - bb)) + (b - bb);
    *s = t;
}

// sin and cos of both lanes, |x| <= 2^12: the reduction and Taylor
// polynomials of sincos_bounded<float> (trig.cuh) in packed arithmetic.  The
// quadrant k = rint(x*2/pi) comes from adding 1.5*2^23, which leaves k in the
// low mantissa bits (round to nearest even, as rintf).
__device__ __forceinline__ void sincos2(V2 x, V2 *sn, V2 *cs) {
    using C = TrigConsts<float>;
    const float MAGIC = 12582912.0f;   // 1.5 * 2^23
    const V2 t = fma2(x, V2(C::TWO_OVER_PI), V2(MAGIC));
    const V2 kq = t - V2(MAGIC);
    V2 r = fma2(kq, V2(-C::P1), x);
    r = fma2(kq, V2(-C::P2), r);
    r = fma2(kq, V2(-C::P3), r);
    const V2 s = r * r;
    V2 p = fma2(V2(-2.5052108385441718775e-8f), s, V2(2.7557319223985890653e-6f));   // -1/11!, 1/9!
    p = fma2(p, s, V2(-1.9841269841269841270e-4f));                                   // -1/7!
    p = fma2(p, s, V2(8.3333333333333333333e-3f));                                    // 1/5!
    p = fma2(p, s, V2(-1.6666666666666666667e-1f));                                   // -1/3!
    const V2 sr = fma2(r * s, p, r);
    V2 q = fma2(V2(-2.7557319223985890653e-7f), s, V2(2.4801587301587301587e-5f));   // -1/10!, 1/8!
    q = fma2(q, s, V2(-1.3888888888888888889e-3f));                                   // -1/6!
    q = fma2(q, s, V2(4.1666666666666666667e-2f));                                    // 1/4!
    q = fma2(q, s, V2(-0.5f));                                                         // -1/2!
    const V2 cr = fma2(s, q, V2(1.0f));
    // x = r + k*pi/2: rotate (sin r, cos r) by k quarter turns, per lane
    const unsigned kx = __float_as_uint(t.v.x), ky = __float_as_uint(t.v.y);
    const unsigned gx = (kx & 2u) << 30, gy = (ky & 2u) << 30;   // sign flip for k = 2, 3 (mod 4)
    const float s1x = (kx & 1u) ? cr.v.x : sr.v.x, c1x = (kx & 1u) ? -sr.v.x : cr.v.x;
    const float s1y = (ky & 1u) ? cr.v.y : sr.v.y, c1y = (ky & 1u) ? -sr.v.y : cr.v.y;
    *sn = V2(__uint_as_float(__float_as_uint(s1x) ^ gx), __uint_as_float(__float_as_uint(s1y) ^ gy));
    *cs = V2(__uint_as_float(__float_as_uint(c1x) ^ gx), __uint_as_float(__float_as_uint(c1y) ^ gy));
}

__device__ __forceinline__ V2 sin2(V2 x) {
    V2 s, c;
    sincos2(x, &s, &c);
    return s;
}

}  // namespace scp

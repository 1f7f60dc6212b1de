// trig.cuh -- branch-free sine/cosine for the bounded angles of the gauged
// stepper (link angles in (-pi, pi], plaquette angles in (-4pi, 4pi]).
//
// Method: additive (Cody-Waite) range reduction r = x - k*pi/2 with
// k = rint(x*2/pi) and pi/2 split into three parts, then the Taylor series of
// sin and cos about 0 evaluated by Horner's rule in r^2 on |r| <= pi/4, and
// the quadrant k mod 4 applied by selects.  FP64: terms through r^17 / r^16
// (truncation below 1e-17); FP32: through r^11 / r^10.  Valid for |x| up to
// about 2^20; tests/test_gpu_trig.py checks the result against CUDA's sin/cos.
#pragma once
#include "common.cuh"

namespace scp {

template <class T>
struct TrigConsts;

template <>
struct TrigConsts<double> {
    // pi/2 = P1 + P2 + P3; P1 and P2 carry 33 significant bits each, so k*P1
    // and k*P2 are exact for |k| < 2^20; P3 is the rounded remainder.
    static constexpr double P1 = 0x1.921fb544p+0;
    static constexpr double P2 = 0x1.0b4611a6p-34;
    static constexpr double P3 = 0x1.3198a2e037073p-69;
    static constexpr double TWO_OVER_PI = 0x1.45f306dc9c883p-1;
};
template <>
struct TrigConsts<float> {
    // same split with 12-bit P1 and P2 (k*P exact for |k| < 2^12)
    static constexpr float P1 = 0x1.922p+0f;
    static constexpr float P2 = -0x1.2aep-18f;
    static constexpr float P3 = -0x1.de973ep-31f;
    static constexpr float TWO_OVER_PI = 0x1.45f306p-1f;
};

__device__ __forceinline__ double scp_rint(double x) { return rint(x); }
__device__ __forceinline__ float scp_rint(float x) { return rintf(x); }

// Taylor polynomials on |r| <= pi/4; s = r*r.
__device__ __forceinline__ void taylor_sc(double r, double *sn, double *cs) {
    const double s = r * r;
    // sin r = r (1 - s/3! + s^2/5! - ... + s^8/17!)
    double p = 2.8114572543455207632e-15;                  // 1/17!
    p = fma(p, s, -7.6471637318198164759e-13);             // -1/15!
    p = fma(p, s, 1.6059043836821614599e-10);              // 1/13!
    p = fma(p, s, -2.5052108385441718775e-8);              // -1/11!
    p = fma(p, s, 2.7557319223985890653e-6);               // 1/9!
    p = fma(p, s, -1.9841269841269841270e-4);              // -1/7!
    p = fma(p, s, 8.3333333333333333333e-3);               // 1/5!
    p = fma(p, s, -1.6666666666666666667e-1);              // -1/3!
    *sn = fma(r * s, p, r);
    // cos r = 1 - s/2! + s^2/4! - ... + s^8/16!
    double q = 4.7794773323873852974e-14;                  // 1/16!
    q = fma(q, s, -1.1470745597729724714e-11);             // -1/14!
    q = fma(q, s, 2.0876756987868098979e-9);               // 1/12!
    q = fma(q, s, -2.7557319223985890653e-7);              // -1/10!
    q = fma(q, s, 2.4801587301587301587e-5);               // 1/8!
    q = fma(q, s, -1.3888888888888888889e-3);              // -1/6!
    q = fma(q, s, 4.1666666666666666667e-2);               // 1/4!
    q = fma(q, s, -0.5);                                   // -1/2!
    *cs = fma(s, q, 1.0);
}
__device__ __forceinline__ void taylor_sc(float r, float *sn, float *cs) {
    const float s = r * r;
    float p = -2.5052108385441718775e-8f;                  // -1/11!
    p = fmaf(p, s, 2.7557319223985890653e-6f);             // 1/9!
    p = fmaf(p, s, -1.9841269841269841270e-4f);            // -1/7!
    p = fmaf(p, s, 8.3333333333333333333e-3f);             // 1/5!
    p = fmaf(p, s, -1.6666666666666666667e-1f);            // -1/3!
    *sn = fmaf(r * s, p, r);
    float q = -2.7557319223985890653e-7f;                  // -1/10!
    q = fmaf(q, s, 2.4801587301587301587e-5f);             // 1/8!
    q = fmaf(q, s, -1.3888888888888888889e-3f);            // -1/6!
    q = fmaf(q, s, 4.1666666666666666667e-2f);             // 1/4!
    q = fmaf(q, s, -0.5f);                                 // -1/2!
    *cs = fmaf(s, q, 1.0f);
}

// sin and cos of x, |x| <~ 2^20
template <class T>
__device__ __forceinline__ void sincos_bounded(T x, T *sn, T *cs) {
    using C = TrigConsts<T>;
    const T k = scp_rint(x * C::TWO_OVER_PI);
    T r = fma(-k, C::P1, x);
    r = fma(-k, C::P2, r);
    r = fma(-k, C::P3, r);
    T s, c;
    taylor_sc(r, &s, &c);
    const int q = ((int)k) & 3;
    // x = r + q*pi/2: rotate (s, c) by q quarter turns
    const T s1 = (q & 1) ? c : s;
    const T c1 = (q & 1) ? -s : c;
    *sn = (q & 2) ? -s1 : s1;
    *cs = (q & 2) ? -c1 : c1;
}

// sin and cos of any x: the bounded routine below 2^19, CUDA's sin / cos
// beyond (angles scaled by a user charge can be large)
__device__ __forceinline__ void sincos_any(double x, double *sn, double *cs) {
    if (fabs(x) < 0x1p19) {
        sincos_bounded(x, sn, cs);
    } else {
        *sn = sin(x);
        *cs = cos(x);
    }
}

template <class T>
__device__ __forceinline__ T sin_bounded(T x) {
    T s, c;
    sincos_bounded(x, &s, &c);
    return s;
}

}  // namespace scp

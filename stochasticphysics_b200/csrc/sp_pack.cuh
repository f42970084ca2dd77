// sp_pack.cuh — two FP32 particles per thread in paired (f32x2) arithmetic, sm_100a.
//
// F2 holds one quantity of two particles: lane x belongs to the thread's first
// particle, lane y to its second.  Adds, multiplies and fused multiply-adds issue as
// one paired instruction (__fadd2_rn, __fmul2_rn, __ffma2_rn; each lane rounds as the
// scalar __fadd_rn / __fmul_rn / __fmaf_rn), so the physics templates instantiated on
// F2 do two particles' work per FP32 instruction.  A product stays unevaluated (Prod)
// until it meets an addend, so a*b + c becomes one fused multiply-add, as the
// compiler's contraction makes of the scalar source; which products fuse follows the
// source order, so both lanes round alike and a particle's result does not depend on
// its partner, but it can differ from the one-particle kernel's in the last bits.
// Transcendentals, comparisons and selects act per lane.
#pragma once

#include "sp_math.cuh"

namespace sp {

struct F2 {
    float2 v;
    F2() = default;
    __device__ __forceinline__ explicit F2(float2 x) : v(x) {}
    __device__ __forceinline__ F2(float a) : v(make_float2(a, a)) {}
    __device__ __forceinline__ explicit F2(double a) : v(make_float2(static_cast<float>(a), static_cast<float>(a))) {}
    __device__ __forceinline__ explicit F2(int a) : v(make_float2(static_cast<float>(a), static_cast<float>(a))) {}
    __device__ __forceinline__ F2(float a, float b) : v(make_float2(a, b)) {}
};

__device__ __forceinline__ float2 neg2(float2 x) { return make_float2(-x.x, -x.y); }

// an unevaluated product a*b
struct Prod {
    float2 a, b;
    __device__ __forceinline__ operator F2() const { return F2(__fmul2_rn(a, b)); }
};

__device__ __forceinline__ Prod operator*(F2 x, F2 y) { return Prod{x.v, y.v}; }
__device__ __forceinline__ Prod operator*(Prod p, F2 y) { return Prod{__fmul2_rn(p.a, p.b), y.v}; }
__device__ __forceinline__ Prod operator*(F2 x, Prod p) { return Prod{x.v, __fmul2_rn(p.a, p.b)}; }
__device__ __forceinline__ Prod operator*(Prod p, Prod q) { return Prod{__fmul2_rn(p.a, p.b), __fmul2_rn(q.a, q.b)}; }
__device__ __forceinline__ F2 operator+(F2 x, F2 y) { return F2(__fadd2_rn(x.v, y.v)); }
__device__ __forceinline__ F2 operator-(F2 x, F2 y) { return F2(__fadd2_rn(x.v, neg2(y.v))); }
__device__ __forceinline__ F2 operator-(F2 x) { return F2(neg2(x.v)); }
__device__ __forceinline__ Prod operator-(Prod p) { return Prod{neg2(p.a), p.b}; }
__device__ __forceinline__ F2 operator+(Prod p, F2 c) { return F2(__ffma2_rn(p.a, p.b, c.v)); }
__device__ __forceinline__ F2 operator+(F2 c, Prod p) { return F2(__ffma2_rn(p.a, p.b, c.v)); }
__device__ __forceinline__ F2 operator+(Prod p, Prod q) { return F2(__ffma2_rn(p.a, p.b, __fmul2_rn(q.a, q.b))); }
__device__ __forceinline__ F2 operator-(Prod p, F2 c) { return F2(__ffma2_rn(p.a, p.b, neg2(c.v))); }
__device__ __forceinline__ F2 operator-(F2 c, Prod p) { return F2(__ffma2_rn(neg2(p.a), p.b, c.v)); }
__device__ __forceinline__ F2 operator-(Prod p, Prod q) {
    return F2(__ffma2_rn(p.a, p.b, neg2(__fmul2_rn(q.a, q.b))));
}
// quotients act per lane (IEEE division, as the scalar form)
__device__ __forceinline__ F2 operator/(F2 x, F2 y) { return F2(x.v.x / y.v.x, x.v.y / y.v.y); }

template <> struct real_of<Prod> { using type = F2; };
__device__ __forceinline__ V3<F2> operator*(Prod s, V3<F2> a) {
    const F2 t = s;
    return t * a;
}

__device__ __forceinline__ float lane0(F2 x) { return x.v.x; }
__device__ __forceinline__ float lane1(F2 x) { return x.v.y; }
__device__ __forceinline__ float lane(F2 x, int k) { return k ? x.v.y : x.v.x; }

template <> struct M<F2> {
    static constexpr bool kColdCalls = false;
    static __device__ __forceinline__ void sincos(F2 x, F2* s, F2* c) {
        float s0, c0, s1, c1;
        M<float>::sincos(x.v.x, &s0, &c0);
        M<float>::sincos(x.v.y, &s1, &c1);
        *s = F2(s0, s1);
        *c = F2(c0, c1);
    }
    static __device__ __forceinline__ F2 acos(F2 x) { return F2(M<float>::acos(x.v.x), M<float>::acos(x.v.y)); }
    static __device__ __forceinline__ F2 atan2(F2 y, F2 x) {
        return F2(M<float>::atan2(y.v.x, x.v.x), M<float>::atan2(y.v.y, x.v.y));
    }
    static __device__ __forceinline__ F2 sqrt(F2 x) { return F2(M<float>::sqrt(x.v.x), M<float>::sqrt(x.v.y)); }
    static __device__ __forceinline__ F2 inv_sin(F2 x) { return F2(M<float>::inv_sin(x.v.x), M<float>::inv_sin(x.v.y)); }
    static __device__ __forceinline__ F2 abs(F2 x) { return F2(fabsf(x.v.x), fabsf(x.v.y)); }
    static __device__ __forceinline__ F2 zero_inf(F2 x) { return F2(M<float>::zero_inf(x.v.x), M<float>::zero_inf(x.v.y)); }
    static constexpr float two_pi = 6.283185307179586f;
    static constexpr float eps = 1.1920929e-7f;
};

// the FP32 wrap x - 2 pi trunc(x / 2 pi) of each lane (wrap_two_pi<float>)
template <>
__device__ __forceinline__ F2 wrap_two_pi<F2>(F2 x) {
    const float2 t = __fmul2_rn(x.v, make_float2(0.159154943f, 0.159154943f));
    return F2(__ffma2_rn(make_float2(-M<float>::two_pi, -M<float>::two_pi), make_float2(truncf(t.x), truncf(t.y)), x.v));
}

}  // namespace sp

// sp_math.cuh — precision-generic device math, 3-vectors and the Philox noise source.
//
// FP64 instantiations call the IEEE double routines.  FP32 instantiations use
// the SFU approximations (__sincosf, __logf) where the stepping tolerates
// them; the field phase, time and ensemble sums never pass through here in
// FP32 (they are computed in double by the kernels).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "sp_types.h"

namespace sp {

template <class R> struct M;

// The FP64 step kernels are bound by instruction fetch: every inlined copy of a double
// transcendental adds a few hundred bytes of code to the step loop.  Their sines and
// cosines and their Box-Muller pairs are therefore one shared, called routine each
// (results are those of the same library calls).
struct SinCosD {
    double s, c;
};
static __device__ __noinline__ SinCosD sincos_d(double x) {
    SinCosD r;
    ::sincos(x, &r.s, &r.c);
    return r;
}
// one Box-Muller pair on the words (a, b): u = (w + 1/2) 2^-32, r = sqrt(-2 ln u_a),
// (r cos 2 pi u_b, r sin 2 pi u_b)
static __device__ __noinline__ SinCosD box_muller_pair_d(uint32_t a, uint32_t b) {
    const double inv = 2.3283064365386963e-10, half = 1.1641532182693481e-10;  // 2^-32, 2^-33
    const double u0 = fma(static_cast<double>(a), inv, half), u1 = fma(static_cast<double>(b), inv, half);
    const double r = ::sqrt(-2.0 * ::log(u0));
    double s, c;
    ::sincospi(2.0 * u1, &s, &c);
    return SinCosD{r * s, r * c};
}

template <> struct M<double> {
    // rare paths (chart rotations, the mixed-chart drift) are called, not inlined
    static constexpr bool kColdCalls = true;
    static constexpr bool kCompensatedState = false;  // FP64 resolves every increment
    static __device__ __forceinline__ double sin(double x) { return ::sin(x); }
    static __device__ __forceinline__ double cos(double x) { return ::cos(x); }
    static __device__ __forceinline__ void sincos(double x, double* s, double* c) {
        const SinCosD r = sincos_d(x);
        *s = r.s;
        *c = r.c;
    }
    static __device__ __forceinline__ double acos(double x) { return ::acos(x); }
    static __device__ __forceinline__ double atan2(double y, double x) { return ::atan2(y, x); }
    static __device__ __forceinline__ double fmod(double x, double y) { return ::fmod(x, y); }
    static __device__ __forceinline__ double sqrt(double x) { return ::sqrt(x); }
    static __device__ __forceinline__ double rcp(double x) { return 1.0 / x; }
    // 1/sin of the spherical angles: exact division in FP64
    static __device__ __forceinline__ double inv_sin(double x) { return 1.0 / x; }
    static __device__ __forceinline__ double abs(double x) { return ::fabs(x); }
    static __device__ __forceinline__ bool isinf(double x) { return ::isinf(x); }
    static __device__ __forceinline__ double zero_inf(double x) { return ::isinf(x) ? 0.0 : x; }
    static __device__ __forceinline__ bool finite(double x) { return ::isfinite(x); }
    static constexpr double two_pi = 6.283185307179586;
    static constexpr double eps = 2.220446049250313e-16;
};

template <> struct M<float> {
    static constexpr bool kColdCalls = false;
    // the slowly moving state components carry their rounding error (Stepper::explicit_from)
    static constexpr bool kCompensatedState = true;
    static __device__ __forceinline__ float sin(float x) { return __sinf(x); }
    static __device__ __forceinline__ float cos(float x) { return __cosf(x); }
    static __device__ __forceinline__ void sincos(float x, float* s, float* c) { __sincosf(x, s, c); }
    static __device__ __forceinline__ float acos(float x) { return ::acosf(x); }
    static __device__ __forceinline__ float atan2(float y, float x) { return ::atan2f(y, x); }
    static __device__ __forceinline__ float fmod(float x, float y) { return ::fmodf(x, y); }
    static __device__ __forceinline__ float sqrt(float x) { return ::sqrtf(x); }
    static __device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }
    // 1/sin of the spherical angles in the FP32 form: the SFU reciprocal (rcp.approx,
    // ~1 ulp) without the IEEE division's slow path; 1/0 stays +-inf
    static __device__ __forceinline__ float inv_sin(float x) {
        float r;
        asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
        return r;
    }
    static __device__ __forceinline__ float abs(float x) { return ::fabsf(x); }
    static __device__ __forceinline__ bool isinf(float x) { return ::isinf(x); }
    static __device__ __forceinline__ float zero_inf(float x) { return ::isinf(x) ? 0.0f : x; }
    static __device__ __forceinline__ bool finite(float x) { return ::isfinite(x); }
    static constexpr float two_pi = 6.283185307179586f;
    static constexpr float eps = 1.1920929e-7f;
};

// fmod(x, 2pi) without the software remainder loop: for |x| < 4pi the single
// subtraction x -/+ 2pi is exact (Sterbenz), so the result equals fmod bit for bit;
// larger arguments, which one step never produces, fall back to fmod.
template <class R>
__device__ __forceinline__ R wrap_two_pi(R x) {
    const R tp = M<R>::two_pi;
    if (M<R>::abs(x) < R(2) * tp) return x >= tp ? x - tp : (x <= -tp ? x + tp : x);
    return M<R>::fmod(x, tp);
}
// FP32 form: x - 2 pi trunc(x / 2 pi) in three instructions.  It equals the form above
// except where x / 2 pi rounds up to the next integer (x within an ulp below a multiple
// of 2 pi); there it returns the same angle less 2 pi.
template <>
__device__ __forceinline__ float wrap_two_pi<float>(float x) {
    return fmaf(-M<float>::two_pi, truncf(x * 0.159154943f), x);
}

template <class R>
struct V3 {
    R x, y, z;
};
// the value type an argument expression stands for (the paired form's unevaluated
// products name their result type here)
template <class T> struct real_of { using type = T; };
template <class A, class B, class C>
__device__ __forceinline__ V3<typename real_of<A>::type> v3(A a, B b, C c) {
    using R = typename real_of<A>::type;
    return V3<R>{R(a), R(b), R(c)};
}
template <class R> __device__ __forceinline__ V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> __device__ __forceinline__ V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> __device__ __forceinline__ V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> __device__ __forceinline__ R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> __device__ __forceinline__ V3<R> cross(V3<R> a, V3<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// ------------------------------------------------------------------ Philox4x32-10
// Counter-based generator of Salmon, Moraes, Dror and Shaw (SC'11).  Particle p
// at integrated step n draws
//   counter = {n_lo, n_hi, pid_lo, (pid_hi & 0xFFFFFF) | call << 24}, key = seed
// so the stream depends on neither launch shape, chunking nor co-scheduling.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

__device__ __forceinline__ uint4 philox_block(unsigned long long seed, unsigned long long pid, unsigned long long step,
                                              uint32_t call) {
    const uint4 c = make_uint4(static_cast<uint32_t>(step), static_cast<uint32_t>(step >> 32),
                               static_cast<uint32_t>(pid),
                               (static_cast<uint32_t>(pid >> 32) & 0xFFFFFFu) | (call << 24));
    return philox4x32_10(c, static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
}

// Box-Muller on u = (w + 1/2) 2^-32.  npairs = 1 or 2 pairs of normals.
// inlined form, for kernels whose step loop is small enough for the instruction cache
__device__ __forceinline__ void box_muller_inline(uint4 w, int npairs, double* z) {
    const double inv = 2.3283064365386963e-10, half = 1.1641532182693481e-10;  // 2^-32, 2^-33
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        if (k >= npairs) break;
        const uint32_t a = k ? w.z : w.x, b = k ? w.w : w.y;
        const double u0 = fma(static_cast<double>(a), inv, half), u1 = fma(static_cast<double>(b), inv, half);
        const double r = ::sqrt(-2.0 * ::log(u0));
        double s, c;
        ::sincospi(2.0 * u1, &s, &c);
        z[2 * k] = r * c;
        z[2 * k + 1] = r * s;
    }
}
__device__ __forceinline__ void box_muller(uint4 w, int npairs, double* z) {
    const SinCosD p = box_muller_pair_d(w.x, w.y);
    z[0] = p.c;
    z[1] = p.s;
    if (npairs > 1) {
        const SinCosD q = box_muller_pair_d(w.z, w.w);
        z[2] = q.c;
        z[3] = q.s;
    }
}
// sqrt of -2 ln u as x * rsqrt(x) on the SFU (rsqrt.approx, ~1 ulp).  In FP32,
// u = (w + 1/2) 2^-32 rounds to exactly 1 for the top 128 words, where -2 ln u is 0
// (and rsqrt(0) = inf); x is kept at or above 1e-30, which gives a radius of 1e-15.
__device__ __forceinline__ float sqrt_pos(float x) {
    x = fmaxf(x, 1e-30f);
    float r;
    asm("rsqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return x * r;
}
__device__ __forceinline__ void box_muller(uint4 w, int npairs, float* z) {
    const float inv = 2.3283064e-10f, half = 1.1641532e-10f;
    {
        const float u0 = fmaf(__uint2float_rn(w.x), inv, half), u1 = fmaf(__uint2float_rn(w.y), inv, half);
        const float r = sqrt_pos(-2.0f * __logf(u0));
        float s, c;
        __sincosf(6.2831853f * u1, &s, &c);
        z[0] = r * c;
        z[1] = r * s;
    }
    if (npairs > 1) {
        const float u2 = fmaf(__uint2float_rn(w.z), inv, half), u3 = fmaf(__uint2float_rn(w.w), inv, half);
        const float r = sqrt_pos(-2.0f * __logf(u2));
        float s, c;
        __sincosf(6.2831853f * u3, &s, &c);
        z[2] = r * c;
        z[3] = r * s;
    }
}

// m unit normals (m = 3 or 6) for (seed, pid, step) from Philox calls call0 and
// call0 + 1.  Calls 0-1 carry dW; Heun_NotConsistent's second increment takes
// calls 2-3, the double-noise draws of WeakTest / ExplicitStrong_1.0 calls 2-166.
template <class R, int Mdim>
__device__ __forceinline__ void philox_normals(unsigned long long seed, unsigned long long pid, unsigned long long step,
                                               R* z, uint32_t call0 = 0u) {
    R t[4];
    box_muller(philox_block(seed, pid, step, call0), 2, t);
    z[0] = t[0];
    z[1] = t[1];
    z[2] = t[2];
    if (Mdim > 3) {
        z[3] = t[3];
        R u[4];
        box_muller(philox_block(seed, pid, step, call0 + 1u), 1, u);
        z[4] = u[0];
        z[5] = u[1];
    }
}

// Wiener increments dW = sqrt(dt) z of one step (m = 3 or 6, calls 0-1).  FP64 scales
// the unit normals (CALLED: through the shared Box-Muller routine, for kernels whose
// physics already fills the instruction cache; else inlined, which keeps a small
// latency-bound step loop free of calls); FP32 folds dt into the Box-Muller radius,
// sqrt(-2 dt ln u), which saves the m multiplications.
template <class R, int Mdim, bool CALLED = true>
__device__ __forceinline__ void philox_increments(unsigned long long seed, unsigned long long pid,
                                                  unsigned long long step, R sqdt, R m2dt, R* w) {
    if constexpr (sizeof(R) == 8) {
        if constexpr (CALLED) {
            philox_normals<R, Mdim>(seed, pid, step, w);
        } else {
            double t[4];
            box_muller_inline(philox_block(seed, pid, step, 0u), 2, t);
            w[0] = t[0]; w[1] = t[1]; w[2] = t[2];
            if (Mdim > 3) {
                w[3] = t[3];
                box_muller_inline(philox_block(seed, pid, step, 1u), 1, t);
                w[4] = t[0]; w[5] = t[1];
            }
        }
#pragma unroll
        for (int j = 0; j < Mdim; ++j) w[j] = w[j] * sqdt;
    } else {
        const float inv = 2.3283064e-10f, half = 1.1641532e-10f;
        const uint4 a = philox_block(seed, pid, step, 0u);
        float r, s, c;
        r = sqrt_pos(m2dt * __logf(fmaf(__uint2float_rn(a.x), inv, half)));
        __sincosf(6.2831853f * fmaf(__uint2float_rn(a.y), inv, half), &s, &c);
        w[0] = r * c; w[1] = r * s;
        r = sqrt_pos(m2dt * __logf(fmaf(__uint2float_rn(a.z), inv, half)));
        __sincosf(6.2831853f * fmaf(__uint2float_rn(a.w), inv, half), &s, &c);
        w[2] = r * c;
        if (Mdim > 3) {
            w[3] = r * s;
            const uint4 b = philox_block(seed, pid, step, 1u);
            r = sqrt_pos(m2dt * __logf(fmaf(__uint2float_rn(b.x), inv, half)));
            __sincosf(6.2831853f * fmaf(__uint2float_rn(b.y), inv, half), &s, &c);
            w[4] = r * c; w[5] = r * s;
        }
    }
}

// B(t) in double: SinusoidalField.h:47-51 / LissajousField.h:98-101.  The phase
// products are rounded separately (no fused multiply-add) like the host code.
__device__ __forceinline__ void field_eval(const FieldParams& f, double t, double* B) {
    switch (f.type) {
        case 0:
            B[0] = B[1] = B[2] = 0.0;
            break;
        case 1:
            B[0] = f.offset[0]; B[1] = f.offset[1]; B[2] = f.offset[2];
            break;
        case 2: {
            const double s = ::sin(__dadd_rn(__dmul_rn(f.omega[0], t), f.phase[0]));
#pragma unroll
            for (int i = 0; i < 3; ++i) B[i] = __dadd_rn(__dmul_rn(f.amplitude[i], s), f.offset[i]);
            break;
        }
        case 3:
#pragma unroll
            for (int i = 0; i < 3; ++i)
                B[i] = __dadd_rn(f.offset[i], __dmul_rn(f.amplitude[i], ::sin(__dadd_rn(__dmul_rn(f.omega[i], t), f.phase[i]))));
            break;
        case 4: {  // TriangularField.h:52-70
            const double nt = __dadd_rn(t, f.time_offset);
            const double pos = nt < 0.0 ? __dadd_rn(f.periode, ::fmod(nt, f.periode)) : ::fmod(nt, f.periode);
            const double r = __ddiv_rn(__dmul_rn(2.0, pos), f.half_periode);
            const double w = pos > f.half_periode ? __dadd_rn(r, -1.0) : __dadd_rn(-r, 3.0);
#pragma unroll
            for (int i = 0; i < 3; ++i) B[i] = __dadd_rn(__dmul_rn(w, f.amplitude[i]), f.offset[i]);
            break;
        }
        case 5: {  // RectangularField.h:46-63
            const double nt = __dadd_rn(t, f.time_offset);
            const double pos = nt < 0.0 ? ::fmod(__dadd_rn(nt, f.periode), f.periode) : ::fmod(nt, f.periode);
            if (pos <= f.half_periode) {
                const double g = -::expm1(-__dmul_rn(pos, f.inv_tau));
#pragma unroll
                for (int i = 0; i < 3; ++i) B[i] = __dadd_rn(__dmul_rn(f.amplitude[i], g), f.offset[i]);
            } else {
                const double g = ::exp(-__dmul_rn(__dadd_rn(pos, -f.half_periode), f.inv_tau));
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    B[i] = __dadd_rn(__dadd_rn(__dmul_rn(f.amplitude[i], g), f.offset[i]),
                                     -__dadd_rn(f.amplitude[i], -f.max_field[i]));
            }
            break;
        }
        default: {  // 6, SincField.h:38-48: sinc(x) = sin(x)/x, 1 - x^2/6 + x^4/120 near 0
            const double pos = __dadd_rn(t < 0.0 ? ::fmod(__dadd_rn(t, f.periode), f.periode) : ::fmod(t, f.periode),
                                         -f.half_periode);
            const double x = __dmul_rn(__dmul_rn(3.14159265358979323846, f.sinc_a), pos);
            const double x2 = __dmul_rn(x, x);
            const double sc = ::fabs(x) < 1e-4 ? __dadd_rn(1.0, __dmul_rn(x2, __dadd_rn(-1.0 / 6.0, __dmul_rn(x2, 1.0 / 120.0))))
                                                : __ddiv_rn(::sin(x), x);
            const double s2 = __dmul_rn(sc, sc);
#pragma unroll
            for (int i = 0; i < 3; ++i) B[i] = __dadd_rn(__dmul_rn(f.amplitude[i], s2), f.offset[i]);
        }
    }
}

}  // namespace sp

// sp_physics.cuh — per-particle SDE right-hand sides and steppers (device code).
//
// One thread integrates one particle; every function works on registers.  The
// stochastic term is applied as b(y)·dW directly (the D x M matrix is never
// formed).  Reference formulas, by problem:
//   Neel (Cartesian LLG)      Problems/NeelRelaxation.h:92-190
//   Neel spherical            Problems/NeelRelaxationSpherical.h:124-516
//   Brown+Neel Euler/sph.     Problems/BrownAndNeelRelaxationEulerSpherical.h:141-735
//   Brown+Neel Cartesian      Problems/BrownAndNeelRelaxation.inl:40-270
//   uniaxial / cubic          Problems/Anisotropy/{Uniaxial,Cubic}Anisotropy.h
// and by solver (Stratonovich forms):
//   EulerMaruyama             SDEFramework/Solver/EulerMaruyama.inl:42-72
//   Heun_Strong               SDEFramework/Solver/Heun_Strong.inl:37-47
//   Millstein                 SDEFramework/Solver/Millstein.inl:35-44
//   Implicit_Midpoint         SDEFramework/Solver/Implicit_Midpoint.inl:40-105,175
// Per-particle prefactors are precomputed in FP64 by the init kernel and
// grouped so that FP32 never forms an overflowing product (c^2 ~ 1e48).
#pragma once

#include "sp_math.cuh"
#include "sp_types.h"

namespace sp {

template <class R>
struct Rot {
    bool rb, rn;          // rotation enabled (Neel spherical uses rb)
    R min1, max1, min2, max2;
};

// ------------------------------------------------------------------ chart rotations
// A chart rotation (coordinates within the configured angle of a pole) happens on few
// steps.  In the FP64 kernels its transcendental code is called, not inlined, so the
// per-step loop stays small enough for the instruction cache; FP32 inlines it.  The
// rotations return the new angles with their sines and cosines (what prepare needs next).
template <class R>
struct SphRot {
    R t, p, st, ct, sp, cp;
};
// NeelRelaxationSpherical.h:568-602 (INV: the inverse rotation)
template <class R, bool INV>
__device__ __forceinline__ SphRot<R> sph_rotate_impl(R t0, R p0) {
    R st, ct, sp, cp;
    M<R>::sincos(t0, &st, &ct);
    M<R>::sincos(p0, &sp, &cp);
    SphRot<R> r;
    if constexpr (!INV) {
        r.t = M<R>::acos(-cp * st); r.p = M<R>::atan2(sp * st, ct);
    } else {
        r.t = M<R>::acos(cp * st); r.p = M<R>::atan2(sp * st, -ct);
    }
    M<R>::sincos(r.t, &r.st, &r.ct);
    M<R>::sincos(r.p, &r.sp, &r.cp);
    return r;
}
template <class R, bool INV>
__device__ __noinline__ SphRot<R> sph_rotate_cold(R t0, R p0) { return sph_rotate_impl<R, INV>(t0, p0); }
template <class R, bool INV>
__device__ __forceinline__ SphRot<R> sph_rotate(R t0, R p0) {
    if constexpr (M<R>::kColdCalls) return sph_rotate_cold<R, INV>(t0, p0);
    else return sph_rotate_impl<R, INV>(t0, p0);
}
template <class R>
struct EulerRot {
    R e0, e1, e2, s0, s1, s2, c0, c1, c2;
};
// BrownAndNeelRelaxationEulerSpherical.h:859-899 (INV: the inverse rotation)
template <class R, bool INV>
__device__ __forceinline__ EulerRot<R> euler_rotate_impl(R a0, R a1, R a2) {
    R S0, C0, S1, C1, S2, C2;
    M<R>::sincos(a0, &S0, &C0); M<R>::sincos(a1, &S1, &C1); M<R>::sincos(a2, &S2, &C2);
    EulerRot<R> r;
    if constexpr (!INV) {
        r.e0 = M<R>::atan2(-C2 * C0 + C1 * S0 * S2, S0 * C2 + C1 * C0 * S2);
        r.e1 = M<R>::acos(-S1 * S2);
        r.e2 = M<R>::atan2(C1, C2 * S1);
    } else {
        r.e0 = M<R>::atan2(C0 * C2 - C1 * S0 * S2, -C2 * S0 - C1 * C0 * S2);
        r.e1 = M<R>::acos(S1 * S2);
        r.e2 = M<R>::atan2(-C1, C2 * S1);
    }
    M<R>::sincos(r.e0, &r.s0, &r.c0); M<R>::sincos(r.e1, &r.s1, &r.c1); M<R>::sincos(r.e2, &r.s2, &r.c2);
    return r;
}
template <class R, bool INV>
__device__ __noinline__ EulerRot<R> euler_rotate_cold(R a0, R a1, R a2) { return euler_rotate_impl<R, INV>(a0, a1, a2); }
template <class R, bool INV>
__device__ __forceinline__ EulerRot<R> euler_rotate(R a0, R a1, R a2) {
    if constexpr (M<R>::kColdCalls) return euler_rotate_cold<R, INV>(a0, a1, a2);
    else return euler_rotate_impl<R, INV>(a0, a1, a2);
}

// ------------------------------------------------------------------ anisotropy
template <class R, int A>
struct Aniso {
    // effective anisotropy field + external field
    static __device__ __forceinline__ V3<R> heff(R pF, V3<R> m, V3<R> x, V3<R> y, V3<R> z, V3<R> B) {
        if constexpr (A == kUniaxial) {
            return (pF * dot(m, z)) * z + B;  // UniaxialAnisotropy.h:140-144
        } else {                              // CubicAnisotropy.h:133-146
            const R c1 = dot(m, x), c2 = dot(m, y), c3 = dot(m, z);
            const R c1s = c1 * c1, c2s = c2 * c2, c3s = c3 * c3;
            return pF * (((c2s + c3s) * c1) * x + ((c1s + c3s) * c2) * y + ((c1s + c2s) * c3) * z) + B;
        }
    }
    // analytic dH/dm.  Uniaxial: pF z z^T (UniaxialAnisotropy.h:130-137, exact already).
    // Cubic: H = pF sum_i c_i (c_j^2 + c_k^2) a_i with c_i = m.a_i, so
    // dH/dm = pF sum_il G_il a_i a_l^T, G_ii = c_j^2 + c_k^2, G_il = 2 c_i c_l (the
    // reference returns the identity here, CubicAnisotropy.h:228-236).
    static __device__ __forceinline__ void jacobian(R pF, V3<R> m, V3<R> x, V3<R> y, V3<R> z, R J[3][3]) {
        if constexpr (A == kUniaxial) {
            const R zz[3] = {z.x, z.y, z.z};
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) J[i][j] = (pF * zz[i]) * zz[j];
        } else {
            const R c[3] = {dot(m, x), dot(m, y), dot(m, z)};
            const R a[3][3] = {{x.x, x.y, x.z}, {y.x, y.y, y.z}, {z.x, z.y, z.z}};  // a[i] = axis i
            R G[3][3];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int l = 0; l < 3; ++l)
                    G[i][l] = (i == l) ? (c[(i + 1) % 3] * c[(i + 1) % 3] + c[(i + 2) % 3] * c[(i + 2) % 3])
                                       : R(2) * c[i] * c[l];
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int col = 0; col < 3; ++col) {
                    R acc = R(0);
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int l = 0; l < 3; ++l) acc = acc + (G[i][l] * a[i][r]) * a[l][col];
                    J[r][col] = pF * acc;
                }
        }
    }
};

// Uniaxial+cubic (UniaxialCubicAnisotropy.hpp:95-133): the uniaxial part on the rotated
// axis zr = R^T z plus the cubic part on the body axes, then the external field.
template <class R>
__device__ __forceinline__ V3<R> heff_uniaxial_cubic(R pFu, V3<R> zr, R pFc, V3<R> m, V3<R> x, V3<R> y, V3<R> z, V3<R> B) {
    const V3<R> zero = v3(R(0), R(0), R(0));
    return (Aniso<R, kUniaxial>::heff(pFu, m, x, y, zr, zero) + Aniso<R, kCubic>::heff(pFc, m, x, y, z, zero)) + B;
}

// ======================================================================= Neel (Cartesian)
template <class R, int A>
struct NeelCart {
    static constexpr int D = 3, Mn = 3, OUT = 3;
    static constexpr bool kHasJacobian = true;
    static constexpr bool kCalledMath = false;  // FP64 Box-Muller through the shared routine
    struct Par {
        R NF1, NF2, Dp, pre1, pre2, pF, twoalpha;
        V3<R> z, x, y;
        R pF2;     // uniaxial+cubic: cubic field prefactor
        V3<R> zr;  // uniaxial+cubic: rotated uniaxial axis R^T z
    };
    struct Cache {};
    static __device__ __forceinline__ Par load(const R* P, unsigned long long Np, unsigned long long p) {
        Par q;
        q.NF1 = P[0 * Np + p]; q.NF2 = P[1 * Np + p]; q.Dp = P[2 * Np + p];
        q.pre1 = P[3 * Np + p]; q.pre2 = P[4 * Np + p]; q.pF = P[5 * Np + p]; q.twoalpha = P[6 * Np + p];
        q.z = v3(P[7 * Np + p], P[8 * Np + p], P[9 * Np + p]);
        if constexpr (A != kUniaxial) {
            q.x = v3(P[10 * Np + p], P[11 * Np + p], P[12 * Np + p]);
            q.y = v3(P[13 * Np + p], P[14 * Np + p], P[15 * Np + p]);
        } else {
            q.x = q.y = v3(R(0), R(0), R(0));
        }
        if constexpr (A == kUniaxialCubic) {
            q.pF2 = P[16 * Np + p];
            q.zr = v3(P[17 * Np + p], P[18 * Np + p], P[19 * Np + p]);
        } else {
            q.pF2 = R(0);
            q.zr = q.z;
        }
        return q;
    }
    static __device__ __forceinline__ V3<R> heff(const Par& q, V3<R> m, const R* B) {
        if constexpr (A == kUniaxialCubic) return heff_uniaxial_cubic(q.pF, q.zr, q.pF2, m, q.x, q.y, q.z, v3(B[0], B[1], B[2]));
        else return Aniso<R, A>::heff(q.pF, m, q.x, q.y, q.z, v3(B[0], B[1], B[2]));
    }
    static __device__ __forceinline__ void prepare(const Par&, const Rot<R>&, R*, Cache&) {}
    static __device__ __forceinline__ void recompute(const Par&, const R*, Cache&) {}
    static __device__ __forceinline__ void finish(const Rot<R>&, R*, const Cache&) {}
    static __device__ __forceinline__ int compensated(const Cache&) { return 0; }  // Neel increments are many ulp
    static __device__ __forceinline__ void det(const Par& q, const R* y, const Cache&, const R* B, R* a) {
        const V3<R> m = v3(y[0], y[1], y[2]);
        const V3<R> H = heff(q, m, B);
        const V3<R> mxH = cross(m, H);
        const V3<R> r = q.NF1 * mxH - q.NF2 * cross(m, mxH);
        a[0] = r.x; a[1] = r.y; a[2] = r.z;
    }
    static __device__ __forceinline__ void drift(const Par& q, const R* y, const Cache&, R* d) {
        d[0] = q.Dp * y[0]; d[1] = q.Dp * y[1]; d[2] = q.Dp * y[2];
    }
    // b(m)·w = pre2 (w - m (m·w)) + pre1 (m x w)          NeelRelaxation.h:92-109
    static __device__ __forceinline__ void bdw(const Par& q, const R* y, const Cache&, const R* w, R* r) {
        const V3<R> m = v3(y[0], y[1], y[2]), W = v3(w[0], w[1], w[2]);
        const V3<R> o = q.pre2 * (W - dot(m, W) * m) + q.pre1 * cross(m, W);
        r[0] = o.x; r[1] = o.y; r[2] = o.z;
    }
    static __device__ __forceinline__ void out(const R* y, R* o) { o[0] = y[0]; o[1] = y[1]; o[2] = y[2]; }
    // no angles: nothing to carry from one step's output to the next step's prepare
    struct Trig {};
    static __device__ __forceinline__ void trig(const R*, Trig&) {}
    static __device__ __forceinline__ void out_t(const R* y, R* o, Trig&) { out(y, o); }
    static __device__ __forceinline__ void prepare_t(const Par& q, const Rot<R>& r, R* y, Cache& c, const Trig&) {
        prepare(q, r, y, c);
    }
    // NeelRelaxation.h:204-208: m / |m| (Eigen normalize: unchanged when |m| = 0)
    static __device__ __forceinline__ void normalize(R* y) {
        const R n2 = (y[0] * y[0] + y[1] * y[1]) + y[2] * y[2];
        if (n2 > R(0)) {
            const R n = M<R>::sqrt(n2);
            y[0] = y[0] / n; y[1] = y[1] / n; y[2] = y[2] / n;
        }
    }
    // S = -I + dt/2 J_det + 1/2 J_sto with the reference Jacobians (NeelRelaxation.h:134-190):
    // J_det = NF1([m]x J_H - [H]x) - (2 alpha/dt)[m]x, J_sto = -pre1 [dW]x, J_H = pF z z^T (cubic: I)
    static __device__ __forceinline__ void newton_matrix(const Par& q, const R* y, const Cache&, const R* B, const R* w,
                                                         R dt, R S[D][D]) {
        const V3<R> m = v3(y[0], y[1], y[2]);
        const V3<R> H = heff(q, m, B);
        // uniaxial: pF z z^T; cubic: I; uniaxial+cubic: the sum, with the unrotated z
        // (UniaxialCubicAnisotropy.hpp:125-131)
        R JH[3][3];
        const R zz[3] = {q.z.x, q.z.y, q.z.z};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const R ju = (A != kCubic) ? (q.pF * zz[i]) * zz[j] : R(0);
                JH[i][j] = (A == kUniaxial) ? ju : (A == kCubic ? R(i == j ? 1 : 0) : ju + R(i == j ? 1 : 0));
            }
        const R mx[3][3] = {{R(0), -m.z, m.y}, {m.z, R(0), -m.x}, {-m.y, m.x, R(0)}};
        const R hx[3][3] = {{R(0), -H.z, H.y}, {H.z, R(0), -H.x}, {-H.y, H.x, R(0)}};
        const R wx[3][3] = {{R(0), -w[2], w[1]}, {w[2], R(0), -w[0]}, {-w[1], w[0], R(0)}};
        const R damp = q.twoalpha / dt;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                R mj = mx[i][0] * JH[0][j] + mx[i][1] * JH[1][j] + mx[i][2] * JH[2][j];
                const R jdet = q.NF1 * (mj - hx[i][j]) - damp * mx[i][j];
                const R jsto = -q.pre1 * wx[i][j];
                S[i][j] = (i == j ? R(-1) : R(0)) + (R(0.5) * dt) * jdet + R(0.5) * jsto;
            }
    }
    static constexpr bool kHasExactJacobian = true;
    // S = -I + dt/2 J_a + 1/2 J_b with the analytic Jacobians at the midpoint m:
    //   a = NF1 u - NF2 (m x u), u = m x H(m):  J_u = [m]x J_H - [H]x,
    //   J_a = NF1 J_u - NF2 ([m]x J_u - [u]x);
    //   b.w = pre2 (w - m (m.w)) + pre1 (m x w):  J_b = -pre2 ((m.w) I + m w^T) - pre1 [w]x.
    // Column j of [v]x is v x e_j.
    static __device__ __forceinline__ void newton_matrix_exact(const Par& q, const R* y, const Cache&, const R* B,
                                                               const R* w, R dt, R S[D][D]) {
        const V3<R> m = v3(y[0], y[1], y[2]);
        const V3<R> H = heff(q, m, B);
        R JH[3][3];
        if constexpr (A == kUniaxialCubic) {
            R J2[3][3];
            Aniso<R, kUniaxial>::jacobian(q.pF, m, q.x, q.y, q.zr, JH);
            Aniso<R, kCubic>::jacobian(q.pF2, m, q.x, q.y, q.z, J2);
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) JH[i][j] = JH[i][j] + J2[i][j];
        } else {
            Aniso<R, A>::jacobian(q.pF, m, q.x, q.y, q.z, JH);
        }
        const V3<R> u = cross(m, H);
        const V3<R> W = v3(w[0], w[1], w[2]);
        const R mw = dot(m, W);
        const R wv[3] = {w[0], w[1], w[2]};
        const R hdt = R(0.5) * dt;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const V3<R> ej = v3(R(j == 0), R(j == 1), R(j == 2));
            const V3<R> Ju = cross(m, v3(JH[0][j], JH[1][j], JH[2][j])) - cross(H, ej);
            const V3<R> Jv = cross(m, Ju) - cross(u, ej);
            const V3<R> Ja = q.NF1 * Ju - q.NF2 * Jv;
            const V3<R> Jb = (-q.pre2) * (mw * ej + wv[j] * m) - q.pre1 * cross(W, ej);
            S[0][j] = (j == 0 ? R(-1) : R(0)) + hdt * Ja.x + R(0.5) * Jb.x;
            S[1][j] = (j == 1 ? R(-1) : R(0)) + hdt * Ja.y + R(0.5) * Jb.y;
            S[2][j] = (j == 2 ? R(-1) : R(0)) + hdt * Ja.z + R(0.5) * Jb.z;
        }
    }
};

// ======================================================================= Neel (spherical)
template <class R, int A>
struct NeelSph {
    static constexpr int D = 2, Mn = 3, OUT = 3;
    static constexpr bool kHasJacobian = true;
    static constexpr bool kCalledMath = true;  // FP64 Box-Muller through the shared routine
    static constexpr bool kHasExactJacobian = false;
    struct Par {
        R NF1, NF2, Dp, DN, pF, twoalpha;
        V3<R> z, x, y;
        R pF2;     // uniaxial+cubic: cubic field prefactor
        V3<R> zr;  // uniaxial+cubic: rotated uniaxial axis R^T z
    };
    struct Cache {
        bool rot;
        R odst, st, ct;
        V3<R> md, eth, eph;
        V3<R> P0, P1;
    };
    static __device__ __forceinline__ Par load(const R* P, unsigned long long Np, unsigned long long p) {
        Par q;
        q.NF1 = P[0 * Np + p]; q.NF2 = P[1 * Np + p]; q.Dp = P[2 * Np + p]; q.DN = P[3 * Np + p];
        q.pF = P[4 * Np + p]; q.twoalpha = P[5 * Np + p];
        q.z = v3(P[6 * Np + p], P[7 * Np + p], P[8 * Np + p]);
        if constexpr (A != kUniaxial) {
            q.x = v3(P[9 * Np + p], P[10 * Np + p], P[11 * Np + p]);
            q.y = v3(P[12 * Np + p], P[13 * Np + p], P[14 * Np + p]);
        } else {
            q.x = q.y = v3(R(0), R(0), R(0));
        }
        if constexpr (A == kUniaxialCubic) {
            q.pF2 = P[15 * Np + p];
            q.zr = v3(P[16 * Np + p], P[17 * Np + p], P[18 * Np + p]);
        } else {
            q.pF2 = R(0);
            q.zr = q.z;
        }
        return q;
    }
    static __device__ __forceinline__ V3<R> heff(const Par& q, V3<R> m, const R* B) {
        if constexpr (A == kUniaxialCubic) return heff_uniaxial_cubic(q.pF, q.zr, q.pF2, m, q.x, q.y, q.z, v3(B[0], B[1], B[2]));
        else return Aniso<R, A>::heff(q.pF, m, q.x, q.y, q.z, v3(B[0], B[1], B[2]));
    }
    // NeelRelaxationSpherical.h:568-602
    static __device__ __forceinline__ void rotate(R* y) {
        const SphRot<R> r = sph_rotate<R, false>(y[0], y[1]);
        y[0] = r.t; y[1] = r.p;
    }
    static __device__ __forceinline__ void unrotate(R* y) {
        const SphRot<R> r = sph_rotate<R, true>(y[0], y[1]);
        y[0] = r.t; y[1] = r.p;
    }
    // :124-237
    static __device__ __forceinline__ void prepare(const Par& q, const Rot<R>& r, R* y, Cache& c) {
        c.rot = r.rb && (y[0] < r.min1 || y[0] > r.max1);
        if (c.rot) rotate(y);
        recompute(q, y, c);
    }
    static __device__ __forceinline__ void recompute(const Par& q, const R* y, Cache& c) {
        R st, ct, sp, cp;
        M<R>::sincos(y[0], &st, &ct);
        M<R>::sincos(y[1], &sp, &cp);
        cache_from(q, st, ct, sp, cp, c);
    }
    // sines and cosines of theta and phi of the state the previous step ended in: the
    // output of step n is evaluated at exactly the state step n+1 prepares, so its
    // sincos are reused whenever prepare keeps the chart (bit-identical to recomputing)
    struct Trig {
        R st, ct, sp, cp;
    };
    static __device__ __forceinline__ void trig(const R* y, Trig& t) {
        M<R>::sincos(y[0], &t.st, &t.ct);
        M<R>::sincos(y[1], &t.sp, &t.cp);
    }
    static __device__ __forceinline__ void out_t(const R* y, R* o, Trig& t) {
        trig(y, t);
        o[0] = t.st * t.cp; o[1] = t.st * t.sp; o[2] = t.ct;
    }
    static __device__ __forceinline__ void prepare_t(const Par& q, const Rot<R>& r, R* y, Cache& c, const Trig& t) {
        c.rot = r.rb && (y[0] < r.min1 || y[0] > r.max1);
        if (c.rot) {
            const SphRot<R> n = sph_rotate<R, false>(y[0], y[1]);
            y[0] = n.t; y[1] = n.p;
            cache_from(q, n.st, n.ct, n.sp, n.cp, c);
        } else {
            cache_from(q, t.st, t.ct, t.sp, t.cp, c);
        }
    }
    static __device__ __forceinline__ void cache_from(const Par& q, R st, R ct, R sp, R cp, Cache& c) {
        c.st = st; c.ct = ct;
        const R odst = M<R>::zero_inf(M<R>::inv_sin(st));
        c.odst = odst;
        if (!c.rot) {
            c.md = v3(st * cp, st * sp, ct);
            c.eth = v3(ct * cp, ct * sp, -st);
            c.eph = v3(-sp, cp, R(0));
        } else {
            c.md = v3(-ct, st * sp, st * cp);
            c.eth = v3(st, ct * sp, ct * cp);
            c.eph = v3(R(0), cp, -sp);
        }
        c.P0 = (-q.NF1) * c.eph + q.NF2 * c.eth;
        c.P1 = odst * (q.NF1 * c.eth + q.NF2 * c.eph);
        if (odst == R(0)) {
            if (!c.rot) c.P1.z = q.NF1;
            else c.P1.x = -q.NF1;
        }
    }
    static __device__ __forceinline__ void finish(const Rot<R>&, R* y, const Cache& c) {
        if (c.rot) unrotate(y);
        else { y[0] = wrap_two_pi(y[0]); y[1] = wrap_two_pi(y[1]); }
    }
    static __device__ __forceinline__ int compensated(const Cache&) { return 0; }
    static __device__ __forceinline__ void det(const Par& q, const R*, const Cache& c, const R* B, R* a) {
        const V3<R> H = heff(q, c.md, B);
        a[0] = dot(c.P0, H);
        a[1] = dot(c.P1, H);
    }
    static __device__ __forceinline__ void drift(const Par& q, const R*, const Cache& c, R* d) {
        const R cos_t = c.rot ? -c.md.x : c.md.z;
        d[0] = R(-0.5) * q.Dp * cos_t * c.odst;
        d[1] = R(0);
    }
    static __device__ __forceinline__ void bdw(const Par& q, const R*, const Cache& c, const R* w, R* r) {
        const V3<R> W = v3(w[0], w[1], w[2]);
        r[0] = q.DN * dot(c.P0, W);
        r[1] = q.DN * dot(c.P1, W);
    }
    static __device__ __forceinline__ void out(const R* y, R* o) {
        R st, ct, sp, cp;
        M<R>::sincos(y[0], &st, &ct);
        M<R>::sincos(y[1], &sp, &cp);
        o[0] = st * cp; o[1] = st * sp; o[2] = ct;
    }
    static __device__ __forceinline__ void normalize(R*) {}  // NeelRelaxationSpherical.h:534-537
    // NeelRelaxationSpherical.h:312-432 and finishJacobiCalculations :473-497
    static __device__ __forceinline__ void newton_matrix(const Par& q, const R*, const Cache& c, const R* B, const R* w,
                                                         R dt, R S[D][D]) {
        const R cos_t = c.rot ? -c.md.x : c.md.z;
        const R sin_t = c.rot ? c.eth.x : -c.eth.z;
        const V3<R> Jer0 = c.eth, Jer1 = sin_t * c.eph;
        const V3<R> Jth0 = (R(-1)) * c.md, Jth1 = cos_t * c.eph;
        const V3<R> Jph0 = v3(R(0), R(0), R(0));
        const V3<R> Jph1 = c.rot ? v3(R(0), c.eph.z, -c.eph.y) : v3(-c.eph.y, c.eph.x, R(0));
        const V3<R> H = heff(q, c.md, B);
        const R a = q.NF1, b = q.NF2;
        // J_H J_er^T columns (3-vectors), c = 0, 1; J_H as in the reference: uniaxial
        // pF z z^T, cubic I, uniaxial+cubic their sum with the unrotated z
        V3<R> HJer[2];
        const V3<R> Jer[2] = {Jer0, Jer1};
        for (int k = 0; k < 2; ++k) {
            if constexpr (A == kUniaxial) HJer[k] = (q.pF * dot(q.z, Jer[k])) * q.z;
            else if constexpr (A == kCubic) HJer[k] = Jer[k];
            else HJer[k] = (q.pF * dot(q.z, Jer[k])) * q.z + Jer[k];
        }
        const V3<R> A0[2] = {(-a) * Jph0 + b * Jth0, (-a) * Jph1 + b * Jth1};  // rows of (-a J_phi + b J_theta)
        const V3<R> B1[2] = {c.odst * (a * Jth0 + b * Jph0), c.odst * (a * Jth1 + b * Jph1)};
        const V3<R> ab = a * c.eth + b * c.eph;
        const R jst = c.odst * c.odst * cos_t;
        const V3<R> W = v3(w[0], w[1], w[2]);
        R Jd[2][2], Js[2][2];
        for (int k = 0; k < 2; ++k) {
            Jd[0][k] = dot(A0[k], H) + dot(c.P0, HJer[k]);
            Js[0][k] = q.DN * dot(A0[k], W);
            const V3<R> rowk = (k == 0) ? B1[0] - jst * ab : B1[1];
            // (P1 J_H) J_er^T
            V3<R> P1JH;
            if constexpr (A == kUniaxial) P1JH = (q.pF * dot(c.P1, q.z)) * q.z;
            else if constexpr (A == kCubic) P1JH = c.P1;
            else P1JH = (q.pF * dot(c.P1, q.z)) * q.z + c.P1;
            Jd[1][k] = dot(H, rowk) + dot(P1JH, Jer[k]);
            Js[1][k] = q.DN * dot(W, rowk);
        }
        for (int i = 0; i < 2; ++i)
            for (int k = 0; k < 2; ++k) S[i][k] = (i == k ? R(-1) : R(0)) + (R(0.5) * dt) * Jd[i][k] + R(0.5) * Js[i][k];
        if (c.rot) {
            const R m_cos_t = c.md.x, sin_t2 = c.eth.x, cos_p = c.eph.y, m_sin_p = c.eph.z;
            const R factor = R(1) / M<R>::sqrt(R(1) - sin_t2 * sin_t2 * cos_p * cos_p);
            const R J00 = factor * m_cos_t * cos_p, J01 = m_sin_p;
            const R J10 = -factor * c.odst * m_sin_p, J11 = c.odst * m_cos_t * cos_p;
            for (int i = 0; i < 2; ++i) {
                const R s0 = S[i][0], s1 = S[i][1];
                S[i][0] = s0 * J00 + s1 * J10;
                S[i][1] = s0 * J01 + s1 * J11;
            }
        }
    }
};

// BrownAndNeelRelaxationEulerSpherical.h:559-594: the drift when exactly one of the two
// charts is rotated (a rare step; called, not inlined, in FP64)
template <class R>
__device__ __forceinline__ V3<R> be_drift_mixed_impl(bool br, R adDN2, R d2fDN2, R cF2h, R csc, R ctheta, R cpsi,
                                                     R spsi, R cos_t, R cos_p, R sin_t, R sin_p) {
    const R cotb = csc * ctheta;
    V3<R> r;
    const R sin_2t = R(2) * cos_t * sin_t;
    const R sin_t_2 = sin_t * sin_t;
    const R cpsi_2 = cpsi * cpsi, spsi_2 = spsi * spsi;
    const R c2psi = cpsi_2 - spsi_2, s2psi = R(2) * cpsi * spsi;
    const R sin_2p = R(2) * cos_p * sin_p;
    const R cos_t_2 = cos_t * cos_t, sin_p_2 = sin_p * sin_p, cos_p_2 = cos_p * cos_p;
    if (br) {  // :559-576
        r.x = csc * (adDN2 * (-spsi * cos_t + sin_p * cpsi * sin_t) +
                      R(2) * d2fDN2 * (-c2psi * cotb * sin_2t * sin_p + cos_p * sin_t * (cos_t * cpsi + sin_t * sin_p * spsi) +
                                         cotb * s2psi * (cos_t_2 - sin_t_2 * sin_p_2)));
        r.y = cF2h * cotb + adDN2 * (-cos_t * cpsi - spsi * sin_t * sin_p) +
               d2fDN2 * (R(2) * cpsi_2 * cotb * (cos_t_2 + cos_p_2 * sin_t_2) + cpsi * sin_t_2 * sin_2p +
                           R(2) * spsi * (-sin_t * cos_t * cos_p + cotb * sin_t_2 * spsi) + cotb * sin_2t * sin_p * s2psi);
        r.z = adDN2 * (sin_t * cos_p - cpsi * cotb * sin_t * sin_p + cotb * cos_t * spsi) -
               d2fDN2 * (cos_t * cpsi + sin_t * sin_p * spsi) *
                   (R(2) * cos_p * cotb * sin_t - (R(3) + c2psi) * csc * csc * (cpsi * sin_t * sin_p - cos_t * spsi));
    } else {  // only Neel rotated, :577-594
        r.x = csc * (adDN2 * (spsi * cos_t + sin_p * cpsi * sin_t) +
                      R(2) * d2fDN2 * (c2psi * cotb * sin_2t * sin_p + cos_p * sin_t * (cos_t * cpsi - sin_t * sin_p * spsi) +
                                         cotb * s2psi * (cos_t_2 - sin_t_2 * sin_p_2)));
        r.y = cF2h * cotb + adDN2 * (cos_t * cpsi - spsi * sin_t * sin_p) +
               d2fDN2 * (R(2) * cpsi_2 * cotb * (cos_t_2 + cos_p_2 * sin_t_2) - cpsi * sin_t_2 * sin_2p +
                           R(2) * spsi * (-sin_t * cos_t * cos_p + cotb * sin_t_2 * spsi) - cotb * sin_2t * sin_p * s2psi);
        r.z = adDN2 * (-sin_t * cos_p - cpsi * cotb * sin_t * sin_p - cotb * cos_t * spsi) -
               d2fDN2 * (cos_t * cpsi - sin_t * sin_p * spsi) *
                   (R(2) * cos_p * cotb * sin_t + (R(3) + c2psi) * csc * csc * (cpsi * sin_t * sin_p + cos_t * spsi));
    }
    return r;
}
template <class R>
__device__ __noinline__ V3<R> be_drift_mixed_cold(bool br, R adDN2, R d2fDN2, R cF2h, R csc, R ctheta, R cpsi, R spsi,
                                                  R cos_t, R cos_p, R sin_t, R sin_p) {
    return be_drift_mixed_impl<R>(br, adDN2, d2fDN2, cF2h, csc, ctheta, cpsi, spsi, cos_t, cos_p, sin_t, sin_p);
}

// ======================================================================= Brown + Neel, Euler/spherical
template <class R, int A>
struct BrownNeelEuler {
    static constexpr int D = 5, Mn = 6, OUT = 9;
    static constexpr bool kHasJacobian = false;  // assert(false) in the reference (:605-626)
    static constexpr bool kCalledMath = true;  // FP64 Box-Muller through the shared routine
    static constexpr bool kHasExactJacobian = false;
    struct Par {
        R a, bpd, d, cT, pF, cF, dDN, bpdDN, aDN, adDN2, d2fDN2, cF2h, nd;
        R pF2, cT2;  // uniaxial+cubic: cubic field and torque prefactors
        R Rm[9];     // uniaxial+cubic: rotation of the uniaxial part, row-major
    };
    struct Cache {
        bool br, nr;
        R S[5], C[5];
        R csc, odst;
        V3<R> md;
    };
    // get(i): prefactor i of the particle (one lane each in the paired form)
    template <class G>
    static __device__ __forceinline__ Par load_with(G get) {
        Par q;
        q.a = get(0); q.bpd = get(1); q.d = get(2); q.cT = get(3);
        q.pF = get(4); q.cF = get(5); q.dDN = get(6); q.bpdDN = get(7);
        q.aDN = get(8); q.adDN2 = get(9); q.d2fDN2 = get(10); q.cF2h = get(11);
        q.nd = get(12);
        if constexpr (A == kUniaxialCubic) {
            q.pF2 = get(13);
            q.cT2 = get(14);
#pragma unroll
            for (int i = 0; i < 9; ++i) q.Rm[i] = get(15 + i);
        }
        return q;
    }
    static __device__ __forceinline__ Par load(const R* P, unsigned long long Np, unsigned long long p) {
        return load_with([&](int i) { return P[i * Np + p]; });
    }
    // :859-899
    static __device__ __forceinline__ void euler_rotate(R* e) {
        const EulerRot<R> r = sp::euler_rotate<R, false>(e[0], e[1], e[2]);
        e[0] = r.e0; e[1] = r.e1; e[2] = r.e2;
    }
    static __device__ __forceinline__ void euler_unrotate(R* e) {
        const EulerRot<R> r = sp::euler_rotate<R, true>(e[0], e[1], e[2]);
        e[0] = r.e0; e[1] = r.e1; e[2] = r.e2;
    }
    static __device__ __forceinline__ void neel_rotate(R* y) { NeelSph<R, A>::rotate(y); }
    static __device__ __forceinline__ void neel_unrotate(R* y) { NeelSph<R, A>::unrotate(y); }
    // :141-361
    static __device__ __forceinline__ void prepare(const Par& q, const Rot<R>& r, R* y, Cache& c) {
        const R tb = M<R>::abs(y[1]);
        c.br = r.rb && (tb < r.min1 || tb > r.max1);
        if (c.br) euler_rotate(y);
        const R tn = M<R>::abs(y[3]);
        c.nr = r.rn && (tn < r.min2 || tn > r.max2);
        if (c.nr) neel_rotate(y + 3);
        recompute(q, y, c);
    }
    static __device__ __forceinline__ void recompute(const Par&, const R* y, Cache& c) {
#pragma unroll
        for (int i = 0; i < 5; ++i) M<R>::sincos(y[i], &c.S[i], &c.C[i]);
        cache_from(c);
    }
    // sines and cosines of the five angles the previous step ended in (its output is
    // evaluated there); reused by prepare for every angle whose chart it keeps
    struct Trig {
        R S[5], C[5];
    };
    static __device__ __forceinline__ void trig(const R* y, Trig& t) {
#pragma unroll
        for (int i = 0; i < 5; ++i) M<R>::sincos(y[i], &t.S[i], &t.C[i]);
    }
    static __device__ __forceinline__ void prepare_t(const Par& q, const Rot<R>& r, R* y, Cache& c, const Trig& t) {
        const R tb = M<R>::abs(y[1]), tn = M<R>::abs(y[3]);
        prepare_flags(q, y, c, t, r.rb && (tb < r.min1 || tb > r.max1), r.rn && (tn < r.min2 || tn > r.max2));
    }
    // prepare_t with the charts given: br (Euler angles rotated), nr (Neel angles rotated)
    static __device__ __forceinline__ void prepare_flags(const Par&, R* y, Cache& c, const Trig& t, bool br, bool nr) {
        c.br = br;
        if (c.br) {
            const EulerRot<R> n = sp::euler_rotate<R, false>(y[0], y[1], y[2]);
            y[0] = n.e0; y[1] = n.e1; y[2] = n.e2;
            c.S[0] = n.s0; c.S[1] = n.s1; c.S[2] = n.s2; c.C[0] = n.c0; c.C[1] = n.c1; c.C[2] = n.c2;
        } else {
#pragma unroll
            for (int i = 0; i < 3; ++i) { c.S[i] = t.S[i]; c.C[i] = t.C[i]; }
        }
        c.nr = nr;
        if (c.nr) {
            const SphRot<R> n = sph_rotate<R, false>(y[3], y[4]);
            y[3] = n.t; y[4] = n.p;
            c.S[3] = n.st; c.C[3] = n.ct; c.S[4] = n.sp; c.C[4] = n.cp;
        } else {
#pragma unroll
            for (int i = 3; i < 5; ++i) { c.S[i] = t.S[i]; c.C[i] = t.C[i]; }
        }
        cache_from(c);
    }
    static __device__ __forceinline__ void cache_from(Cache& c) {
        c.csc = M<R>::zero_inf(M<R>::inv_sin(c.S[1]));
        c.odst = M<R>::zero_inf(M<R>::inv_sin(c.S[3]));
        const R ct = c.C[3], cp = c.C[4], st = c.S[3], sp = c.S[4];
        c.md = c.nr ? v3(-ct, st * sp, st * cp) : v3(st * cp, st * sp, ct);
    }
    // body axes (columns of the cached Euler rotation matrix, :183-304)
    static __device__ __forceinline__ void axes(const Cache& c, V3<R>& x, V3<R>& y, V3<R>& z) {
        const R cphi = c.C[0], ctheta = c.C[1], cpsi = c.C[2], sphi = c.S[0], stheta = c.S[1], spsi = c.S[2];
        const R cphicpsi = cphi * cpsi, sphicpsi = sphi * cpsi, cphispsi = cphi * spsi, sphispsi = sphi * spsi;
        if (!c.br) {
            x = v3(cphicpsi - ctheta * sphispsi, ctheta * sphicpsi + cphispsi, stheta * sphi);
            y = v3(-sphicpsi - ctheta * cphispsi, ctheta * cphicpsi - sphispsi, stheta * cphi);
            z = v3(stheta * spsi, -stheta * cpsi, ctheta);
        } else {
            x = v3(-stheta * sphi, ctheta * sphicpsi + cphispsi, cphicpsi - ctheta * sphispsi);
            y = v3(-stheta * cphi, ctheta * cphicpsi - sphispsi, -sphicpsi - ctheta * cphispsi);
            z = v3(-ctheta, -stheta * cpsi, stheta * spsi);
        }
    }
    // E313^-1 applied to v (EulerProjectionMatrix, :228-237 and :293-302)
    static __device__ __forceinline__ V3<R> eproj(const Cache& c, V3<R> v) {
        const R ctheta = c.C[1], cpsi = c.C[2], spsi = c.S[2], csc = c.csc;
        if (!c.br)
            return v3(spsi * csc * v.x - cpsi * csc * v.y, cpsi * v.x + spsi * v.y,
                      -(ctheta * spsi) * csc * v.x + (ctheta * cpsi) * csc * v.y + v.z);
        return v3(-cpsi * csc * v.y + spsi * csc * v.z, spsi * v.y + cpsi * v.z,
                  -v.x + (ctheta * cpsi) * csc * v.y - (ctheta * spsi) * csc * v.z);
    }
    // spherical projection (:324-329 and :354-359), 2 rows applied to v
    static __device__ __forceinline__ void sproj(const Cache& c, V3<R> v, R* o) {
        const R ct = c.C[3], cp = c.C[4], sp = c.S[4], od = c.odst;
        if (!c.nr) {
            o[0] = -sp * v.x + cp * v.y;
            o[1] = -(cp * ct * od) * v.x - (sp * ct * od) * v.y + v.z;
        } else {
            o[0] = cp * v.y - sp * v.z;
            o[1] = -v.x - (sp * ct * od) * v.y - (cp * ct * od) * v.z;
        }
    }
    // c*Teff of the cubic part (CubicAnisotropy.h:162-193)
    static __device__ __forceinline__ V3<R> ctorque_cubic(R cT, const Cache& c, V3<R> m, V3<R> x, V3<R> y, V3<R> z) {
        const R c1 = dot(m, x), c2 = dot(m, y), c3 = dot(m, z);
        const R c1s = c1 * c1, c2s = c2 * c2;
        const R ctheta = c.C[1], cpsi = c.C[2], stheta = c.S[1], spsi = c.S[2];
        const V3<R> th = v3(ctheta * spsi, -ctheta * cpsi, -stheta);
        const V3<R> sym = cross(z, (c3 * (c1s + c2s)) * m);
        const V3<R> asdir = (ctheta / stheta) * th + z;
        return cT * (sym + (c1 * c2 * (c2s - c1s)) * asdir);
    }
    static __device__ __forceinline__ V3<R> rot_apply(const Par& q, V3<R> v) {  // R v
        return v3(q.Rm[0] * v.x + q.Rm[1] * v.y + q.Rm[2] * v.z, q.Rm[3] * v.x + q.Rm[4] * v.y + q.Rm[5] * v.z,
                  q.Rm[6] * v.x + q.Rm[7] * v.y + q.Rm[8] * v.z);
    }
    static __device__ __forceinline__ V3<R> rot_apply_t(const Par& q, V3<R> v) {  // R^T v
        return v3(q.Rm[0] * v.x + q.Rm[3] * v.y + q.Rm[6] * v.z, q.Rm[1] * v.x + q.Rm[4] * v.y + q.Rm[7] * v.z,
                  q.Rm[2] * v.x + q.Rm[5] * v.y + q.Rm[8] * v.z);
    }
    // c*Teff: uniaxial (UniaxialAnisotropy.h:146-150), cubic, or uniaxial+cubic, whose
    // uniaxial torque is taken of R m on the unrotated axis (UniaxialCubicAnisotropy.hpp:112-121)
    static __device__ __forceinline__ V3<R> ctorque(const Par& q, const Cache& c, V3<R> m, V3<R> x, V3<R> y, V3<R> z) {
        if constexpr (A == kUniaxial) {
            return (q.cT * dot(m, z)) * cross(z, m);
        } else if constexpr (A == kCubic) {
            return ctorque_cubic(q.cT, c, m, x, y, z);
        } else {
            const V3<R> rm = rot_apply(q, m);
            return (q.cT * dot(rm, z)) * cross(z, rm) + ctorque_cubic(q.cT2, c, m, x, y, z);
        }
    }
    static __device__ __forceinline__ V3<R> heff(const Par& q, V3<R> m, V3<R> x, V3<R> y, V3<R> z, const R* B) {
        if constexpr (A == kUniaxialCubic)
            return heff_uniaxial_cubic(q.pF, rot_apply_t(q, z), q.pF2, m, x, y, z, v3(B[0], B[1], B[2]));
        else return Aniso<R, A>::heff(q.pF, m, x, y, z, v3(B[0], B[1], B[2]));
    }
    // the Euler angles of the particle (Brown rotation: a few ulp of FP32 angles per step),
    // while their chart is not rotated
    static __device__ __forceinline__ int compensated(const Cache& c) { return c.br ? 0 : 3; }
    static __device__ __forceinline__ void finish(const Rot<R>&, R* y, const Cache& c) {
        if (c.br) euler_unrotate(y);
        else { y[0] = wrap_two_pi(y[0]); y[1] = wrap_two_pi(y[1]); y[2] = wrap_two_pi(y[2]); }
        if (c.nr) neel_unrotate(y + 3);
        else { y[3] = wrap_two_pi(y[3]); y[4] = wrap_two_pi(y[4]); }
    }
    // :363-425
    static __device__ __forceinline__ void det(const Par& q, const R*, const Cache& c, const R* B, R* a) {
        V3<R> x, y, z;
        axes(c, x, y, z);
        const V3<R> H = heff(q, c.md, x, y, z, B);
        const V3<R> cTe = ctorque(q, c, c.md, x, y, z);
        const V3<R> mxH = cross(c.md, H);
        const V3<R> wb = eproj(c, cTe + q.d * mxH);
        a[0] = wb.x; a[1] = wb.y; a[2] = wb.z;
        sproj(c, (-q.a) * H + q.bpd * mxH + cTe, a + 3);
    }
    // :427-497 applied to w = (wA, wB)
    static __device__ __forceinline__ void bdw(const Par& q, const R*, const Cache& c, const R* w, R* r) {
        const V3<R> wA = v3(w[0], w[1], w[2]), wB = v3(w[3], w[4], w[5]);
        const V3<R> cwA = q.cF * wA;
        const V3<R> mxw = cross(c.md, wB);  // shared by both rows
        const V3<R> b = eproj(c, cwA + q.dDN * mxw);
        r[0] = b.x; r[1] = b.y; r[2] = b.z;
        sproj(c, cwA + q.bpdDN * mxw - q.aDN * wB, r + 3);
    }
    // :499-601 with the prefactors grouped: adDN2 = a d DN^2, d2fDN2 = d^2 DN^2 / 4, cF2h = (c DB)^2 / 2
    static __device__ __forceinline__ void drift(const Par& q, const R* y, const Cache& c, R* r) {
        const R ctheta = c.C[1], cpsi = c.C[2], spsi = c.S[2];
        const R cos_t = c.C[3], cos_p = c.C[4], sin_t = c.S[3], sin_p = c.S[4];
        const R csc = c.csc;
        const R cotb = csc * ctheta;
        if (c.br == c.nr) {
            const R cos_2t = cos_t * cos_t - sin_t * sin_t;
            const R sin_2t = R(2) * cos_t * sin_t;
            const R sin_t_2 = sin_t * sin_t;
            const R cph = cos_p * cpsi + spsi * sin_p;  // cos(phi_N - psi)
            const R sph = cpsi * sin_p - cos_p * spsi;  // sin(phi_N - psi)
            // sin and cos of 2 (phi_N - psi) by the double-angle identities
            const R s2 = R(2) * sph * cph, c2 = cph * cph - sph * sph;
            r[0] = csc * sin_t * (q.adDN2 * sph - R(2) * q.d2fDN2 * (cos_t * cph + cotb * sin_t * s2));
            r[1] = q.cF2h * cotb - q.adDN2 * (cph * sin_t) +
                   q.d2fDN2 * (R(0.5) * (R(3) + cos_2t + R(2) * c2 * sin_t_2) * cotb - sin_2t * sph);
            r[2] = -(q.adDN2 * (cos_t + sin_t * cotb * sph) -
                     q.d2fDN2 * sin_t * (R(2) * cos_t * cotb * cph + (R(-1) + R(2) * csc * csc) * sin_t * s2));
        } else {
            V3<R> m;
            if constexpr (M<R>::kColdCalls)
                m = be_drift_mixed_cold<R>(c.br, q.adDN2, q.d2fDN2, q.cF2h, csc, ctheta, cpsi, spsi, cos_t, cos_p, sin_t, sin_p);
            else
                m = be_drift_mixed_impl<R>(c.br, q.adDN2, q.d2fDN2, q.cF2h, csc, ctheta, cpsi, spsi, cos_t, cos_p, sin_t, sin_p);
            r[0] = m.x; r[1] = m.y; r[2] = m.z;
        }
        r[3] = q.nd * c.odst * cos_t;  // :597
        r[4] = R(0);
    }
    // :673-735: x-axis, y-axis, magnetisation
    static __device__ __forceinline__ void out_t(const R* y, R* o, Trig& t) {
        trig(y, t);
        const R* s = t.S;
        const R* c = t.C;
        const R cphicpsi = c[0] * c[2], sphicpsi = s[0] * c[2], cphispsi = c[0] * s[2], sphispsi = s[0] * s[2];
        o[0] = cphicpsi - c[1] * sphispsi; o[1] = c[1] * sphicpsi + cphispsi; o[2] = s[1] * s[0];
        o[3] = -sphicpsi - c[1] * cphispsi; o[4] = c[1] * cphicpsi - sphispsi; o[5] = s[1] * c[0];
        o[6] = s[3] * c[4]; o[7] = s[3] * s[4]; o[8] = c[3];
    }
    static __device__ __forceinline__ void out(const R* y, R* o) {
        Trig t;
        out_t(y, o, t);
    }
    static __device__ __forceinline__ void normalize(R*) {}  // BrownAndNeelRelaxationEulerSpherical.h:738-741
    static __device__ __forceinline__ void newton_matrix(const Par&, const R*, const Cache&, const R*, const R*, R,
                                                         R S[D][D]) {
        for (int i = 0; i < D; ++i) for (int j = 0; j < D; ++j) S[i][j] = R(i == j ? -1 : 0);
    }
};

// ======================================================================= Brown + Neel (Cartesian)
template <class R, int A>
struct BrownNeelCart {
    static constexpr int D = 6, Mn = 6, OUT = 6;
    static constexpr bool kHasJacobian = true;  // both Jacobians are zero in the reference (.h:119-128)
    static constexpr bool kCalledMath = false;  // FP64 Box-Muller through the shared routine
    static constexpr bool kHasExactJacobian = false;
    struct Par {
        R a, bpd, d, cT, pF, cF, dDN, bpdDN, aDN, cF2, adDN2, hd2DN2, ndrift, cFe;
    };
    struct Cache {};
    static __device__ __forceinline__ Par load(const R* P, unsigned long long Np, unsigned long long p) {
        Par q;
        q.a = P[0 * Np + p]; q.bpd = P[1 * Np + p]; q.d = P[2 * Np + p]; q.cT = P[3 * Np + p];
        q.pF = P[4 * Np + p]; q.cF = P[5 * Np + p]; q.dDN = P[6 * Np + p]; q.bpdDN = P[7 * Np + p];
        q.aDN = P[8 * Np + p]; q.cF2 = P[9 * Np + p]; q.adDN2 = P[10 * Np + p]; q.hd2DN2 = P[11 * Np + p];
        q.ndrift = P[12 * Np + p]; q.cFe = P[13 * Np + p];
        return q;
    }
    static __device__ __forceinline__ void prepare(const Par&, const Rot<R>&, R*, Cache&) {}
    static __device__ __forceinline__ void recompute(const Par&, const R*, Cache&) {}
    static __device__ __forceinline__ void finish(const Rot<R>&, R*, const Cache&) {}
    static __device__ __forceinline__ int compensated(const Cache&) { return 3; }  // the particle axis n
    // .inl:222-271 (the reference returns zero for cubic anisotropy, .inl:225-229)
    static __device__ __forceinline__ void det(const Par& q, const R* y, const Cache&, const R* B, R* a) {
        if constexpr (A == kCubic) {
            for (int i = 0; i < 6; ++i) a[i] = R(0);
        } else {
            const V3<R> n = v3(y[0], y[1], y[2]), e = v3(y[3], y[4], y[5]);
            const R en = dot(e, n);
            const V3<R> H = (q.pF * en) * n + v3(B[0], B[1], B[2]);
            const V3<R> cTe = (q.cT * en) * cross(n, e);
            const V3<R> mxH = cross(e, H);
            const V3<R> br = cross(cTe + q.d * mxH, n);
            const V3<R> ne = cross((-q.a) * H + q.bpd * mxH + cTe, e);
            a[0] = br.x; a[1] = br.y; a[2] = br.z; a[3] = ne.x; a[4] = ne.y; a[5] = ne.z;
        }
    }
    // .inl:40-170 applied to w = (wA, wB)
    static __device__ __forceinline__ void bdw(const Par& q, const R* y, const Cache&, const R* w, R* r) {
        const V3<R> n = v3(y[0], y[1], y[2]), e = v3(y[3], y[4], y[5]);
        const V3<R> wA = v3(w[0], w[1], w[2]), wB = v3(w[3], w[4], w[5]);
        const V3<R> br = (-q.cF) * cross(n, wA) + q.dDN * (dot(n, e) * wB - dot(n, wB) * e);
        const V3<R> ne = (-q.cFe) * cross(e, wA) + q.bpdDN * (wB - dot(e, wB) * e) + q.aDN * cross(e, wB);
        r[0] = br.x; r[1] = br.y; r[2] = br.z; r[3] = ne.x; r[4] = ne.y; r[5] = ne.z;
    }
    // .inl:179-219
    static __device__ __forceinline__ void drift(const Par& q, const R* y, const Cache&, R* r) {
        const V3<R> n = v3(y[0], y[1], y[2]), e = v3(y[3], y[4], y[5]);
        const V3<R> br = (-q.cF2) * n + q.adDN2 * cross(n, e) - q.hd2DN2 * (dot(e, e) * n - n);
        const V3<R> ne = (-q.ndrift) * e;
        r[0] = br.x; r[1] = br.y; r[2] = br.z; r[3] = ne.x; r[4] = ne.y; r[5] = ne.z;
    }
    static __device__ __forceinline__ void out(const R* y, R* o) {
#pragma unroll
        for (int i = 0; i < 6; ++i) o[i] = y[i];
    }
    struct Trig {};
    static __device__ __forceinline__ void trig(const R*, Trig&) {}
    static __device__ __forceinline__ void out_t(const R* y, R* o, Trig&) { out(y, o); }
    static __device__ __forceinline__ void prepare_t(const Par& q, const Rot<R>& r, R* y, Cache& c, const Trig&) {
        prepare(q, r, y, c);
    }
    // BrownAndNeelRelaxation.h:168-172: n and m normalised separately
    static __device__ __forceinline__ void normalize(R* y) {
#pragma unroll
        for (int h = 0; h < 6; h += 3) {
            const R n2 = (y[h] * y[h] + y[h + 1] * y[h + 1]) + y[h + 2] * y[h + 2];
            if (n2 > R(0)) {
                const R n = M<R>::sqrt(n2);
                y[h] = y[h] / n; y[h + 1] = y[h + 1] / n; y[h + 2] = y[h + 2] / n;
            }
        }
    }
    static __device__ __forceinline__ void newton_matrix(const Par&, const R*, const Cache&, const R*, const R*, R,
                                                         R S[D][D]) {
        for (int i = 0; i < D; ++i) for (int j = 0; j < D; ++j) S[i][j] = R(i == j ? -1 : 0);
    }
};

// ======================================================================= steppers
struct NewtonCount {
    unsigned int iterations, unconverged;
};

// Gaussian elimination with partial pivoting (D <= 3; larger systems here are -I)
template <class R, int D>
__device__ __forceinline__ bool solve_small(R A[D][D], R* b, R* x) {
#pragma unroll
    for (int k = 0; k < D; ++k) {
        int piv = k;
#pragma unroll
        for (int i = k + 1; i < D; ++i)
            if (M<R>::abs(A[i][k]) > M<R>::abs(A[piv][k])) piv = i;
        if (A[piv][k] == R(0)) return false;
        if (piv != k) {
#pragma unroll
            for (int j = 0; j < D; ++j) { const R t = A[k][j]; A[k][j] = A[piv][j]; A[piv][j] = t; }
            const R t = b[k]; b[k] = b[piv]; b[piv] = t;
        }
#pragma unroll
        for (int i = k + 1; i < D; ++i) {
            const R f = A[i][k] / A[k][k];
#pragma unroll
            for (int j = k; j < D; ++j) A[i][j] = A[i][j] - f * A[k][j];
            b[i] = b[i] - f * b[k];
        }
    }
#pragma unroll
    for (int i = D - 1; i >= 0; --i) {
        R s = b[i];
#pragma unroll
        for (int j = i + 1; j < D; ++j) s = s - A[i][j] * x[j];
        x[i] = s / A[i][i];
    }
    return true;
}

// ------------------------------------------------------------ double noise matrix
// Approximate double Stratonovich integrals J(j1, j2) of one step for WeakTest and
// ExplicitStrong_1.0 (DoubleNoiseMatrix.h; Kloeden & Platen 1992, sec. 5.8).  The
// symmetric part is dW_j1 dW_j2 / 2; the antisymmetric part A of each pair
// j1 > j2 is, for order p >= 1,
//   A = -1/(2 pi) sum_{r=1}^{p} 1/r [z1 (sqrt2 dW_j2 - z2) - z3 (sqrt2 dW_j1 - z4)]
//       + rho_p (mu1 dW_j2 - mu2 dW_j1),
// for p = 0 the rho term alone and for p = -1 zero.  As in the reference every
// z and mu is a fresh N(0, dt) draw per pair (its generators advance on every
// call).  Draws come from Philox calls 2, 3, ... of the step: per pair, one block
// of four normals per r (z1..z4), then one block whose first two normals are mu1, mu2.
// Pairs in the reference's loop order: j1 = Mn-1 .. 1, j2 = j1-1 .. 0.
template <int Mn>
__host__ __device__ constexpr int dn_pair(int j1, int j2) {
    return (Mn - 1) * Mn / 2 - j1 * (j1 + 1) / 2 + (j1 - 1 - j2);
}
template <class R, int Mn>
__device__ __forceinline__ void double_noise_antisym(unsigned long long seed, unsigned long long pid,
                                                     unsigned long long step, int p, R rho, R sqdt, const R* w, R* A) {
    const R kSqrt2 = R(1.4142135623730951), kInv2Pi = R(0.15915494309189535);
    uint32_t call = 2u;
#pragma unroll
    for (int j1 = Mn - 1; j1 >= 1; --j1) {
#pragma unroll
        for (int j2 = j1 - 1; j2 >= 0; --j2) {
            R t = R(0);
            if (p >= 1) {
                R s = R(0);
                for (int r = 1; r <= p; ++r) {
                    R z[4];
                    box_muller(philox_block(seed, pid, step, call++), 2, z);
                    const R z1 = z[0] * sqdt, z2 = z[1] * sqdt, z3 = z[2] * sqdt, z4 = z[3] * sqdt;
                    s = s + (R(1) / R(r)) * (z1 * (kSqrt2 * w[j2] - z2) - z3 * (kSqrt2 * w[j1] - z4));
                }
                t = -s * kInv2Pi;
            }
            if (p >= 0) {
                R u[4];
                box_muller(philox_block(seed, pid, step, call++), 1, u);
                t = t + rho * ((u[0] * sqdt) * w[j2] - (u[1] * sqdt) * w[j1]);
            }
            A[dn_pair<Mn>(j1, j2)] = t;
        }
    }
}
// column c of J: v[r] = J(r, c)
template <class R, int Mn>
__device__ __forceinline__ void dn_column(const R* w, const R* A, int c, R* v) {
#pragma unroll
    for (int r = 0; r < Mn; ++r) {
        if (r == c) v[r] = (R(0.5) * w[r]) * w[r];
        else if (r > c) v[r] = (R(0.5) * w[r]) * w[c] + A[dn_pair<Mn>(r, c)];
        else v[r] = (R(0.5) * w[c]) * w[r] - A[dn_pair<Mn>(c, r)];
    }
}

template <class P, class R, int SOLVER>
struct Stepper {
    static constexpr int D = P::D, Mn = P::Mn;
    using Par = typename P::Par;
    using Cache = typename P::Cache;
    using Trig = typename P::Trig;

    static constexpr bool kExplicit = SOLVER == kEulerMaruyama || SOLVER == kHeun ||
                                      SOLVER == kEulerMaruyamaNormalized || SOLVER == kMillstein;

    // y + inc with the update's rounding error carried in lo (Fast2Sum: exact when
    // |y| >= |inc + lo|, which holds for the small increments it is used for)
    static __device__ __forceinline__ void add_compensated(R& y, R& lo, R inc) {
        const R t = inc + lo;
        const R s = y + t;
        lo = t - (s - y);
        y = s;
    }
    // whether component i of the update in chart c keeps its rounding error: in the FP32
    // form the components a problem names (P::compensated), whose per-step increments are
    // only a few ulp (the particle's Brown rotation: rounded plainly, they would pick up a
    // spurious diffusion of several per cent and bias the ensemble mean); lo of the other
    // components is cleared (a rotated chart re-parameterises the angles)
    static __device__ __forceinline__ bool keep_error(const Cache& c, R* lo, int i) {
        if constexpr (!M<R>::kCompensatedState || !(SOLVER == kEulerMaruyama || SOLVER == kHeun || SOLVER == kMillstein)) {
            return false;
        } else {
            if (!lo) return false;
            if (i < P::compensated(c)) return true;
            lo[i] = R(0);
            return false;
        }
    }

    // one explicit step from y already prepared into the chart c by prepare_t; ends with
    // finishCalculations.  lo: the FP32 form's carried rounding errors of y (or nullptr)
    static __device__ __forceinline__ void explicit_from(const Par& q, const Rot<R>& rot, R* y, Cache& c, const R* B,
                                                         const R* w, R dt, R* lo = nullptr) {
        if constexpr (SOLVER == kEulerMaruyama) {
            R a[D], d[D], bw[D];
            P::det(q, y, c, B, a);
            P::drift(q, y, c, d);
            P::bdw(q, y, c, w, bw);
#pragma unroll
            for (int i = 0; i < D; ++i) {
                const R inc = (a[i] + d[i]) * dt + bw[i];
                if (keep_error(c, lo, i)) add_compensated(y[i], lo[i], inc);
                else y[i] = y[i] + inc;
            }
            P::finish(rot, y, c);
        } else if constexpr (SOLVER == kHeun) {
            R a1[D], d[D], bw[D], s[D];
            P::det(q, y, c, B, a1);
            P::drift(q, y, c, d);
            P::bdw(q, y, c, w, bw);
#pragma unroll
            for (int i = 0; i < D; ++i) {
                a1[i] = a1[i] + d[i];
                s[i] = (y[i] + a1[i] * dt) + bw[i];
            }
            P::recompute(q, s, c);  // second stage in the chart chosen for y_n
            R a2[D];
            P::det(q, s, c, B, a2);
            P::drift(q, s, c, d);
#pragma unroll
            for (int i = 0; i < D; ++i) {
                if (keep_error(c, lo, i)) add_compensated(y[i], lo[i], (R(0.5) * ((a2[i] + d[i]) + a1[i])) * dt + bw[i]);
                else y[i] = (y[i] + (R(0.5) * ((a2[i] + d[i]) + a1[i])) * dt) + bw[i];
            }
            P::finish(rot, y, c);
        } else if constexpr (SOLVER == kEulerMaruyamaNormalized) {
            R a[D], d[D], bw[D];
            P::det(q, y, c, B, a);
            P::drift(q, y, c, d);
            P::bdw(q, y, c, w, bw);
#pragma unroll
            for (int i = 0; i < D; ++i) y[i] = y[i] + ((a[i] + d[i]) * dt + bw[i]);
            P::finish(rot, y, c);
            P::normalize(y);
        } else if constexpr (SOLVER == kMillstein) {
            R a[D], d[D], bw[D];
            P::det(q, y, c, B, a);
            P::drift(q, y, c, d);
            P::bdw(q, y, c, w, bw);
            R ww = R(0);
#pragma unroll
            for (int j = 0; j < Mn; ++j) ww = ww + w[j] * w[j];
#pragma unroll
            for (int i = 0; i < D; ++i) {
                if (keep_error(c, lo, i)) add_compensated(y[i], lo[i], (a[i] * dt + bw[i]) + d[i] * ww);
                else y[i] = ((y[i] + a[i] * dt) + bw[i]) + d[i] * ww;
            }
            P::finish(rot, y, c);
        }
    }

    // tr: sines and cosines of y (from the previous step's output), reused by prepare_t
    static __device__ __forceinline__ void step(const Par& q, const Rot<R>& rot, R* y, const R* B, const R* w, R dt,
                                                int max_iter, double tol, NewtonCount& nc, const Trig& tr,
                                                R* lo = nullptr) {
        if constexpr (kExplicit) {
            Cache c;
            P::prepare_t(q, rot, y, c, tr);
            explicit_from(q, rot, y, c, B, w, dt, lo);
        } else {
            if constexpr (P::kHasJacobian) {
                // Newton on f(yj) = finish(prepare((yj+yn)/2) + a dt + b dW) + yn/2 - 3yj/2,
                // accepted when |dy| <= tol, evaluated in FP64 (FP32: tol raised to what
                // the FP32 state can resolve)
                R yn[D], yj[D];
#pragma unroll
                for (int i = 0; i < D; ++i) { yn[i] = y[i]; yj[i] = y[i]; }
                bool conv = false;
                for (int it = 0; it < max_iter; ++it) {
                    R r[D];
#pragma unroll
                    for (int i = 0; i < D; ++i) r[i] = (yj[i] + yn[i]) * R(0.5);
                    Cache c;
                    P::prepare(q, rot, r, c);
                    R a[D], bw[D], S[D][D];
                    P::det(q, r, c, B, a);
                    P::bdw(q, r, c, w, bw);
                    if constexpr (SOLVER == kImplicitMidpointExact) P::newton_matrix_exact(q, r, c, B, w, dt, S);
                    else P::newton_matrix(q, r, c, B, w, dt, S);
#pragma unroll
                    for (int i = 0; i < D; ++i) r[i] = r[i] + (a[i] * dt + bw[i]);
                    P::finish(rot, r, c);
                    R rhs[D], dx[D];
#pragma unroll
                    for (int i = 0; i < D; ++i) rhs[i] = -(r[i] + (yn[i] * R(0.5) - yj[i] * R(1.5)));
                    ++nc.iterations;
                    bool ok;
                    if constexpr (D > 3) {  // S == -I for the coupled Cartesian problem
#pragma unroll
                        for (int i = 0; i < D; ++i) dx[i] = -rhs[i];
                        ok = true;
                    } else {
                        ok = solve_small<R, D>(S, rhs, dx);
                    }
                    if (!ok) break;
                    double n2 = 0.0, y2 = 0.0;
#pragma unroll
                    for (int i = 0; i < D; ++i) {
                        yj[i] = yj[i] + dx[i];
                        n2 += static_cast<double>(dx[i]) * static_cast<double>(dx[i]);
                        y2 += static_cast<double>(yj[i]) * static_cast<double>(yj[i]);
                    }
                    const double tol_eff = (sizeof(R) == 4) ? fmax(tol, 8.0 * 1.1920929e-7 * ::sqrt(y2)) : tol;
                    if (::sqrt(n2) <= tol_eff) { conv = true; break; }
                }
                if (!conv) ++nc.unconverged;
#pragma unroll
                for (int i = 0; i < D; ++i) y[i] = yj[i];
            }
        }
    }

    // Heun_NotConsistent.inl:35-47 (Stratonovich): the support point takes dW, the
    // corrector the average of b at both points times an independent dW2.  Both
    // points are evaluated in the chart prepareCalculations chose for y_n.
    static __device__ __forceinline__ void step_heun_nc(const Par& q, const Rot<R>& rot, R* y, const R* B, const R* w,
                                                        const R* w2, R dt, const Trig& tr) {
        Cache c;
        P::prepare_t(q, rot, y, c, tr);
        R a1[D], d[D], bw[D], s[D], b1[D];
        P::det(q, y, c, B, a1);
        P::drift(q, y, c, d);
        P::bdw(q, y, c, w, bw);
        P::bdw(q, y, c, w2, b1);
#pragma unroll
        for (int i = 0; i < D; ++i) {
            a1[i] = a1[i] + d[i];
            s[i] = (y[i] + a1[i] * dt) + bw[i];
        }
        P::recompute(q, s, c);
        R a2[D], b2[D];
        P::det(q, s, c, B, a2);
        P::drift(q, s, c, d);
        P::bdw(q, s, c, w2, b2);
#pragma unroll
        for (int i = 0; i < D; ++i) y[i] = (y[i] + (R(0.5) * ((a2[i] + d[i]) + a1[i])) * dt) + R(0.5) * (b2[i] + b1[i]);
        P::finish(rot, y, c);
    }

    // b(y) e_j: column j of the noise matrix at the prepared point
    static __device__ __forceinline__ void b_column(const Par& q, const R* y, const Cache& c, int j, R* col) {
        R e[Mn];
#pragma unroll
        for (int k = 0; k < Mn; ++k) e[k] = R(k == j ? 1 : 0);
        P::bdw(q, y, c, e, col);
    }

    // Explicit_Strong_1.inl:20-78: no drift correction; support points
    // Y +- b_j sqrt(dt) around Y = y + a dt for the first D noise columns j, and
    //   y' = Y + b dW + sum_j (b(Y + b_j sqrt dt) - b(Y - b_j sqrt dt)) J(:, j) / sqrt(dt).
    static __device__ __forceinline__ void step_es1(const Par& q, const Rot<R>& rot, R* y, const R* B, const R* w,
                                                    const R* A, R dt, R sqdt, const Trig& tr) {
        Cache c;
        P::prepare_t(q, rot, y, c, tr);
        R a[D], bw[D], t[D], acc[D];
        P::det(q, y, c, B, a);
        P::bdw(q, y, c, w, bw);
#pragma unroll
        for (int i = 0; i < D; ++i) { t[i] = y[i] + a[i] * dt; acc[i] = R(0); }
#pragma unroll
        for (int j = D - 1; j >= 0; --j) {
            R col[D], v[Mn], sp[D], sm[D], bp[D], bm[D];
            b_column(q, y, c, j, col);
            dn_column<R, Mn>(w, A, j, v);
#pragma unroll
            for (int i = 0; i < D; ++i) { sp[i] = t[i] + col[i] * sqdt; sm[i] = t[i] - col[i] * sqdt; }
            Cache cp = c, cm = c;
            P::recompute(q, sp, cp);
            P::recompute(q, sm, cm);
            P::bdw(q, sp, cp, v, bp);
            P::bdw(q, sm, cm, v, bm);
#pragma unroll
            for (int i = 0; i < D; ++i) acc[i] = acc[i] + (bp[i] - bm[i]);
        }
#pragma unroll
        for (int i = 0; i < D; ++i) y[i] = acc[i] / sqdt + (t[i] + bw[i]);
        P::finish(rot, y, c);
    }

    // WeakTest.inl:18-63: as ExplicitStrong_1.0 for the support points, plus the
    // drift at Y + b dW, and a two-stage average:
    //   T = (sum_j [(b(S+_j) - b(S-_j)) J(:, j) / sqrt(dt) + (b(S+_j) + b(S-_j)) dW]) / 4 + b dW / 2
    //   y2 = y + a(Y + b dW) dt/2 + a dt/2 + T;   y' = y + a(y2) dt/2 + a dt/2 + T
    static __device__ __forceinline__ void step_weak(const Par& q, const Rot<R>& rot, R* y, const R* B, const R* w,
                                                     const R* A, R dt, R sqdt, const Trig& tr) {
        Cache c;
        P::prepare_t(q, rot, y, c, tr);
        R a[D], bw[D], adt[D], t[D], acc[D], ys[D], as[D];
        P::det(q, y, c, B, a);
        P::bdw(q, y, c, w, bw);
#pragma unroll
        for (int i = 0; i < D; ++i) {
            adt[i] = a[i] * dt;
            t[i] = y[i] + adt[i];
            ys[i] = t[i] + bw[i];
            acc[i] = R(0);
        }
        {
            Cache cs = c;
            P::recompute(q, ys, cs);
            P::det(q, ys, cs, B, as);
        }
#pragma unroll
        for (int j = D - 1; j >= 0; --j) {
            R col[D], v[Mn], sp[D], sm[D], bpv[D], bmv[D], bpw[D], bmw[D];
            b_column(q, y, c, j, col);
            dn_column<R, Mn>(w, A, j, v);
#pragma unroll
            for (int i = 0; i < D; ++i) { sp[i] = t[i] + col[i] * sqdt; sm[i] = t[i] - col[i] * sqdt; }
            Cache cp = c, cm = c;
            P::recompute(q, sp, cp);
            P::recompute(q, sm, cm);
            P::bdw(q, sp, cp, v, bpv);
            P::bdw(q, sm, cm, v, bmv);
            P::bdw(q, sp, cp, w, bpw);
            P::bdw(q, sm, cm, w, bmw);
#pragma unroll
            for (int i = 0; i < D; ++i) {
                acc[i] = acc[i] + (bpv[i] - bmv[i]) / sqdt;
                acc[i] = acc[i] + (bpw[i] + bmw[i]);
            }
        }
        R y2[D];
#pragma unroll
        for (int i = 0; i < D; ++i) {
            acc[i] = acc[i] / R(4) + R(0.5) * bw[i];
            y2[i] = ((y[i] + (R(0.5) * as[i]) * dt) + R(0.5) * adt[i]) + acc[i];
        }
        R a2[D];
        {
            Cache c2 = c;
            P::recompute(q, y2, c2);
            P::det(q, y2, c2, B, a2);
        }
#pragma unroll
        for (int i = 0; i < D; ++i) y[i] = ((y[i] + (R(0.5) * a2[i]) * dt) + R(0.5) * adt[i]) + acc[i];
        P::finish(rot, y, c);
    }
};

}  // namespace sp
